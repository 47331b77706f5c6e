"""The FP64 network oracle (oracle/mlp_fp64.py) checks itself: its analytical
gradients against central finite differences, on the CPU.  The GPU kernels'
gradients are then checked against this oracle (tests/test_learned.py)."""
import numpy as np

import mlp_fp64 as M


def test_analytical_gradients_match_finite_differences():
    rng = np.random.default_rng(3)
    shape = (7, 9, 2, 11)  # inputs, hidden, layers, outputs
    n = sum((shape[0] if l == 0 else shape[1]) * (shape[3] if l == shape[2] else shape[1]) +
            (shape[3] if l == shape[2] else shape[1]) for l in range(shape[2] + 1))
    flat = rng.normal(0.0, 0.5, n)
    x = rng.normal(0.0, 1.0, (5, shape[0]))
    targets = rng.integers(-1, shape[3], (5, 3))
    targets[:, 0] = np.abs(targets[:, 0])  # every row has a target
    _, g = M.loss_and_gradients(flat, shape, x, targets, round_weights=False)
    idx = rng.choice(n, 40, replace=False)
    num = M.numeric_gradients(flat, shape, x, targets, idx)
    assert np.allclose(g[idx], num, rtol=1e-5, atol=1e-8)


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, -2.5, 3.0e-39], np.float32)
    got = M.bf16(x)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: even (1.0); 1 + 1.5 * 2^-8 rounds up
    assert got[0] == 1.0 and got[1] == 1.0 and got[2] == 1.0078125 and got[3] == -2.5
