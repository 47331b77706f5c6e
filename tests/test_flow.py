"""Flow-guided search: the vnlb plugin's mvfw / mvbw MVTools clips.

With motion vectors, the search window of an anchor in candidate frame f is
centred where the anchor's position lands after walking the vectors frame by
frame from the anchor frame to f (MVToolsFlowProvider::center_for,
src/flow/flow.hpp:341-389); everything else is the plain path.

CPU: the C restatement against the compiled reference (when built here) and
against the committed outputs of the reference's flow-guided chain
(tests/golden/flow_outputs.npz).
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import mvtools_blobs as M
import oracle as O

GOLDEN = Path(__file__).resolve().parent / "golden" / "flow_outputs.npz"
CASE_IDS = [c[0] for c in M.FLOW_CASES]


def params_of(case):
    name, w, h, f, planes, sigma, seed, kw, fw_spec, bw_spec = case
    return O.cpu_params(O.BASIC, sigma, **kw), O.cpu_params(O.FINAL, sigma, **kw)


def oracle_chain(o, case):
    noisy, fw, bw = M.flow_case(*case)
    flow = (M.flow_grids(fw), M.flow_grids(bw))
    bp, fp = params_of(case)
    bs = o.stage_stacks(O.BASIC, bp, noisy, flow=flow)
    basic = o.aggregate(bs, noisy, bp.search_bwd, bp.search_fwd, bp.patch_time)
    fs = o.stage_stacks(O.FINAL, fp, noisy, basic, flow=flow)
    return basic, o.aggregate(fs, noisy, fp.search_bwd, fp.search_fwd, fp.patch_time)


@pytest.fixture(scope="module")
def golden_flow():
    return np.load(GOLDEN)


@pytest.mark.parametrize("case", M.FLOW_CASES, ids=CASE_IDS)
def test_restatement_matches_reference_flow_outputs(case, golden_flow):
    basic, final = oracle_chain(O.Oracle("port"), case)
    assert np.array_equal(basic, golden_flow[f"{case[0]}/basic"])
    assert np.array_equal(final, golden_flow[f"{case[0]}/final"])


@pytest.mark.skipif(not O.REF_LIB.exists(), reason="reference build absent (make -C oracle ref)")
def test_restatement_matches_reference_build_live():
    rng = np.random.default_rng(31)
    import synth
    for planes, pel, overlap, reach in ((1, 1, 0, 3), (3, 2, 2, 7), (1, 4, 4, 20)):
        _, noisy = synth.make_clip(40, 32, 5, planes, 20.0, seed=int(rng.integers(1 << 30)))
        fw = M.random_direction(rng, 5, 40, 32, 8, overlap, pel, False, reach, unusable=0.4)
        bw = M.random_direction(rng, 5, 40, 32, 8, overlap, pel, True, reach, unusable=0.4)
        for flow in ((M.flow_grids(fw), None), (None, M.flow_grids(bw)), (M.flow_grids(fw), M.flow_grids(bw))):
            bp = O.cpu_params(O.BASIC, 20.0, radius=2, block_step=4, bm_range=4)
            a = O.Oracle("ref").stage_stacks(O.BASIC, bp, noisy, flow=flow, threads=4)
            b = O.Oracle("port").stage_stacks(O.BASIC, bp, noisy, flow=flow, threads=4)
            assert np.array_equal(a, b)


def test_flow_moves_the_windows():
    """Not vacuous: the vectors change the result, and all-unusable grids do
    not (the centre stays on the anchor)."""
    case = M.FLOW_CASES[0]
    noisy, fw, bw = M.flow_case(*case)
    bp, _ = params_of(case)
    o = O.Oracle("port")
    plain = o.stage_stacks(O.BASIC, bp, noisy)
    moved = o.stage_stacks(O.BASIC, bp, noisy, flow=(M.flow_grids(fw), M.flow_grids(bw)))
    assert not np.array_equal(plain, moved)
    dead = M.Direction(fw.block_size, fw.overlap, fw.pel, False, fw.vectors, np.zeros_like(fw.valid),
                       np.zeros_like(fw.scene))
    still = o.stage_stacks(O.BASIC, bp, noisy, flow=(M.flow_grids(dead), None))
    assert np.array_equal(plain, still)
