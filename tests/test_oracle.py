"""The CPU oracle, pinned against the reference's own fixtures and build.

* The C restatement (oracle/vnlb_oracle.c) equals the reference CPU core
  compiled out of tree (oracle/_ref) bit for bit, on the committed golden
  outputs and (when the reference build is present) on fresh cases.
* The oracle reproduces the reference's end-to-end fixtures made by the
  original pariasm/vnlb (tests/reference_cases, compare_reference.py
  parameters) within the reference's own tolerance.
* Unit behaviour from tests/cpp/test_core.cpp: constant videos reproduce the
  constant, parameter validation messages.
"""
import json
from pathlib import Path

import numpy as np
import pytest

import oracle as O
import synth

ROOT = Path(__file__).resolve().parents[1]


def _chain_params(meta, sigma):
    bp = O.cpu_params(O.BASIC, sigma, **meta["shared"], **meta["basic"])
    fp = O.cpu_params(O.FINAL, sigma, **meta["shared"], **meta["final"])
    return bp, fp


def test_port_equals_reference_golden(golden):
    data, meta = golden
    port = O.Oracle("port")
    for name, m in meta.items():
        noisy = data[f"{name}/noisy"]
        bp, fp = _chain_params(m, m["sigma"])
        basic, final = port.chain(noisy, bp, fp)
        assert np.array_equal(basic, data[f"{name}/basic"]), name
        assert np.array_equal(final, data[f"{name}/final"]), name


@pytest.mark.skipif(not O.REF_LIB.exists(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("planes,kw", [
    (1, {}),
    (3, dict(block_size=7, patch_time=2, bm_range=5, group_size=16, rank=15, block_step=3)),
    (3, dict(chroma=0, group_size=12, rank=10)),
    (1, dict(block_size=4, patch_time=2, bm_range=3, radius=6, group_size=40, rank=16, beta=3.0, block_step=2)),
    (3, dict(cap_factor=0.0, tau=900.0)),
    (3, dict(weight_alpha=0.0, weight_beta=0.0, weight_gamma=0.0)),
    (3, dict(chroma=0, block_size=7, patch_time=2, block_step=3, bm_range=4, group_size=16, rank=8)),
    (1, dict(block_size=10, patch_time=2, block_step=5, bm_range=4, group_size=16, rank=15)),
    (1, dict(patch_time=2, radius=2, block_step=4, bm_range=4, group_size=16, rank=16, tau=400.0)),
    (3, dict(model_cap_factor=2.0, cap_factor=4.0, tau=600.0, group_size=8, rank=8)),
])
def test_port_equals_reference_build(planes, kw):
    _, noisy = synth.make_clip(56, 40, 4, planes, 18.0, seed=21)
    bp = O.cpu_params(O.BASIC, 18.0, **kw)
    fp = O.cpu_params(O.FINAL, 18.0, **kw)
    b0, f0 = O.Oracle("ref").chain(noisy, bp, fp)
    b1, f1 = O.Oracle("port").chain(noisy, bp, fp)
    assert np.array_equal(b0, b1)
    assert np.array_equal(f0, f1)


def test_reference_cases_within_reference_tolerance():
    """tests/compare_reference.py semantics on the pariasm/vnlb fixtures."""
    data = np.load(ROOT / "tests" / "golden" / "reference_cases.npz")
    meta = json.loads(str(data["meta"]))
    assert len(meta) == 6
    port = O.Oracle("port")
    for name, m in meta.items():
        v = m["vnlb"]
        sigma = float(m["noise"]["sigma_8bit"])
        common = dict(block_size=int(v["block_size"]), patch_time=int(v["patch_time"]), bm_range=int(v["bm_range"]),
                      radius=int(v["radius"]), group_size=int(v["group_size"]), rank=int(v["rank"]),
                      beta=float(v["beta"]), block_step=max(1, int(v["block_size"]) // 2),
                      weight_alpha=0.0, weight_beta=0.0, weight_gamma=0.0)
        bp = O.cpu_params(O.BASIC, sigma, tau=0.0, variance_threshold=float(v["basic_variance_threshold"]), **common)
        fp = O.cpu_params(O.FINAL, sigma, tau=float(v["final_tau_8bit"]),
                          variance_threshold=float(v["final_variance_threshold"]), flat_areas=1, sigma_basic=0.0,
                          **common)
        noisy = data[f"{name}/noisy"][:, None]
        basic, final = port.chain(noisy, bp, fp)
        tol = m["tolerance"]
        for stage, got, want in (("basic", basic[:, 0], data[f"{name}/basic"]),
                                 ("final", final[:, 0], data[f"{name}/final"])):
            diff = np.abs(got - want)
            assert diff.max() <= tol["max_abs"], (name, stage, diff.max())
            assert diff.mean() <= tol["mean_abs"], (name, stage, diff.mean())
            assert np.sqrt(np.mean(diff ** 2)) <= tol["rmse"], (name, stage)


@pytest.mark.parametrize("planes", [1, 3])
def test_constant_video_reproduces_constant(planes):
    """tests/cpp/test_core.cpp:247-356: constant input -> constant output."""
    clip = np.full((4, planes, 40, 48), 0.375, np.float32)
    bp = O.cpu_params(O.BASIC, 10.0)
    fp = O.cpu_params(O.FINAL, 10.0)
    basic, final = O.Oracle("port").chain(clip, bp, fp)
    assert np.allclose(basic, 0.375, atol=1e-6)
    assert np.allclose(final, 0.375, atol=1e-6)


@pytest.mark.parametrize("kw,message", [
    (dict(rank=9), "group_size must cover the effective VNLB rank"),
    (dict(cap_factor=0.5), "cap_factor must be zero or at least 1.0"),
    (dict(block_size=100), "block_size must fit inside the frame"),
    (dict(beta=0.0), "beta must be finite and positive"),
    (dict(block_step=-1), "block_step must be non-negative"),
])
def test_validation_messages(kw, message):
    clip = np.zeros((3, 1, 32, 32), np.float32)
    p = O.cpu_params(O.BASIC, 10.0, **kw)
    with pytest.raises(ValueError, match=message):
        O.Oracle("port").stage_stacks(O.BASIC, p, clip)


def test_matches_are_sorted_and_capped():
    _, noisy = synth.make_clip(48, 40, 4, 1, 25.0, seed=5)
    p = O.cpu_params(O.FINAL, 25.0, tau=4000.0, cap_factor=2.0)
    stack, groups, rows = O.anchor_groups(O.FINAL, p, noisy, noisy, 1)
    assert groups
    cap = 16
    for x, y, s, first in groups:
        assert 8 <= s <= cap
        d = rows["distance"][first:first + s]
        assert np.all(np.diff(d[:8]) >= 0)  # the K nearest lead, ascending
        assert d[0] == 0.0 and rows["x"][first] == x and rows["y"][first] == y
