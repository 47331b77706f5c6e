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

import struct
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


# ---------------------------------------------------------------- parsers (host code of the native library)
def lib_or_skip():
    import vnlbgpu_lib as lib
    try:
        lib.load()
    except Exception as error:  # the library is not built
        pytest.skip(str(error))
    return lib


def test_parse_analysis_fields():
    lib = lib_or_skip()
    d = M.Direction(16, 4, 2, True, np.zeros((1, 3, 5, 2), np.int32), np.ones(1, bool), np.zeros(1, bool))
    a = lib.parse_mvtools_analysis(M.analysis_blob(d, 64, 48, delta=1, levels=3))
    assert (a.block_size_x, a.block_size_y, a.pel, a.level_count, a.delta_frame, a.backwards) == (16, 16, 2, 3, 1, 1)
    assert (a.width, a.height, a.overlap_x, a.overlap_y, a.block_count_x, a.block_count_y) == (64, 48, 4, 4, 5, 3)
    assert lib.parse_mvtools_analysis(M.analysis_blob(d, 64, 48, delta=-1)).delta_frame == -1


@pytest.mark.parametrize("field,value,message", [
    (None, None, "must contain 21 32-bit fields"),
    (2, 0, "invalid MVTools horizontal block size"),
    (4, 0, "invalid MVTools pel"),
    (12, 16, "overlap must be smaller than block size"),
    (14, 0, "invalid MVTools horizontal block count"),
])
def test_parse_analysis_errors(field, value, message):
    lib = lib_or_skip()
    d = M.Direction(16, 4, 2, False, np.zeros((1, 3, 5, 2), np.int32), np.ones(1, bool), np.zeros(1, bool))
    blob = M.analysis_blob(d, 64, 48)
    blob = blob[:-4] if field is None else blob[:4 * field] + struct.pack("<I", value) + blob[4 * field + 4:]
    with pytest.raises(lib.VNLBError, match=message):
        lib.parse_mvtools_analysis(blob)


def test_parse_vectors_takes_the_finest_level():
    lib = lib_or_skip()
    rng = np.random.default_rng(3)
    v = rng.integers(-50, 50, (3, 5, 2)).astype(np.int32)
    d = M.Direction(16, 4, 2, False, v[None], np.ones(1, bool), np.zeros(1, bool))
    a = lib.parse_mvtools_analysis(M.analysis_blob(d, 64, 48))
    for coarse in (0, 1, 3):
        valid, xy = lib.parse_mvtools_vectors(M.vectors_blob(v, True, coarse), a)
        assert valid and np.array_equal(xy.reshape(3, 5, 2), v)
    valid, xy = lib.parse_mvtools_vectors(M.vectors_blob(v, False), a)
    assert not valid and len(xy) == 0


def bad_vectors(kind: str) -> bytes:
    """A malformed MVTools_vectors property for a 5 x 3 block grid."""
    v = np.zeros((3, 5, 2), np.int32)
    b = M.vectors_blob(v, True, 1)
    if kind == "too small":
        return b[:4]
    if kind == "size header":
        return struct.pack("<I", len(b) + 4) + b[4:]
    if kind == "count":  # a finest level of 10 vectors for 15 blocks
        return M.vectors_blob(np.zeros((2, 5, 2), np.int32), True, 1)
    if kind == "truncated level header":
        return struct.pack("<I", len(b) + 2) + b[4:] + b"\0\0"
    if kind == "level past the end":
        return b[:8] + struct.pack("<I", len(b)) + b[12:]
    if kind == "level shorter than its header":
        return struct.pack("<I", len(b) + 4) + b[4:] + struct.pack("<I", 2)
    if kind == "finest level size":
        return struct.pack("<I", len(b) + 12) + b[4:] + struct.pack("<I", 12) + b"\0" * 8
    raise ValueError(kind)


@pytest.mark.parametrize("kind,message", [
    ("too small", "MVTools_vectors is too small"),
    ("size header", "MVTools_vectors size header is invalid"),
    ("count", "finest level vector count does not match analysis data"),
    ("truncated level header", "truncated MVTools level header"),
    ("level past the end", "invalid MVTools level size"),
    ("level shorter than its header", "invalid MVTools level size"),
    ("finest level size", "finest level has invalid vector size"),
])
def test_parse_vectors_errors(kind, message):
    lib = lib_or_skip()
    d = M.Direction(16, 4, 2, False, np.zeros((1, 3, 5, 2), np.int32), np.ones(1, bool), np.zeros(1, bool))
    a = lib.parse_mvtools_analysis(M.analysis_blob(d, 64, 48))
    with pytest.raises(lib.VNLBError, match=message):
        lib.parse_mvtools_vectors(bad_vectors(kind), a)


# ---------------------------------------------------------------- the GPU path
def gpu_chain(case):
    import vnlb
    name, w, h, f, planes, sigma, seed, kw, fw_spec, bw_spec = case
    noisy, fw, bw = M.flow_case(*case)
    flow = dict(mvfw=M.props(fw, w, h) if fw else None, mvbw=M.props(bw, w, h) if bw else None,
                clip_props=M.clip_props(fw, bw, f))
    layout = dict(radius=kw.get("radius", 1), patch_time=kw.get("patch_time", 1))  # the stacks' slots
    stacks = vnlb.Basic(noisy, sigma=sigma, **kw, **flow)
    basic = vnlb.Aggregate(stacks, src=noisy, **layout)
    stacks = vnlb.Final(noisy, ref=basic, sigma=sigma, **kw, **flow)
    return basic, vnlb.Aggregate(stacks, src=noisy, **layout)


@pytest.mark.gpu
@pytest.mark.parametrize("case", M.FLOW_CASES, ids=CASE_IDS)
def test_gpu_chain_with_flow_bit_exact(case, golden_flow):
    basic, final = gpu_chain(case)
    assert np.array_equal(basic, golden_flow[f"{case[0]}/basic"])
    assert np.array_equal(final, golden_flow[f"{case[0]}/final"])


@pytest.mark.gpu
def test_gpu_flow_checks_the_clips():
    import vnlb
    import vnlbgpu_lib as lib
    case = M.FLOW_CASES[0]
    name, w, h, f, planes, sigma, seed, kw, fw_spec, bw_spec = case
    noisy, fw, bw = M.flow_case(*case)
    with pytest.raises(lib.VNLBError, match="mvfw analysis dimensions must match clip"):
        vnlb.Basic(noisy, sigma=sigma, mvfw=M.props(fw, w + 8, h), **kw)
    with pytest.raises(lib.VNLBError, match="mvfw must be generated with isb=False"):
        vnlb.Basic(noisy, sigma=sigma, mvfw=M.props(bw, w, h), **kw)
    with pytest.raises(lib.VNLBError, match="mvbw frame count must match clip"):
        vnlb.Basic(noisy, sigma=sigma, mvbw=M.props(bw, w, h)[:-1], **kw)
    bad = M.props(fw, w, h)
    bad[0] = dict(bad[0], MVTools_MVAnalysisData=M.analysis_blob(fw, w, h, delta=2))
    with pytest.raises(lib.VNLBError, match="must use MVTools delta=1 vectors"):
        vnlb.Basic(noisy, sigma=sigma, mvfw=bad, **kw)
