"""Host logic without a GPU: the C ABI library exports what include/*.h
declares, the plugin argument rules of vnlbcu (src/vs/cuda_plugin.cpp:370-807)
and vnlb (src/vs/plugin.cpp:236-449, src/core/core.cpp:1948-2024), and the
synthetic workload generator."""
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

import synth
import vnlb
import vnlbcu
import vnlbgpu_lib as lib

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    names = set()
    for header in (ROOT / "include").glob("*.h"):
        text = header.read_text()
        names |= set(re.findall(r"^\s*(?:const\s+)?[\w\s\*]+?\b(vnlbgpu_\w+)\s*\(", text, re.M))
    return names


def test_library_exports_every_declared_symbol():
    assert lib.LIB_PATH.exists(), "run vapoursynth-vnlb_b200/build_native.py"
    out = subprocess.run(["nm", "-D", "--defined-only", str(lib.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    declared = declared_functions()
    assert len(declared) >= 17
    missing = declared - exported
    assert not missing, missing
    assert set(lib.EXPORTS) <= exported


def test_library_loads_without_device():
    handle = lib.load()
    for name in lib.EXPORTS:
        assert hasattr(handle, name)


def _yuv(frames=16, h=1080, w=1920):
    return np.empty((frames, 3, h, w), np.float32)


def test_vnlbcu_defaults_yuv():
    p = vnlbcu.parse_parameters(lib.STAGE_BASIC, _yuv(), 20.0, {})
    assert (p.patch_size, p.patch_time, p.search_window, p.search_bwd, p.search_fwd) == (7, 2, 27, 1, 1)
    assert (p.similar, p.rank, p.proc_step) == (16, 15, 3)
    assert p.variance_threshold == pytest.approx(2.7)
    assert p.sigma == np.float32(20.0) / np.float32(255.0)
    f = vnlbcu.parse_parameters(lib.STAGE_FINAL, _yuv(), 20.0, {})
    assert f.tau == pytest.approx(400.0 / 65025.0)
    assert f.flat_areas == 1 and f.weight_alpha == 1.0 and f.weight_beta == 0.5
    assert f.variance_threshold == pytest.approx(1.2)


def test_vnlbcu_defaults_gray_and_clamps():
    p = vnlbcu.parse_parameters(lib.STAGE_BASIC, np.empty((1, 1, 64, 64), np.float32), 10.0, {})
    assert (p.patch_size, p.patch_time, p.search_bwd) == (10, 1, 0)
    assert p.variance_threshold == pytest.approx(3.7)
    f = vnlbcu.parse_parameters(lib.STAGE_FINAL, np.empty((3, 1, 64, 64), np.float32), 10.0, {})
    assert f.variance_threshold == pytest.approx(1.87 - 0.028 * 10, abs=1e-6)
    # defaults clamp to the candidate count of a tiny clip (cuda_plugin.cpp:508-534)
    tiny = np.empty((1, 1, 12, 12), np.float32)
    t = vnlbcu.parse_parameters(lib.STAGE_BASIC, tiny, 10.0, dict(block_size=8, bm_range=1))
    assert t.similar == 9 and t.rank == 9


@pytest.mark.parametrize("args,message", [
    (dict(radius=-1), "radius must be non-negative"),
    (dict(bm_range=-2), "bm_range must be non-negative"),
    (dict(model_cap_factor=2.0), "requires model_cap_factor=1"),
    (dict(chroma=0), "requires chroma=1"),
    (dict(num_streams=0), "num_streams must be in the range 1..32"),
    (dict(chunk_size=0), "chunk_size must be positive"),
    (dict(group_size=200), "at most 128 model samples"),
    (dict(group_size=8, rank=9), "rank must not exceed min"),
    (dict(block_size=2, patch_time=1, group_size=16, rank=2), "dual-PCA path"),
    (dict(cap_factor=0.5), "cap_factor must be zero or at least 1.0"),
])
def test_vnlbcu_validation_messages(args, message):
    with pytest.raises(lib.VNLBError, match=message):
        vnlbcu.parse_parameters(lib.STAGE_BASIC, _yuv(4, 64, 64), 20.0, args)


def test_vnlbcu_requires_sigma_and_format():
    with pytest.raises(lib.VNLBError, match="missing required argument: sigma"):
        vnlbcu.parse_parameters(lib.STAGE_BASIC, _yuv(4, 64, 64), None, {})
    with pytest.raises(lib.VNLBError, match="only constant GrayS and YUV444PS"):
        vnlbcu.Basic(np.zeros((4, 2, 16, 16), np.float32), sigma=10.0)
    with pytest.raises(lib.VNLBError, match="ref clip properties must match"):
        vnlbcu.Final(np.zeros((4, 1, 16, 16), np.float32), ref=np.zeros((3, 1, 16, 16), np.float32), sigma=1.0)


def test_vnlb_stage_parameters():
    b = vnlb.parse_stage_parameters(lib.STAGE_BASIC, 10.0, {})
    assert (b["patch_size"], b["proc_step"], b["similar"], b["search_window"], b["rank"]) == (8, 8, 8, 19, 8)
    f = vnlb.parse_stage_parameters(lib.STAGE_FINAL, 10.0, dict(radius=2, tau=100.0, sigma_basic=5.0))
    assert f["search_bwd"] == f["search_fwd"] == 2
    assert f["tau"] == np.float32(100.0) / np.float32(65025.0)
    assert f["variance_threshold"] == np.float32(1.7) and f["flat_areas"] == 1
    assert f["sigma_basic"] == np.float32(5.0) / np.float32(255.0)
    with pytest.raises(lib.VNLBError, match="radius must be non-negative"):
        vnlb.parse_stage_parameters(lib.STAGE_BASIC, 10.0, dict(radius=-3))
    with pytest.raises(lib.VNLBError, match="group_size must cover the effective VNLB rank"):
        vnlb.validate_stage_configuration(vnlb.parse_stage_parameters(lib.STAGE_BASIC, 10.0, dict(rank=9)),
                                          np.empty((3, 1, 32, 32), np.float32))


def test_vnlb_aggregate_layout_checks():
    src = np.zeros((3, 1, 8, 8), np.float32)
    with pytest.raises(lib.VNLBError, match="contribution stack layout does not match"):
        vnlb.Aggregate(np.zeros((3, 1, 8, 8), np.float32), src=src)


def test_synth_is_seeded_and_shaped():
    c1, n1 = synth.make_clip(40, 24, 3, 3, 20.0, seed=4)
    c2, n2 = synth.make_clip(40, 24, 3, 3, 20.0, seed=4)
    _, n3 = synth.make_clip(40, 24, 3, 3, 20.0, seed=5)
    assert n1.shape == (3, 3, 24, 40) and n1.dtype == np.float32
    assert np.array_equal(n1, n2) and not np.array_equal(n1, n3)
    assert 0.0 <= c1.min() and c1.max() <= 1.0
    noise = (n1 - c1).std()
    assert noise == pytest.approx(20.0 / 255.0, rel=0.1)
    assert synth.psnr(c1, c1) == float("inf")
