"""vnlbcu's own defaults at full size: 1920x1080 YUV444PS with block 7,
automatic step 3, group 16, bm_range 13, patch_time 2 and rank 15 (about 230k
groups of up to 64 retained rows of dimension 294 per anchor frame,
cuda_plugin.cpp:380-403).  A Basic and a Final session are alive together, as
in a script that chains them; each takes as many pipeline lanes as half of
the free device memory holds.  The oracle cannot run this size in seconds,
so the checks are size-independent: the outputs are finite, Final is not
worse than Basic, Basic beats the noisy clip, and re-rendering reproduces the
same bits.  Parity of these parameters against the oracle is pinned at small
sizes in test_gpu_parity.py (test_vnlbcu_defaults_match_oracle)."""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "vapoursynth-vnlb_b200"))

import synth  # noqa: E402


@pytest.mark.gpu
def test_vnlbcu_defaults_1080p_yuv_basic_and_final():
    import vnlbcu
    import vnlbgpu_lib as lib

    w, h, frames, planes, sigma = 1920, 1080, 4, 3, 20.0
    clean, noisy = synth.make_clip(w, h, frames, planes, sigma, seed=3)
    bp = vnlbcu.parse_parameters(lib.STAGE_BASIC, noisy, sigma, {})
    fp = vnlbcu.parse_parameters(lib.STAGE_FINAL, noisy, sigma, {})
    assert (bp.patch_size, bp.patch_time, bp.similar, bp.rank, bp.search_window) == (7, 2, 16, 15, 27)
    sb = lib.Session(bp, w, h, frames, planes)
    sf = lib.Session(fp, w, h, frames, planes)
    try:
        sb.set_clip(lib.SOURCE_CLIP, noisy)
        basic = sb.render_clip()
        sf.set_clip(lib.SOURCE_CLIP, noisy)
        sf.set_clip(lib.SOURCE_REF, basic)
        final = sf.render_clip()
        lanes = (sb.stats()["pipeline_lanes"], sf.stats()["pipeline_lanes"])
        assert all(1 <= n <= 4 for n in lanes), lanes
        assert np.isfinite(basic).all() and np.isfinite(final).all()
        p_noisy, p_basic, p_final = (synth.psnr(x, clean) for x in (noisy, basic, final))
        # 16 samples in dimension 294 leave noise eigenvalues near sigma^2 D / B,
        # far above the shrinkage threshold: a small but positive gain
        assert p_basic > p_noisy + 0.05, (p_noisy, p_basic)
        assert p_final >= p_basic - 0.05, (p_basic, p_final)
        # a second render of one frame after the cache is dropped (re-upload)
        sb.set_clip(lib.SOURCE_CLIP, noisy)
        assert np.array_equal(sb.render_frame(2), basic[2])
    finally:
        sb.close()
        sf.close()


@pytest.mark.gpu
@pytest.mark.timeout(1500)
def test_vnlbcu_defaults_full_width_band_bit_exact():
    """vnlbcu's defaults on a full-width band (1920x136 YUV444PS, 4 frames:
    three anchor frames with patch_time 2, 640 x 45 grid anchors each with
    groups of up to 64 rows of dimension 294): Basic and Final of the plain
    form equal the reference CPU core's (oracle/_ref, or the C restatement
    when that build is absent) bit for bit, every frame."""
    import os

    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    import vnlbcu
    import vnlbgpu_lib as lib

    _, noisy = synth.make_clip(1920, 136, 4, 3, 20.0, seed=5)
    basic = vnlbcu.Basic(noisy, sigma=20.0)
    final = vnlbcu.Final(noisy, ref=basic, sigma=20.0)
    pb = vnlbcu.parse_parameters(lib.STAGE_BASIC, noisy, 20.0, {})
    pf = vnlbcu.parse_parameters(lib.STAGE_FINAL, noisy, 20.0, {})
    to_stage = lambda p: O.StageParams(**{f: getattr(p, f) for f in O.StageParams.__dataclass_fields__})
    kind = "ref" if O.REF_LIB.exists() else "port"
    o = O.Oracle(kind)
    threads = os.cpu_count()
    ob = o.aggregate(o.stage_stacks(O.BASIC, to_stage(pb), noisy, threads=threads), noisy, pb.search_bwd,
                     pb.search_fwd, pb.patch_time)
    of = o.aggregate(o.stage_stacks(O.FINAL, to_stage(pf), noisy, ob, threads=threads), noisy, pf.search_bwd,
                     pf.search_fwd, pf.patch_time)
    bits = lambda a: np.ascontiguousarray(a, np.float32).view(np.uint32)
    for name, g, r in (("basic", basic, ob), ("final", final, of)):
        diff = np.flatnonzero(bits(g) != bits(r))
        assert diff.size == 0, (name, kind, diff.size, float(np.max(np.abs(g - r))))
