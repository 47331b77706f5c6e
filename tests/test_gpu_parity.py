"""GPU parity: the plain B200 path against the CPU oracle, through the C ABI.

The bar is bit-exactness (the reference's own CUDA matcher test is bit-exact
too, tests/cpp/test_cuda_block_match.cpp:640-672): the retained rows of every
grid anchor, the paste-mask active set, the aggregation weights, the
contribution stacks and the aggregated Basic/Final frames must equal the
oracle's float for float.  Sizes are small enough for the oracle to finish in
seconds, except one full-size (1920x1080 YUV444PS) check on three anchor
frames.
"""
import threading

import numpy as np
import pytest

import oracle as O
import synth
import vnlb
import vnlbcu
import vnlbgpu_lib as lib

pytestmark = pytest.mark.gpu


def session_for(stage, p: O.StageParams, clip, basic=None):
    d = {f: getattr(p, f) for f in p.__dataclass_fields__}
    params = lib.Params(stage=stage, device_id=0, num_streams=1, chunk_size=768,
                        **{k: (float(v) if isinstance(v, (float, np.floating)) else int(v)) for k, v in d.items()})
    frames, planes, h, w = clip.shape
    s = lib.Session(params, w, h, frames, planes)
    s.set_clip(lib.SOURCE_CLIP, clip)
    if stage == lib.STAGE_FINAL:
        s.set_clip(lib.SOURCE_REF, basic)
    return s


def vnlb_kwargs(p: O.StageParams, stage):
    kw = dict(sigma=float(np.float32(p.sigma) * np.float32(255.0)), block_size=p.patch_size,
              patch_time=p.patch_time, bm_range=(p.search_window - 1) // 2, search_bwd=p.search_bwd,
              search_fwd=p.search_fwd, group_size=p.similar, rank=p.rank, cap_factor=p.similar_cap_factor,
              beta=p.beta, tau=float(np.float32(p.tau) * np.float32(65025.0)),
              variance_threshold=p.variance_threshold, weight_alpha=p.weight_alpha, weight_beta=p.weight_beta,
              weight_gamma=p.weight_gamma, block_step=p.proc_step, model_cap_factor=p.model_cap_factor,
              chroma=p.couple_channels)
    if stage == lib.STAGE_FINAL:
        kw.update(flat_areas=p.flat_areas, gamma=p.gamma)
    return kw


def gpu_chain(noisy, bp, fp):
    bs = vnlb.Basic(noisy, **vnlb_kwargs(bp, 0))
    basic = vnlb.Aggregate(bs, src=noisy, patch_time=bp.patch_time, search_bwd=bp.search_bwd,
                           search_fwd=bp.search_fwd)
    fs = vnlb.Final(noisy, ref=basic, **vnlb_kwargs(fp, 1))
    final = vnlb.Aggregate(fs, src=noisy, patch_time=fp.patch_time, search_bwd=fp.search_bwd,
                           search_fwd=fp.search_fwd)
    return bs, basic, fs, final


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.int32)


def test_golden_reference_outputs(golden):
    """Committed outputs of the reference CPU core (tests/golden/ref_outputs.npz)."""
    data, meta = golden
    for name, m in meta.items():
        noisy = data[f"{name}/noisy"]
        bp = O.cpu_params(O.BASIC, m["sigma"], **m["shared"], **m["basic"])
        fp = O.cpu_params(O.FINAL, m["sigma"], **m["shared"], **m["final"])
        _, basic, _, final = gpu_chain(noisy, bp, fp)
        assert np.array_equal(bits(basic), bits(data[f"{name}/basic"])), name
        assert np.array_equal(bits(final), bits(data[f"{name}/final"])), name


CASES = [
    ("gray_defaults", 64, 48, 4, 1, 20.0, {}),
    # a row pitch that is not a multiple of 16 bytes: the matcher stages its
    # regions with plain loads instead of tensor-memory-accelerator tiles
    ("yuv_odd_width", 66, 50, 4, 3, 20.0, {}),
    ("yuv_defaults", 96, 80, 5, 3, 20.0, {}),
    ("yuv_cuda_like", 96, 72, 4, 3, 20.0, dict(block_size=7, patch_time=2, bm_range=6, group_size=16, rank=15,
                                               block_step=3)),
    ("gray_k32_tau", 80, 64, 4, 1, 30.0, dict(group_size=32, rank=20, tau=1500.0, cap_factor=2.0,
                                              block_step=5)),
    ("yuv_no_weights", 72, 56, 3, 3, 12.0, dict(weight_alpha=0.0, weight_beta=0.0, weight_gamma=0.0)),
    ("yuv_alpha_only", 72, 56, 3, 3, 12.0, dict(weight_beta=0.0, cap_factor=0.0)),
    # model rows beyond group_size (vnlb.* semantics: model_cap_factor 0 or >= 1)
    ("yuv_model_cap2_tau", 96, 72, 4, 3, 20.0, dict(tau=800.0, model_cap_factor=2.0)),
    ("gray_model_cap0", 80, 64, 4, 1, 25.0, dict(group_size=12, rank=10, tau=1500.0, cap_factor=3.0,
                                                 model_cap_factor=0.0)),
    # uncoupled planes (chroma=0): one model per plane, weights combined over the planes
    ("yuv_uncoupled", 96, 72, 4, 3, 20.0, dict(chroma=0)),
    ("yuv_uncoupled_tau", 80, 64, 4, 3, 25.0, dict(chroma=0, tau=800.0, group_size=12, rank=10)),
    # covariance models: dimension below 64 (core.cpp:656-658)
    ("gray_covariance_p4", 48, 40, 4, 1, 15.0, dict(block_size=4, block_step=2, group_size=12, rank=6, bm_range=3)),
    ("gray_covariance_p7", 64, 48, 4, 1, 20.0, dict(block_size=7, block_step=4, group_size=16, rank=8)),
    ("yuv_uncoupled_covariance", 48, 40, 3, 3, 15.0, dict(chroma=0, block_size=4, block_step=2, group_size=10,
                                                          rank=5, bm_range=3)),
    # the reference's large-model profiles (tests/vs/integration_cuda.py:380-398, 436-448): 100 and 60 model
    # rows of dimension 294 (block 7, patch_time 2, YUV), rank 39
    ("yuv_k100_rank39", 64, 56, 3, 3, 8.0, dict(block_size=7, group_size=100, rank=39, cap_factor=1.0, bm_range=13,
                                                patch_time=2, block_step=16, radius=0, variance_threshold=2.7)),
    ("yuv_k60_rank39", 64, 56, 3, 3, 8.0, dict(block_size=7, group_size=60, rank=39, cap_factor=1.0, bm_range=13,
                                               patch_time=2, block_step=16, radius=0, variance_threshold=1.8)),
]


@pytest.mark.parametrize("name,w,h,f,planes,sigma,kw", CASES, ids=[c[0] for c in CASES])
def test_stagewise_bit_exact(name, w, h, f, planes, sigma, kw):
    _, noisy = synth.make_clip(w, h, f, planes, sigma, seed=sum(map(ord, name)))
    bp = O.cpu_params(O.BASIC, sigma, **kw)
    fp = O.cpu_params(O.FINAL, sigma, **kw)
    ob, of = O.Oracle("port").chain(noisy, bp, fp)
    for stage, p, ref in ((lib.STAGE_BASIC, bp, None), (lib.STAGE_FINAL, fp, ob)):
        s = session_for(stage, p, noisy, ref)
        for anchor in range(f - p.patch_time + 1):
            d = s.diag_anchor(anchor)
            for gi, (x, y) in enumerate(d["xy"]):
                want = O.match_anchor(stage, p, noisy, ref, anchor, int(x), int(y))
                got = d["grid_rows"][gi][:d["counts"][gi]]
                assert len(got) == len(want), (stage, anchor, gi)
                for field in ("x", "y", "frame"):
                    assert np.array_equal(got[field], want[field]), (stage, anchor, gi, field)
                assert np.array_equal(bits(got["distance"]), bits(want["distance"])), (stage, anchor, gi)
            stack, groups, rows = O.anchor_groups(stage, p, noisy, ref, anchor)
            assert [tuple(d["xy"][i]) for i in d["active"]] == [(g[0], g[1]) for g in groups]
            ar = d["active_rows"]
            assert len(ar) == len(rows)
            for field in ("x", "y", "frame"):
                assert np.array_equal(ar[field], rows[field])
            assert np.array_equal(bits(ar["weight"]), bits(rows["weight"]))
            assert np.array_equal(bits(s.render_stack(anchor)), bits(stack))
        s.close()
    bs, basic, fs, final = gpu_chain(noisy, bp, fp)
    assert np.array_equal(bits(basic), bits(ob))
    assert np.array_equal(bits(final), bits(of))


def test_vnlbcu_defaults_match_oracle():
    """vnlbcu.Basic/Final with every default (block 7, patch_time 2, bm_range
    13, group 16, rank 15, step 3) against the oracle on the same parameters."""
    _, noisy = synth.make_clip(80, 64, 5, 3, 20.0, seed=31)
    basic = vnlbcu.Basic(noisy, sigma=20.0)
    final = vnlbcu.Final(noisy, ref=basic, sigma=20.0)

    def to_stage(params):
        return O.StageParams(**{f: getattr(params, f) for f in O.StageParams.__dataclass_fields__})

    pb = vnlbcu.parse_parameters(lib.STAGE_BASIC, noisy, 20.0, {})
    pf = vnlbcu.parse_parameters(lib.STAGE_FINAL, noisy, 20.0, {})
    o = O.Oracle("port")
    ob = o.aggregate(o.stage_stacks(O.BASIC, to_stage(pb), noisy), noisy, pb.search_bwd, pb.search_fwd, pb.patch_time)
    of = o.aggregate(o.stage_stacks(O.FINAL, to_stage(pf), noisy, ob), noisy, pf.search_bwd, pf.search_fwd,
                     pf.patch_time)
    assert np.array_equal(bits(basic), bits(ob))
    assert np.array_equal(bits(final), bits(of))


def test_random_access_and_threads():
    _, noisy = synth.make_clip(64, 48, 6, 3, 20.0, seed=41)
    f = vnlbcu.BasicFilter(noisy, sigma=20.0, block_size=8, block_step=8, group_size=8, rank=8, bm_range=5)
    whole = f.render()
    order = [5, 0, 3, 1, 4, 2]
    for n in order:
        assert np.array_equal(f.get_frame(n), whole[n])
    results = {}

    def worker(n):
        results[n] = f.get_frame(n)

    threads = [threading.Thread(target=worker, args=(n,)) for n in range(6)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for n in range(6):
        assert np.array_equal(results[n], whole[n])


def test_pinned_host_pipeline_matches_pageable():
    """Pinned host clips go up frame by frame on an upload stream and pinned
    outputs come down frame by frame while later anchor frames compute; the
    result must equal the pageable path (whole-clip copies) bit for bit, for
    Basic and for Final reading both sources, and again after re-uploading."""
    import torch

    _, noisy = synth.make_clip(96, 64, 7, 3, 20.0, seed=61)
    p = O.cpu_params(O.BASIC, 20.0, radius=2, patch_time=2, group_size=12, rank=10)
    pf = O.cpu_params(O.FINAL, 20.0, radius=2, patch_time=2, group_size=12, rank=10, tau=400.0)
    sb = session_for(lib.STAGE_BASIC, p, noisy)
    want_b = sb.render_clip()
    sf = session_for(lib.STAGE_FINAL, pf, noisy, want_b)
    want_f = sf.render_clip()
    h_noisy = torch.from_numpy(noisy).pin_memory()
    h_basic = torch.empty_like(h_noisy).pin_memory()
    h_final = torch.empty_like(h_noisy).pin_memory()
    for _ in range(2):
        sb.set_clip_ptr(lib.SOURCE_CLIP, h_noisy.data_ptr())
        sb.render_clip_into(h_basic.data_ptr())
        sf.set_clip_ptr(lib.SOURCE_CLIP, h_noisy.data_ptr())
        sf.set_clip_ptr(lib.SOURCE_REF, h_basic.data_ptr())
        sf.render_clip_into(h_final.data_ptr())
        assert np.array_equal(bits(h_basic.numpy()), bits(want_b))
        assert np.array_equal(bits(h_final.numpy()), bits(want_f))
    sb.close()
    sf.close()


def test_aggregate_matches_oracle():
    _, noisy = synth.make_clip(48, 40, 4, 3, 20.0, seed=51)
    p = O.cpu_params(O.BASIC, 20.0, radius=2, patch_time=2, group_size=12, rank=10)
    stacks = O.Oracle("port").stage_stacks(O.BASIC, p, noisy)
    want = O.Oracle("port").aggregate(stacks, noisy, 2, 2, 2)
    got = vnlb.Aggregate(stacks, src=noisy, patch_time=2, radius=2)
    assert np.array_equal(bits(got), bits(want))


@pytest.mark.parametrize("planes", [1, 3])
def test_constant_video(planes):
    """Equal groups pass through unfiltered (core.cpp:110-131, 516-531); the
    output reproduces the constant (tests/cpp/test_core.cpp:247-356, 1e-5)
    and equals the oracle bit for bit."""
    clip = np.full((4, planes, 40, 48), 0.625, np.float32)
    kw = dict(block_size=8, block_step=4, group_size=8, rank=8, bm_range=4)
    out = vnlbcu.Basic(clip, sigma=10.0, **kw)
    pb = vnlbcu.parse_parameters(lib.STAGE_BASIC, clip, 10.0, kw)
    p = O.StageParams(**{f: getattr(pb, f) for f in O.StageParams.__dataclass_fields__})
    want = O.Oracle("port").aggregate(O.Oracle("port").stage_stacks(O.BASIC, p, clip), clip, p.search_bwd,
                                      p.search_fwd, p.patch_time)
    assert np.array_equal(bits(out), bits(want))
    assert np.allclose(out, 0.625, atol=1e-5)


def test_unsupported_configurations_raise():
    gray = np.zeros((3, 1, 32, 32), np.float32)
    with pytest.raises(lib.VNLBError, match="dual-PCA"):
        # vnlbcu keeps its rule min(group_size, candidates) < dimension (here 2 x 2 x 2 = 8)
        vnlbcu.Basic(gray, sigma=10.0, block_size=2, group_size=8, rank=4)
    with pytest.raises(lib.VNLBError, match="chroma=1"):
        vnlbcu.Basic(np.zeros((3, 3, 32, 32), np.float32), sigma=10.0, chroma=0)  # vnlbcu keeps its rule
    with pytest.raises(lib.VNLBError, match="at most 128 model samples"):
        # derive_geometry's limit (cuda_plugin.cpp:43, 730): 130 model rows of dimension 294
        vnlbcu.Basic(np.zeros((3, 3, 64, 64), np.float32), sigma=10.0, group_size=130, rank=20, cap_factor=1.0)


def test_full_size_anchor_frames_bit_exact():
    """1920x1080 YUV444PS, CPU-default parameters: GPU stacks of anchor frames
    0-2 of both stages equal the oracle's."""
    _, noisy = synth.make_clip(1920, 1080, 4, 3, 20.0, seed=0)
    bp = O.cpu_params(O.BASIC, 20.0)
    fp = O.cpu_params(O.FINAL, 20.0)
    sb = session_for(lib.STAGE_BASIC, bp, noisy)
    basic = sb.render_clip()
    sf = session_for(lib.STAGE_FINAL, fp, noisy, basic)
    o = O.Oracle("port")
    for stage, s, p, ref in ((lib.STAGE_BASIC, sb, bp, None), (lib.STAGE_FINAL, sf, fp, basic)):
        want = o.stage_stacks(stage, p, noisy, ref, first_anchor=0, anchor_count=3, threads=3)
        for a in range(3):
            assert np.array_equal(bits(s.render_stack(a)), bits(want[a])), (stage, a)
    again = session_for(lib.STAGE_BASIC, bp, noisy).render_clip()
    assert np.array_equal(bits(again), bits(basic))  # deterministic


@pytest.mark.parametrize("kw", [dict(block_size=8, block_step=8, group_size=8, bm_range=9, radius=1, patch_time=1,
                                     rank=8),
                                dict(block_size=7, block_step=3, group_size=16, bm_range=6, search_bwd=2,
                                     search_fwd=1, patch_time=2, rank=15)],
                         ids=["cpu_defaults", "patch_time2_asymmetric"])
def test_chain_render_matches_oracle(kw):
    """Basic into Final with the two stages overlapped on the device
    (vnlbgpu_render_chain_device) equals the oracle's chain bit for bit, the
    sessions sharing one caller stream as the bench runs them."""
    import torch

    _, noisy = synth.make_clip(72, 56, 9, 3, 20.0, seed=77)
    bp = O.cpu_params(O.BASIC, 20.0, **kw)
    fp = O.cpu_params(O.FINAL, 20.0, **kw)
    ob, of = O.Oracle("port").chain(noisy, bp, fp)
    d_noisy = torch.from_numpy(noisy).cuda()
    d_basic = torch.empty_like(d_noisy)
    d_final = torch.empty_like(d_noisy)
    sessions = []
    for stage, p in ((lib.STAGE_BASIC, bp), (lib.STAGE_FINAL, fp)):
        d = {f: getattr(p, f) for f in p.__dataclass_fields__}
        params = lib.Params(stage=stage, device_id=0, num_streams=1, chunk_size=768,
                            **{k: (float(v) if isinstance(v, (float, np.floating)) else int(v)) for k, v in d.items()})
        sessions.append(lib.Session(params, 72, 56, 9, 3))
    sb, sf = sessions
    stream = torch.cuda.Stream()
    for s in sessions:
        s.set_stream(stream.cuda_stream)
    sb.set_clip_device(lib.SOURCE_CLIP, d_noisy.data_ptr())
    sf.set_clip_device(lib.SOURCE_CLIP, d_noisy.data_ptr())
    sf.set_clip_device(lib.SOURCE_REF, d_basic.data_ptr())
    for _ in range(2):  # the second pass reuses the cached stacks' slots
        d_basic.fill_(float("nan"))
        d_final.fill_(float("nan"))
        torch.cuda.synchronize()
        sb.set_clip_device(lib.SOURCE_CLIP, d_noisy.data_ptr())  # drops the cached stacks
        sf.set_clip_device(lib.SOURCE_CLIP, d_noisy.data_ptr())
        sf.set_clip_device(lib.SOURCE_REF, d_basic.data_ptr())
        lib.render_chain_device(sb, sf, d_basic.data_ptr(), d_final.data_ptr())
        sb.synchronize()
        sf.synchronize()
        stream.synchronize()
        assert np.array_equal(bits(d_basic.cpu().numpy()), bits(ob))
        assert np.array_equal(bits(d_final.cpu().numpy()), bits(of))
    with pytest.raises(lib.VNLBError, match="ref must be the chain's Basic output"):
        lib.render_chain_device(sb, sf, d_final.data_ptr(), d_basic.data_ptr())


def test_autotuned_session_stays_bit_exact():
    """The autotuner times strip widths and apply kernels and keeps the
    fastest; every candidate computes the same bits, so the tuned session
    still equals the oracle."""
    _, noisy = synth.make_clip(160, 96, 4, 3, 20.0, seed=78)
    bp = O.cpu_params(O.BASIC, 20.0)
    ob = O.Oracle("port").chain(noisy, bp, O.cpu_params(O.FINAL, 20.0))[0]
    s = session_for(lib.STAGE_BASIC, bp, noisy)
    choice = s.autotune(1)
    assert choice["match_warps"] in (2, 4, 8)
    assert len(choice["timings"]) >= 2, choice
    out = s.render_clip()
    assert np.array_equal(bits(out), bits(ob))
