"""The chosen matchers against the plain one, through the C ABI.

The chosen forms run the CPU's selection on the approximate distance
||a||^2 + ||b||^2 - 2 a.b (FP32 dot products for "chosen", BF16 tensor-core
dot products for "chosen_tc"), re-compute the exact FP32 distance of every
retained candidate and select on the exact values.  They are not
bit-identical to the plain form; the bar is the one stated for them: PSNR
against the clean clip at most 0.05 dB below the plain form's.  The share of
groups whose retained rows are exactly the plain form's is bounded from
below, and the exact distances of rows both forms keep must be equal bit for
bit.
"""
import numpy as np
import pytest

import synth
import vnlbcu
import vnlbgpu_lib as lib

pytestmark = pytest.mark.gpu

CPU_DEFAULTS = dict(block_size=8, block_step=8, group_size=8, bm_range=9, radius=1, patch_time=1, rank=8,
                    cap_factor=4.0)
BASIC = dict(variance_threshold=1.1, weight_alpha=0.75, weight_beta=0.35, weight_gamma=1.0)
FINAL = dict(tau=400.0, variance_threshold=1.7, flat_areas=1, weight_alpha=1.0, weight_beta=0.5, weight_gamma=1.0)


def chain(noisy, form, **extra):
    kw = dict(CPU_DEFAULTS, form=form, **extra)
    basic = vnlbcu.Basic(noisy, sigma=20.0, **kw, **BASIC)
    final = vnlbcu.Final(noisy, ref=basic, sigma=20.0, **kw, **FINAL)
    return basic, final


@pytest.mark.parametrize("form", ["chosen", "chosen_tc"])
@pytest.mark.parametrize("planes,shape,seed", [(3, (192, 160, 6), 81), (1, (256, 192, 6), 82)])
def test_chosen_psnr_within_tolerance_of_plain(form, planes, shape, seed):
    w, h, f = shape
    clean, noisy = synth.make_clip(w, h, f, planes, 20.0, seed=seed)
    pb, pf = chain(noisy, "plain")
    cb, cf = chain(noisy, form)
    for plain, chosen in ((pb, cb), (pf, cf)):
        loss = synth.psnr(plain, clean) - synth.psnr(chosen, clean)
        assert loss <= 0.05, loss
        assert np.isfinite(chosen).all()


def rows_of(stage, form, noisy, ref=None, anchor=2, base=CPU_DEFAULTS):
    kw = dict(base, form=form)
    if base is CPU_DEFAULTS:
        kw.update(FINAL if stage == lib.STAGE_FINAL else BASIC)
    params = vnlbcu.parse_parameters(stage, noisy, 20.0, kw)
    frames, planes, h, w = noisy.shape
    s = lib.Session(params, w, h, frames, planes)
    s.set_clip(lib.SOURCE_CLIP, noisy)
    if ref is not None:
        s.set_clip(lib.SOURCE_REF, ref)
    d = s.diag_anchor(anchor)
    s.close()
    return d


@pytest.mark.parametrize("form,agree", [("chosen", 0.98), ("chosen_tc", 0.9)])
@pytest.mark.parametrize("stage", [lib.STAGE_BASIC, lib.STAGE_FINAL])
def test_chosen_selects_the_plain_rows(stage, form, agree):
    _, noisy = synth.make_clip(160, 128, 5, 3, 20.0, seed=83)
    ref = None
    if stage == lib.STAGE_FINAL:
        ref = vnlbcu.Basic(noisy, sigma=20.0, **CPU_DEFAULTS, **BASIC)
    plain = rows_of(stage, "plain", noisy, ref)
    chosen = rows_of(stage, form, noisy, ref)
    assert np.array_equal(plain["xy"], chosen["xy"])
    same = ordered = 0
    groups = len(plain["counts"])
    place = lambda r: (int(r["x"]), int(r["y"]), int(r["frame"]))
    for gi in range(groups):
        a = plain["grid_rows"][gi][: plain["counts"][gi]]
        b = chosen["grid_rows"][gi][: chosen["counts"][gi]]
        ka = {place(x): x["distance"] for x in a}
        kb = {place(x): x["distance"] for x in b}
        for pos in set(ka) & set(kb):  # exact re-rank: the plain form's distance bits
            assert np.float32(ka[pos]).view(np.uint32) == np.float32(kb[pos]).view(np.uint32)
        if set(ka) != set(kb):
            continue
        same += 1
        # the same rows: both forms put the K nearest first, in ascending
        # distance (partial_sort's sorted front); with no tie among them the
        # order is unique and must be the same
        k = min(8, len(a))
        if len(set(np.float32(a["distance"][:k]).view(np.uint32).tolist())) == k:
            assert [place(r) for r in a[:k]] == [place(r) for r in b[:k]], gi
            ordered += 1
    assert same / groups >= agree, (same, groups)
    assert ordered >= 0.5 * same, (ordered, same)  # the order check ran on most of the agreeing groups


@pytest.mark.parametrize("form,block", [("chosen", 7), ("chosen_tc", 6), ("chosen_tc", 10)])
def test_unsupported_patch_sizes_keep_the_plain_matcher(form, block):
    """The FP32 chosen form takes 8 x 8 patches, the tensor-core form 7 x 7
    and 8 x 8; other sizes keep the plain matcher: the output is the plain
    one."""
    _, noisy = synth.make_clip(64, 48, 4, 1, 20.0, seed=84)
    kw = dict(block_size=block, block_step=4, group_size=8, bm_range=5, rank=8)
    plain = vnlbcu.Basic(noisy, sigma=20.0, **kw)
    chosen = vnlbcu.Basic(noisy, sigma=20.0, form=form, **kw)
    assert np.array_equal(plain, chosen)


def sorted_rows(rows):
    d = rows["distance"]
    return bool(np.all(d[1:] >= d[:-1]))


@pytest.mark.parametrize("stage,tau", [(lib.STAGE_BASIC, None), (lib.STAGE_FINAL, None), (lib.STAGE_FINAL, 1e8)],
                         ids=["basic", "final", "final_tau1e8"])
def test_tensor_core_matcher_on_vnlbcu_defaults(stage, tau):
    """vnlbcu's own defaults on a YUV444 clip: 7 x 7 patches, patch_time 2 (six
    planes: two shared-memory stages of planes per frame, accumulated in
    tensor memory), step 3, group 16 with cap factor 4 (buffers of 64, two
    slots per lane).  The retained rows agree with the plain form's, with the
    plain form's exact distance bits; every group's rows come out sorted by
    distance (the chosen forms' step 4).  With tau raised to 1e8 (above any
    distance of 294 samples in [-0.5, 1.5]) every candidate passes the
    threshold, so every group keeps a full buffer of 64
    rows: the buffer's second register per lane and the replacement of its
    worst entry carry the selection, and the plain form's heap replay leaves
    rows past the K-th unsorted where the tensor-core path sorts them, which
    shows that path ran."""
    _, noisy = synth.make_clip(128, 96, 5, 3, 20.0, seed=86)
    ref = vnlbcu.Basic(noisy, sigma=20.0) if stage == lib.STAGE_FINAL else None
    base = {} if tau is None else {"tau": tau}
    plain = rows_of(stage, "plain", noisy, ref, base=base)
    tc = rows_of(stage, "chosen_tc", noisy, ref, base=base)
    assert plain["max_rows"] == 64
    assert np.array_equal(plain["xy"], tc["xy"])
    place = lambda r: (int(r["x"]), int(r["y"]), int(r["frame"]))
    groups = len(plain["counts"])
    same = unsorted_plain = shared = total = 0
    for gi in range(groups):
        a = plain["grid_rows"][gi][: plain["counts"][gi]]
        b = tc["grid_rows"][gi][: tc["counts"][gi]]
        assert sorted_rows(b), gi
        unsorted_plain += not sorted_rows(a)
        ka = {place(x): x["distance"] for x in a}
        kb = {place(x): x["distance"] for x in b}
        for pos in set(ka) & set(kb):
            assert np.float32(ka[pos]).view(np.uint32) == np.float32(kb[pos]).view(np.uint32)
        same += set(ka) == set(kb)
        shared += len(set(ka) & set(kb))
        total += len(ka)
    if tau is None:
        assert same / groups >= 0.9, (same, groups)
    else:
        assert np.all(plain["counts"] == 64), np.unique(plain["counts"])
        assert np.all(tc["counts"] == 64), np.unique(tc["counts"])
        assert unsorted_plain > 0
        # the boundary of 64 of 2187 candidates moves under BF16 distances
        assert shared / total >= 0.97, (shared, total)


def test_tensor_core_psnr_on_vnlbcu_defaults():
    """Basic then Final with vnlbcu's defaults: the tensor-core form within
    0.05 dB of the plain form's PSNR."""
    clean, noisy = synth.make_clip(160, 128, 6, 3, 20.0, seed=87)
    pb = vnlbcu.Basic(noisy, sigma=20.0)
    pf = vnlbcu.Final(noisy, ref=pb, sigma=20.0)
    tb = vnlbcu.Basic(noisy, sigma=20.0, form="chosen_tc")
    tf = vnlbcu.Final(noisy, ref=tb, sigma=20.0, form="chosen_tc")
    for plain, tc in ((pb, tb), (pf, tf)):
        assert np.isfinite(tc).all()
        assert synth.psnr(plain, clean) - synth.psnr(tc, clean) <= 0.05


def test_tensor_core_waits_run_out_and_report():
    """The tensor-core matcher's MMA-completion waits are bounded: with its
    MMA warp told to issue nothing (a test switch; no MMA is in flight), every
    wait runs out, the kernel returns, and the render raises; the session then
    renders normally again and equals a fresh session's output (up to the
    order of the atomic additions of filtered rows into the stacks, which the
    chosen forms use: 1e-5 max abs)."""
    _, noisy = synth.make_clip(96, 64, 4, 3, 20.0, seed=85)
    params = vnlbcu.parse_parameters(lib.STAGE_BASIC, noisy, 20.0, dict(CPU_DEFAULTS, form="chosen_tc", **BASIC))
    frames, planes, h, w = noisy.shape
    s = lib.Session(params, w, h, frames, planes)
    s.set_clip(lib.SOURCE_CLIP, noisy)
    s.stall_tensor_waits(True)
    with pytest.raises(lib.VNLBError, match="timed out waiting for its MMAs"):
        s.render_clip()
    s.stall_tensor_waits(False)
    again = s.render_clip()
    s.close()
    fresh = vnlbcu.Basic(noisy, sigma=20.0, form="chosen_tc", **CPU_DEFAULTS, **BASIC)
    assert float(np.max(np.abs(again - fresh))) <= 1e-5


def test_tensor_core_buffers_of_96():
    """group_size 24 with cap factor 4: buffers of 96 entries, three slots per
    lane in the selection replay (the mixed stream's sigma-5 setting); rank
    24, patch_time 2 on a gray clip (two planes).  Rows agree with the plain
    form's on most groups with its exact distance bits, and the output is
    within 0.05 dB of the plain form's."""
    clean, noisy = synth.make_clip(128, 96, 6, 1, 5.0, seed=88)
    kw = dict(block_size=8, block_step=8, group_size=24, bm_range=9, radius=1, patch_time=2, rank=24,
              cap_factor=4.0, tau=200.0)
    frames, planes, h, w = noisy.shape
    rows = {}
    for form in ("plain", "chosen_tc"):
        params = vnlbcu.parse_parameters(lib.STAGE_BASIC, noisy, 5.0, dict(kw, form=form))
        s = lib.Session(params, w, h, frames, planes)
        s.set_clip(lib.SOURCE_CLIP, noisy)
        rows[form] = s.diag_anchor(2)
        s.close()
    assert rows["plain"]["max_rows"] == 96
    place = lambda r: (int(r["x"]), int(r["y"]), int(r["frame"]))
    same = 0
    groups = len(rows["plain"]["counts"])
    for gi in range(groups):
        a = rows["plain"]["grid_rows"][gi][: rows["plain"]["counts"][gi]]
        b = rows["chosen_tc"]["grid_rows"][gi][: rows["chosen_tc"]["counts"][gi]]
        ka = {place(x): np.float32(x["distance"]).view(np.uint32) for x in a}
        kb = {place(x): np.float32(x["distance"]).view(np.uint32) for x in b}
        for pos in set(ka) & set(kb):
            assert ka[pos] == kb[pos]
        same += set(ka) == set(kb)
    assert same / groups >= 0.8, (same, groups)
    plain = vnlbcu.Basic(noisy, sigma=5.0, **kw)
    tc = vnlbcu.Basic(noisy, sigma=5.0, form="chosen_tc", **kw)
    assert synth.psnr(plain, clean) - synth.psnr(tc, clean) <= 0.05


def test_autotuned_tensor_core_session():
    """The autotuner times the tensor-core matcher's planes per shared-memory
    stage (YUV444, 3 planes: 3, 2 and 1 per stage) and keeps the fastest; the
    tuned session's output stays within 1e-3 dB of the untuned one's (the
    grouping only moves the approximate distances' last bits)."""
    clean, noisy = synth.make_clip(160, 128, 5, 3, 20.0, seed=89)
    kw = dict(CPU_DEFAULTS, form="chosen_tc", **FINAL)
    ref = vnlbcu.Basic(noisy, sigma=20.0, **CPU_DEFAULTS, **BASIC)
    params = vnlbcu.parse_parameters(lib.STAGE_FINAL, noisy, 20.0, kw)
    frames, planes, h, w = noisy.shape
    s = lib.Session(params, w, h, frames, planes)
    s.set_clip(lib.SOURCE_CLIP, noisy)
    s.set_clip(lib.SOURCE_REF, ref)
    untuned = s.render_clip()
    tuning = s.autotune(1)
    tuned = s.render_clip()
    s.close()
    assert any(t.startswith("tensor-core planes per stage") for t in tuning["timings"]), tuning
    assert abs(synth.psnr(tuned, clean) - synth.psnr(untuned, clean)) <= 1e-3


@pytest.mark.parametrize("w,h,planes,kw", [
    (97, 61, 1, dict(block_size=8, block_step=5, group_size=8, bm_range=9, radius=1, patch_time=1, rank=8)),
    (70, 50, 3, dict(block_size=7, block_step=3, group_size=16, bm_range=6, radius=1, patch_time=2, rank=12)),
    (130, 45, 1, dict(block_size=7, block_step=4, group_size=12, bm_range=13, radius=2, patch_time=2, rank=8)),
], ids=["gray_odd_97x61", "yuv_p7_pt2_70x50", "gray_p7_radius2_130x45"])
def test_tensor_core_odd_shapes(w, h, planes, kw):
    """Frame sizes that are no multiple of 4, 8 or the strip width, windows
    clipped by the frame edges, 7 x 7 and 8 x 8 patches, patch_time 1 and 2,
    radius 1 and 2: the tensor-core form stays finite and within 0.05 dB of
    the plain form, Basic and Final."""
    clean, noisy = synth.make_clip(w, h, 6, planes, 20.0, seed=90)
    pb = vnlbcu.Basic(noisy, sigma=20.0, **kw)
    pf = vnlbcu.Final(noisy, ref=pb, sigma=20.0, **kw)
    tb = vnlbcu.Basic(noisy, sigma=20.0, form="chosen_tc", **kw)
    tf = vnlbcu.Final(noisy, ref=tb, sigma=20.0, form="chosen_tc", **kw)
    for plain, tc in ((pb, tb), (pf, tf)):
        assert np.isfinite(tc).all()
        assert synth.psnr(plain, clean) - synth.psnr(tc, clean) <= 0.05


@pytest.mark.parametrize("planes", [1, 3])
def test_interleaved_stacks_read_back(planes):
    """The chosen forms add filtered rows into pixel-interleaved stacks
    (value planes and weight of a pixel side by side, one vector addition per
    pixel) at 1 and 3 planes.  Both readers must agree on that layout: the
    stacks read back in the vnlb.* frame layout, normalised here in anchor
    order, give the device's output frame bit for bit, and their weights
    cover the frame like the plain form's planar stacks do."""
    w, h, f, n = 96, 80, 6, 2
    clean, noisy = synth.make_clip(w, h, f, planes, 20.0, seed=93)
    kw = dict(CPU_DEFAULTS, **BASIC)
    out = {}
    for form in ("plain", "chosen_tc"):
        params = vnlbcu.parse_parameters(lib.STAGE_BASIC, noisy, 20.0, dict(kw, form=form))
        s = lib.Session(params, w, h, f, planes)
        s.set_clip(lib.SOURCE_CLIP, noisy)
        bwd, fwd, pt = params.search_bwd, params.search_fwd, params.patch_time
        anchors = [a for a in range(max(0, n - (fwd + pt - 1)), min(f - 1, n + bwd) + 1) if a <= f - pt]
        stacks = {a: s.render_stack(a) for a in anchors}
        frame = s.render_frame(n)
        s.close()
        num = np.zeros((planes, h, w), np.float32)
        wsum = np.zeros((h, w), np.float32)
        for a in anchors:
            slot = n - a + bwd
            num += stacks[a][:, 2 * slot * h:(2 * slot + 1) * h]
            wsum += stacks[a][0, (2 * slot + 1) * h:(2 * slot + 2) * h]
        safe = np.where(wsum > 0, wsum, np.float32(1))
        host = np.where(wsum > 0, num / safe, noisy[n])
        assert np.array_equal(host.view(np.uint32), frame.view(np.uint32)), form
        out[form] = (wsum, frame)
    (wp, fp), (wt, ft) = out["plain"], out["chosen_tc"]
    assert abs(float(wt.sum()) / float(wp.sum()) - 1.0) < 0.02
    assert synth.psnr(fp, clean[n]) - synth.psnr(ft, clean[n]) <= 0.05
