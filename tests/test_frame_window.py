"""The per-frame drop-in sequence, the way a VapourSynth plugin drives it.

A vnlbcu filter's getFrame asks for the required source range of output frame
n (request_frames / required_source_range, src/vs/cuda_plugin.cpp:809-858),
then renders frame n from those frames (render_frame, :1635-1864).  Here
several threads play VapourSynth's frame threads: each takes output frames in
a shuffled order, reads vnlbgpu_required_source_range, and calls
vnlbgpu_render_frame_window with per-plane frames whose rows are padded (a
VapourSynth stride).  The clip is longer than the session's source store, so
frames are pushed out and copied again.  Outputs must equal the CPU oracle's
aggregated Basic and Final frames bit for bit.
"""
import queue
import threading

import numpy as np
import pytest

import oracle as O
import synth
import vnlbgpu_lib as lib

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.int32)


def session(stage, p: O.StageParams, shape, num_streams):
    d = {f: getattr(p, f) for f in p.__dataclass_fields__}
    params = lib.Params(stage=stage, device_id=0, num_streams=num_streams, chunk_size=768,
                        **{k: (float(v) if isinstance(v, (float, np.floating)) else int(v)) for k, v in d.items()})
    frames, planes, h, w = shape
    return lib.Session(params, w, h, frames, planes)


def vs_frames(clip, pad=7):
    """Each frame as VapourSynth hands it over: one 2-D array per plane, rows
    `pad` floats longer than the frame (a stride of (W + pad) * 4 bytes)."""
    frames, planes, h, w = clip.shape
    out = []
    for f in range(frames):
        per_plane = []
        for c in range(planes):
            buf = np.full((h, w + pad), np.nan, np.float32)
            buf[:, :w] = clip[f, c]
            per_plane.append(buf[:, :w])
        out.append(per_plane)
    return out


def render_threaded(s, clip_frames, ref_frames, order, threads):
    """Output frames `order` rendered by `threads` threads through the window
    call; returns [frames][planes][H][W]."""
    frames = len(clip_frames)
    planes, h, w = len(clip_frames[0]), *clip_frames[0][0].shape
    out = np.full((frames, planes, h, w), np.nan, np.float32)
    work = queue.Queue()
    for n in order:
        work.put(int(n))
    errors = []

    def worker():
        try:
            while True:
                try:
                    n = work.get_nowait()
                except queue.Empty:
                    return
                first, last = s.required_source_range(n)
                cf = clip_frames[first:last + 1]
                rf = ref_frames[first:last + 1] if ref_frames is not None else None
                s.render_frame_window(n, cf, rf, first=first, out=out[n])
        except Exception as e:  # noqa: BLE001 - reported below
            errors.append(e)

    pool = [threading.Thread(target=worker) for _ in range(threads)]
    for t in pool:
        t.start()
    for t in pool:
        t.join(timeout=300)
        assert not t.is_alive(), "a render thread did not finish"
    if errors:
        raise errors[0]
    return out


CASES = [
    # name, width, height, frames, planes, sigma, shared kwargs
    ("gray_radius1", 64, 48, 14, 1, 20.0, dict(block_size=8, block_step=8, group_size=8, bm_range=9, radius=1,
                                                patch_time=1, rank=8)),
    ("yuv_patch_time2", 48, 40, 12, 3, 20.0, dict(block_size=7, block_step=3, group_size=16, bm_range=6, radius=1,
                                                   patch_time=2, rank=15)),
]


@pytest.mark.timeout(600)
@pytest.mark.parametrize("name,w,h,frames,planes,sigma,kw", CASES, ids=[c[0] for c in CASES])
def test_threaded_window_renders_match_oracle(name, w, h, frames, planes, sigma, kw):
    _, noisy = synth.make_clip(w, h, frames, planes, sigma, seed=91)
    bp = O.cpu_params(O.BASIC, sigma, **kw)
    fp = O.cpu_params(O.FINAL, sigma, **kw)
    ob, of = O.Oracle("port").chain(noisy, bp, fp)
    rng = np.random.default_rng(5)
    # output frames in a locally shuffled order, as frame threads request them
    order = np.arange(frames)
    for i in range(0, frames, 4):
        rng.shuffle(order[i:i + 4])

    threads = 3
    sb = session(lib.STAGE_BASIC, bp, noisy.shape, threads)
    clip_frames = vs_frames(noisy)
    basic = render_threaded(sb, clip_frames, None, order, threads)
    st = sb.stats()
    assert st["source_slots"] < frames  # a bounded store, not the whole clip
    assert np.array_equal(bits(basic), bits(ob)), (name, np.abs(basic - ob).max())

    sf = session(lib.STAGE_FINAL, fp, noisy.shape, threads)
    final = render_threaded(sf, clip_frames, vs_frames(basic, pad=3), order, threads)
    assert sf.stats()["source_slots"] < frames
    assert np.array_equal(bits(final), bits(of)), (name, np.abs(final - of).max())


@pytest.mark.timeout(300)
def test_in_order_renders_compute_each_anchor_frame_once():
    """One thread, output frames in order: every anchor frame's stack is
    computed once and reused by the later output frames that need it, and
    every source frame crosses to the device once (the reference's
    contribution and source caches)."""
    w, h, frames, planes = 64, 48, 12, 1
    kw = dict(block_size=8, block_step=8, group_size=8, bm_range=9, radius=1, patch_time=1, rank=8)
    _, noisy = synth.make_clip(w, h, frames, planes, 20.0, seed=92)
    bp = O.cpu_params(O.BASIC, 20.0, **kw)
    ob = O.Oracle("port").chain(noisy, bp, O.cpu_params(O.FINAL, 20.0, **kw))[0]
    s = session(lib.STAGE_BASIC, bp, noisy.shape, 1)
    clip_frames = vs_frames(noisy)
    out = render_threaded(s, clip_frames, None, np.arange(frames), 1)
    assert np.array_equal(bits(out), bits(ob))
    st = s.stats()
    assert st["anchor_frames"] == frames  # patch_time 1: every frame is an anchor frame, once
    assert st["source_uploads"] == frames


@pytest.mark.timeout(300)
def test_set_frame_then_render_frame():
    """The two-call form: set_frame over the required range (a frame already
    on the device is not copied again), then render_frame."""
    w, h, frames, planes = 48, 40, 9, 3
    kw = dict(block_size=8, block_step=8, group_size=8, bm_range=9, radius=1, patch_time=1, rank=8)
    _, noisy = synth.make_clip(w, h, frames, planes, 20.0, seed=93)
    bp = O.cpu_params(O.BASIC, 20.0, **kw)
    ob = O.Oracle("port").chain(noisy, bp, O.cpu_params(O.FINAL, 20.0, **kw))[0]
    s = session(lib.STAGE_BASIC, bp, noisy.shape, 1)
    clip_frames = vs_frames(noisy)
    with pytest.raises(lib.VNLBError, match="clip frames were not provided"):
        s.render_frame(0)
    s.set_frame(lib.SOURCE_CLIP, frames - 1, clip_frames[frames - 1])
    with pytest.raises(lib.VNLBError, match="frame 0 of clip is not on the device"):
        s.render_frame(0)
    for n in range(frames):
        first, last = s.required_source_range(n)
        for f in range(first, last + 1):
            s.set_frame(lib.SOURCE_CLIP, f, clip_frames[f])
        got = s.render_frame(n)
        assert np.array_equal(bits(got), bits(ob[n])), n
    # every frame once, and the last frame twice: given first, pushed out of
    # its slot by frame 3, given again for output frame 6
    assert s.stats()["source_uploads"] == frames + 1


@pytest.mark.timeout(120)
def test_window_larger_than_the_store_is_refused():
    w, h, frames, planes = 32, 32, 20, 1
    kw = dict(block_size=8, block_step=8, group_size=8, bm_range=3, radius=1, patch_time=1, rank=8)
    _, noisy = synth.make_clip(w, h, frames, planes, 20.0, seed=94)
    s = session(lib.STAGE_BASIC, O.cpu_params(O.BASIC, 20.0, **kw), noisy.shape, 1)
    slots = s.stats()["source_slots"]
    assert slots == 5  # source window 2 * (1 + 1 + 1 - 1) + 1, one stream
    with pytest.raises(lib.VNLBError, match="exceed the 5 frame slots"):
        s.render_frame_window(8, vs_frames(noisy)[2:14], first=2)
