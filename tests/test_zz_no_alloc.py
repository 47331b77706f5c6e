"""The per-frame aggregate without allocation, against the whole-clip one.

vnlbgpu_aggregate_frame_noalloc stages the contributing stack rows of one
output frame through a fixed device scratch; vnlbgpu_aggregate allocates
device buffers for the whole clip.  Both are called through the C ABI and
must agree bit for bit, call after call (the scratch carries nothing from one
call to the next).  This file is collected last, so it also runs after every
other GPU test in the same process.
"""
import numpy as np
import pytest

import synth
import vnlb
import vnlbgpu_lib as lib

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def test_matches_whole_clip_aggregate_on_plugin_stacks():
    _, noisy = synth.make_clip(48, 40, 5, 3, 20.0, seed=71)
    stacks = vnlb.Basic(noisy, sigma=20.0, radius=2, patch_time=2, group_size=12, rank=10)
    whole = lib.aggregate(stacks, noisy, 2, 2, 2)
    for n in (1, 2, 1):  # two calls in a row, then the first again
        got = lib.aggregate_frame_noalloc(stacks, noisy, n, 2, 2, 2)
        assert np.array_equal(bits(got), bits(whole[n])), n


def test_matches_whole_clip_aggregate_in_several_bands():
    # 1024 x 600 YUV444: (3 stacks * 2 + 2) * 3 planes * 1024 * 4 bytes per
    # row, so a 32 MiB scratch takes the frame in two bands of rows
    rng = np.random.default_rng(72)
    frames, planes, h, w = 3, 3, 600, 1024
    slots = 3  # search_bwd 1, search_fwd 1, patch_time 1
    stacks = rng.uniform(0.0, 4.0, (frames, planes, slots * 2 * h, w)).astype(np.float32)
    for c in range(planes):  # weight rows: some zero, so the source is taken there
        for s in range(slots):
            rows = stacks[:, c, (2 * s + 1) * h:(2 * s + 2) * h]
            rows[rng.random(rows.shape) < 0.3] = 0.0
    source = rng.uniform(0.0, 1.0, (frames, planes, h, w)).astype(np.float32)
    whole = lib.aggregate(stacks, source, 1, 1, 1)
    for n in (0, 1):
        got = lib.aggregate_frame_noalloc(stacks, source, n, 1, 1, 1)
        assert np.array_equal(bits(got), bits(whole[n])), n


def test_rejects_a_row_larger_than_the_scratch():
    w = 700_000  # (1 stack * 2 + 2) * 3 planes * 700000 * 4 bytes > 32 MiB
    stacks = np.zeros((1, 3, 2, w), np.float32)
    source = np.zeros((1, 3, 1, w), np.float32)
    with pytest.raises(lib.VNLBError, match="one row of this frame needs"):
        lib.aggregate_frame_noalloc(stacks, source, 0, 0, 0, 1)
    with pytest.raises(lib.VNLBError, match="outside the clip"):
        lib.aggregate_frame_noalloc(stacks[:, :, :, :16], source[:, :, :, :16], 1, 0, 0, 1)


def test_rejects_a_device_or_slot_count_outside_its_limits():
    stacks = np.zeros((1, 1, 2, 16), np.float32)
    source = np.zeros((1, 1, 1, 16), np.float32)
    with pytest.raises(lib.VNLBError, match="outside the 64 devices"):
        lib.aggregate_frame_noalloc(stacks, source, 0, 0, 0, 1, device_id=64)
    # search_bwd + search_fwd + patch_time = 33 slots
    with pytest.raises(lib.VNLBError, match="at most 32 contribution slots"):
        lib.aggregate_frame_noalloc(stacks, source, 0, 16, 16, 1)
