"""One clip over several GPUs: the halo shard plan (vnlbgpu_shard_plan), on the CPU.

Each rank renders a contiguous block of Final output frames.  It renders the
Basic frames those read and uploads the source frames those Basic frames read
(the plan's halos), and nothing crosses between ranks.  The proof here runs
the CPU oracle per rank on a copy of the clip whose frames outside the rank's
source range are replaced by random values, and whose Basic frames outside
the rank's Basic range are replaced too: if the plan's halos were short, the
garbage would reach the rank's outputs.  The blocks joined must equal the
whole-clip oracle output bit for bit.  The second test runs the same plan as
two gloo ranks that gather their blocks.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import oracle as O
import synth
import vnlbgpu_lib as lib

CASES = [
    # name, frames, world, basic kwargs, final kwargs
    ("radius1", 11, 2, dict(radius=1, patch_time=1), dict(radius=1, patch_time=1)),
    ("radius1_world3", 11, 3, dict(radius=1, patch_time=1), dict(radius=1, patch_time=1)),
    ("asymmetric_patch_time2", 12, 3, dict(search_bwd=2, search_fwd=1, patch_time=2),
     dict(search_bwd=1, search_fwd=2, patch_time=1)),
]
SHARED = dict(block_size=8, block_step=8, group_size=8, bm_range=5, rank=8)


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.int32)


def stage_params(case):
    _, _, _, bk, fk = case
    bp = O.cpu_params(O.BASIC, 20.0, **SHARED, **bk)
    fp = O.cpu_params(O.FINAL, 20.0, **SHARED, **fk)
    return bp, fp


def clip_of(case):
    name, frames = case[0], case[1]
    return synth.make_clip(40, 32, frames, 1, 20.0, seed=sum(map(ord, name)))[1]


def whole(case):
    bp, fp = stage_params(case)
    return O.Oracle("port").chain(clip_of(case), bp, fp)


def shard(case, rank):
    """Rank's Final block from its plan alone: (first, last, frames) or None."""
    _, frames, world, _, _ = case
    bp, fp = stage_params(case)
    plan = lib.shard_plan(frames, world, rank, (bp.search_bwd, bp.search_fwd, bp.patch_time),
                          (fp.search_bwd, fp.search_fwd, fp.patch_time))
    if plan["out"] is None:
        return None
    noisy = clip_of(case)
    rng = np.random.default_rng(rank + 100)
    s0, s1 = plan["source"]
    local = noisy.copy()
    outside = np.ones(frames, bool)
    outside[s0:s1 + 1] = False
    local[outside] = rng.uniform(-1.0, 2.0, local[outside].shape).astype(np.float32)
    o = O.Oracle("port")
    basic = o.aggregate(o.stage_stacks(O.BASIC, bp, local), local, bp.search_bwd, bp.search_fwd, bp.patch_time)
    b0, b1 = plan["basic"]
    outside_b = np.ones(frames, bool)
    outside_b[b0:b1 + 1] = False
    basic[outside_b] = rng.uniform(-1.0, 2.0, basic[outside_b].shape).astype(np.float32)
    final = o.aggregate(o.stage_stacks(O.FINAL, fp, local, basic), local, fp.search_bwd, fp.search_fwd,
                        fp.patch_time)
    f0, f1 = plan["out"]
    return f0, f1, final[f0:f1 + 1]


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_blocks_with_halos_join_into_the_whole_clip(case):
    _, frames, world, _, _ = case
    _, want = whole(case)
    got = np.full_like(want, np.nan)
    covered = np.zeros(frames, int)
    for rank in range(world):
        r = shard(case, rank)
        if r is None:
            continue
        f0, f1, block = r
        got[f0:f1 + 1] = block
        covered[f0:f1 + 1] += 1
    assert (covered == 1).all()  # the blocks partition the clip
    assert np.array_equal(bits(got), bits(want))


def test_plan_ranges():
    # 16 frames, radius 1, patch_time 1 on both stages, 3 ranks: blocks of 5,
    # 5, 6; a Final frame reads frames n-2 .. n+2, a Basic frame the same
    got = [lib.shard_plan(16, 3, r, (1, 1, 1), (1, 1, 1)) for r in range(3)]
    assert [g["out"] for g in got] == [(0, 4), (5, 9), (10, 15)]
    assert [g["basic"] for g in got] == [(0, 6), (3, 11), (8, 15)]
    assert [g["source"] for g in got] == [(0, 8), (1, 13), (6, 15)]
    # more ranks than frames: blocks floor(r * 2 / 4) .. floor((r + 1) * 2 / 4) - 1
    assert [lib.shard_plan(2, 4, r, (1, 1, 1), (1, 1, 1))["out"] for r in range(4)] == [None, (0, 0), None, (1, 1)]
    with pytest.raises(lib.VNLBError, match="0 <= rank < world"):
        lib.shard_plan(16, 2, 2, (1, 1, 1), (1, 1, 1))


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank: int, world: int, port: int, out_dir: str):
    import torch
    import torch.distributed as dist
    from datetime import timedelta

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    case = CASES[0]
    frames = case[1]
    block = torch.full((frames, 1, 32, 40), float("nan"))
    r = shard((case[0], frames, world, case[3], case[4]), rank)
    if r is not None:
        f0, f1, out = r
        block[f0:f1 + 1] = torch.from_numpy(out)
    # the test gathers the blocks to check them; the ranks' data paths
    # exchanged nothing
    gathered = [torch.empty_like(block) for _ in range(world)]
    dist.all_gather(gathered, block)
    if rank == 0:
        joined = torch.full_like(block, float("nan"))
        for g in gathered:
            mask = ~torch.isnan(g)
            joined[mask] = g[mask]
        np.save(os.path.join(out_dir, "joined.npy"), joined.numpy())
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_gloo_ranks_render_their_blocks(tmp_path):
    world = 2
    mp.start_processes(rank_main, args=(world, free_port(), str(tmp_path)), nprocs=world, start_method="spawn",
                       join=True)
    joined = np.load(tmp_path / "joined.npy")
    _, want = whole(CASES[0])
    assert np.array_equal(bits(joined), bits(want))
