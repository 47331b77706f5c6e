"""The multi-rank plumbing of bench.py on the CPU: two gloo ranks.

Under torchrun each rank denoises its own clip; the ranks meet only at the
barriers around the timed regions and in the max of their timings, and the
whole-job rate counts every rank's frames over the slowest rank's time.  The
reference arm runs on rank 0 alone; the other ranks exit at once.
"""
import json
import os
import socket

import pytest
import torch.multiprocessing as mp

import bench


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank: int, world: int, port: int, out_dir: str):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    ranks = bench.RankGroup("gloo", timeout_s=60.0)
    ranks.barrier()
    elapsed_ms = 100.0 * (rank + 1)  # rank 1 is the slow one
    max_ms = ranks.max(elapsed_ms)
    rate = bench.whole_job_rate(ranks.world, bench.FRAMES, 4, max_ms)
    ranks.close()
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump({"rank": ranks.rank, "world": ranks.world, "max_ms": max_ms, "rate": rate}, f)


def test_two_gloo_ranks_take_the_max_and_count_all_frames(tmp_path):
    world = 2
    mp.start_processes(rank_main, args=(world, free_port(), str(tmp_path)), nprocs=world, start_method="spawn",
                       join=True)
    results = [json.loads((tmp_path / f"rank{r}.json").read_text()) for r in range(world)]
    for r, res in enumerate(results):
        assert res["rank"] == r and res["world"] == world
        assert res["max_ms"] == 200.0
        # 2 ranks x 16 frames x 4 steps over the slowest rank's 0.2 s
        assert res["rate"] == pytest.approx(2 * bench.FRAMES * 4 / 0.2)


def test_single_rank_needs_no_process_group(monkeypatch):
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    ranks = bench.RankGroup("gloo")
    assert (ranks.rank, ranks.world) == (0, 1)
    assert ranks.max(12.5) == 12.5
    ranks.barrier()
    ranks.close()


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")

    class Args:
        gpus, steps, warmup = 2, 1, 0

    assert bench.run_reference(Args()) == 0
    assert capsys.readouterr().out == ""


def test_parameter_sets_of_the_bench(monkeypatch):
    """The headline passes the CPU core's defaults explicitly; --params vnlbcu
    takes vnlbcu's own (block 7, automatic step 3, group 16, bm_range 13,
    patch_time 2, rank 15; cuda_plugin.cpp:380-403) for both stages."""
    import vnlbgpu_lib as lib

    monkeypatch.setattr(bench, "PARAMS", "cpu")
    b = bench.stage_params(lib.STAGE_BASIC)
    assert (b.patch_size, b.proc_step, b.similar, b.search_window, b.patch_time, b.rank) == (8, 8, 8, 19, 1, 8)
    monkeypatch.setattr(bench, "PARAMS", "vnlbcu")
    for stage in (lib.STAGE_BASIC, lib.STAGE_FINAL):
        p = bench.stage_params(stage)
        assert (p.patch_size, p.proc_step, p.similar, p.search_window, p.patch_time, p.rank) == (7, 3, 16, 27, 2, 15)
    assert bench.workload_config("plain")["params"]["block_size"] == 7


def test_reference_arm_refuses_the_vnlbcu_parameter_set(monkeypatch, capsys):
    monkeypatch.setattr(bench, "PARAMS", "vnlbcu")
    monkeypatch.delenv("RANK", raising=False)
    assert bench.run_reference(None) == 0
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and "unavailable" in line
