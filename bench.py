#!/usr/bin/env python
"""Throughput of the VNLB hot path: 1080p YUV444PS frames/s, Basic + Final.

Workload (one step): a 16-frame 1920x1080 YUV444PS float32 clip, sigma 20 on
the 8-bit scale, denoised by vnlbcu.Basic and then vnlbcu.Final with the
reference CPU core's default parameter set passed explicitly (block 8, step 8,
group 8, bm_range 9, radius 1, patch_time 1, rank 8, cap_factor 4; Final: tau
400, variance_threshold 1.7, flat areas, alpha 1, beta 0.5), which makes the
coupled estimator dimension 192 and the rank 8.  The clip is synthetic
(vapoursynth-vnlb_b200/synth.py, seed = rank): no public dataset is named for
this path.  The plain GPU form computes bit-identical output to the reference
CPU core.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--params cpu|vnlbcu]

`--params vnlbcu` runs the same clip with vnlbcu's own defaults instead (block
7, automatic step 3, group 16, bm_range 13, radius 1, patch_time 2, rank 15:
estimator dimension 294, about 230k groups per anchor frame), in the plain
form and the tensor-core form (the FP32 chosen form needs 8x8 patches),
without the CPU sample.

Under torchrun every rank (one GPU each) denoises its own clip for `value`
(weak scaling, no collective on the data path); rank 0 prints one JSON line.
`value` is measured with the clip already resident in HBM, Basic into Final
chained on the device (vnlbgpu_render_chain_device: a Final anchor frame
starts once the Basic frames of its window are out).  `e2e` is the same
metric through the plugin's per-frame call, vnlbgpu_render_frame_window (the
vnlbcu getFrame), from eight frame threads per stage with pageable host
frames, over a long clip through bounded source stores: every frame's copies
up and down are inside the timed region.  Under torchrun that clip is split
between the ranks by vnlbgpu_shard_plan (blocks of output frames with their
halos, no exchange).  `config.e2e_whole_clip` is the whole-clip host path
(pinned buffers: clip up for Basic and for Final, Basic frames down and up
again, Final frames down).  The roofline is taken from one more step with one
pipeline lane per session, so that each timed launch runs alone.  `--impl
reference` times the reference CPU implementation
(oracle/_ref, the reference's own sources; the C restatement if that build is
absent) on a bounded sample of the same workload on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "vapoursynth-vnlb_b200"))

import synth  # noqa: E402

METRIC = "1080p 444 frames/s Basic+Final: chosen vs plain GPU at ≤0.05 dB PSNR loss"
UNIT = "frames/s"
WIDTH, HEIGHT, FRAMES, PLANES, SIGMA = 1920, 1080, 16, 3, 20.0
CPU_DEFAULTS = dict(block_size=8, block_step=8, group_size=8, bm_range=9, radius=1, patch_time=1, rank=8,
                    cap_factor=4.0)
# nominal FP32 issue rate of a B200 (148 SMs x 128 lanes at the 1965 MHz max clock)
FP32_LANE_OPS = 148 * 128 * 1.965e9


# parameter set of the run: "cpu" (the CPU core's defaults, the headline) or
# "vnlbcu" (vnlbcu's own defaults, a secondary row)
PARAMS = "cpu"


def workload_config(form: str) -> dict:
    if PARAMS == "vnlbcu":
        return {"workload": "vnlbcu.Basic+Final 1920x1080 YUV444PS 16 frames sigma 20, vnlbcu default parameters",
                "form": form, "width": WIDTH, "height": HEIGHT, "frames_per_clip": FRAMES, "planes": PLANES,
                "sigma": SIGMA, "params": dict(block_size=7, block_step=3, group_size=16, bm_range=13, radius=1,
                                               patch_time=2, rank=15, cap_factor=4.0),
                "l2": "inputs larger than L2 (398 MB clip per rank)"}
    return {"workload": "vnlbcu.Basic+Final 1920x1080 YUV444PS 16 frames sigma 20, CPU-default parameter set",
            "form": form, "width": WIDTH, "height": HEIGHT, "frames_per_clip": FRAMES, "planes": PLANES,
            "sigma": SIGMA, "params": CPU_DEFAULTS, "l2": "inputs larger than L2 (398 MB clip per rank)"}


def stage_params(stage: int, form: str = "plain"):
    import vnlbgpu_lib as lib
    import vnlbcu
    clip_shape = np.empty((FRAMES, PLANES, HEIGHT, WIDTH), np.float32)  # shape only for the parser
    if PARAMS == "vnlbcu":
        return vnlbcu.parse_parameters(stage, clip_shape, SIGMA, dict(form=form))
    kw = dict(CPU_DEFAULTS, form=form)
    if stage == lib.STAGE_FINAL:
        kw.update(tau=400.0, variance_threshold=1.7, flat_areas=1, weight_alpha=1.0, weight_beta=0.5,
                  weight_gamma=1.0)
    else:
        kw.update(variance_threshold=1.1, weight_alpha=0.75, weight_beta=0.35, weight_gamma=1.0)
    return vnlbcu.parse_parameters(stage, clip_shape, SIGMA, kw)


class ClockSampler:
    """nvidia-smi clock/throttle samples while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, sm_max, reasons = [], 0.0, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                sm_max = max(sm_max, float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": sm_max or None,
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------------------- CPU reference
def cpu_reference_sample(threads: int | None = None):
    """Times the reference CPU implementation on a bounded sample of the
    workload: a 1920 x 136 horizontal band of the clip (1/7.94 of a frame),
    Basic + Final anchor-frame processing of `threads` anchor frames in
    parallel (one thread per anchor frame, as VapourSynth's frame threading
    does).  Each output frame needs exactly one Basic and one Final anchor
    frame, so frames/s = threads * band_fraction / step_seconds."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    try:
        o, kind = O.Oracle("ref"), "reference"
    except FileNotFoundError:
        o, kind = O.Oracle("port"), "port"
    threads = threads or min(os.cpu_count() or 1, 64)
    band_rows = 136
    frames = threads + 2
    _, noisy = synth.make_clip(WIDTH, band_rows, frames, PLANES, SIGMA, seed=0)
    bp = O.cpu_params(O.BASIC, SIGMA, **CPU_DEFAULTS)
    fp = O.cpu_params(O.FINAL, SIGMA, **CPU_DEFAULTS)
    stacks = o.stage_stacks(O.BASIC, bp, noisy, threads=threads)
    basic = o.aggregate(stacks, noisy, bp.search_bwd, bp.search_fwd, bp.patch_time)

    def step():
        o.stage_stacks(O.BASIC, bp, noisy, first_anchor=1, anchor_count=threads, threads=threads)
        o.stage_stacks(O.FINAL, fp, noisy, basic, first_anchor=1, anchor_count=threads, threads=threads)

    fraction = band_rows / HEIGHT
    sample = (f"Basic+Final anchor frames 1..{threads} of a 1920x{band_rows} band ({frames} frames) of the "
              f"workload clip, {threads} threads; frames/s = {threads} x {fraction:.4f} / step seconds")
    return o, kind, threads, fraction, step, sample


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if PARAMS != "cpu":
        print(json.dumps({"impl": "reference", "unavailable": "the CPU sample is defined for the CPU-default "
                          "parameter set only (run without --params)"}), flush=True)
        return 0
    _, kind, threads, fraction, step, sample = cpu_reference_sample()
    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    seconds = (time.perf_counter() - t0) / args.steps
    value = threads * fraction / seconds
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": seconds * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": workload_config("reference CPU core"),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line, default=json_scalar), flush=True)
    return 0


# --------------------------------------------------------------------------- ranks
class RankGroup:
    """The ranks of one job: one process per GPU under torchrun (RANK,
    WORLD_SIZE, LOCAL_RANK, MASTER_ADDR/MASTER_PORT from the environment).
    Each rank denoises its own clip (seeded by its rank), so the data path
    exchanges nothing; the only collectives are the barriers around the timed
    regions and the max of the timings.  The GPU run uses backend "nccl" with
    the rank's device; the same code runs with "gloo" on the CPU."""

    def __init__(self, backend: str = "nccl", device=None, timeout_s: float = 300.0):
        import torch.distributed as dist
        self.dist = dist
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.device = device
        if self.world > 1:
            from datetime import timedelta
            kw = {"device_id": device} if device is not None else {}
            dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s), **kw)

    def barrier(self):
        if self.world > 1:
            self.dist.barrier()

    def max(self, value: float) -> float:
        """The maximum of `value` over the ranks (every rank gets it)."""
        if self.world == 1:
            return float(value)
        import torch
        t = torch.tensor([float(value)], dtype=torch.float64, device=self.device or "cpu")
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.world > 1:
            self.dist.barrier()
            self.dist.destroy_process_group()


def whole_job_rate(world: int, frames_per_step: int, steps: int, max_ms: float) -> float:
    """Frames/s of the whole job: every rank's frames over the slowest rank's time."""
    return world * frames_per_step * steps / (max_ms / 1e3)


# --------------------------------------------------------------------------- GPU path
def measure_form(form, args, ranks, stream, noisy, clean, d_noisy, local):
    """Times one matcher form over the workload: device-resident steps, then
    end-to-end steps through the C ABI with pinned host buffers."""
    import torch
    import vnlbgpu_lib as lib

    d_basic = torch.empty_like(d_noisy)
    d_final = torch.empty_like(d_noisy)
    bp, fp = stage_params(lib.STAGE_BASIC, form), stage_params(lib.STAGE_FINAL, form)
    bp.device_id = fp.device_id = local
    sb = lib.Session(bp, WIDTH, HEIGHT, FRAMES, PLANES)
    sf = lib.Session(fp, WIDTH, HEIGHT, FRAMES, PLANES)
    for s in (sb, sf):
        s.set_stream(stream.cuda_stream)

    def step():
        sb.set_clip_device(lib.SOURCE_CLIP, d_noisy.data_ptr())
        sf.set_clip_device(lib.SOURCE_CLIP, d_noisy.data_ptr())
        sf.set_clip_device(lib.SOURCE_REF, d_basic.data_ptr())
        sb.render_clip_device(d_basic.data_ptr())
        sf.render_clip_device(d_final.data_ptr())

    def chain_step():
        # Basic into Final on the device, the stages overlapped frame by frame
        # (a Final anchor frame starts once its window's Basic frames are out)
        sb.set_clip_device(lib.SOURCE_CLIP, d_noisy.data_ptr())
        sf.set_clip_device(lib.SOURCE_CLIP, d_noisy.data_ptr())
        sf.set_clip_device(lib.SOURCE_REF, d_basic.data_ptr())
        lib.render_chain_device(sb, sf, d_basic.data_ptr(), d_final.data_ptr())

    step()  # Basic output for Final's ref, then the tile-shape autotuner on anchor frame 1 of each stage
    torch.cuda.synchronize()
    tuning = {"basic": sb.autotune(1), "final": sf.autotune(1)}
    for _ in range(args.warmup):
        step()
    sb.synchronize()
    sf.synchronize()
    torch.cuda.synchronize()
    basic_out, final_out = d_basic.cpu().numpy(), d_final.cpu().numpy()
    psnr = {"noisy": synth.psnr(noisy, clean), "basic": synth.psnr(basic_out, clean),
            "final": synth.psnr(final_out, clean)}
    stats0 = [sb.stats(), sf.stats()]
    lanes = {"basic": stats0[0]["pipeline_lanes"], "final": stats0[1]["pipeline_lanes"]}
    sb.kernel_timing(True)
    sf.kernel_timing(True)
    ranks.barrier()
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(args.steps):
        step()
    end.record(stream)
    torch.cuda.synchronize()
    sb.synchronize()
    sf.synchronize()
    elapsed_ms = start.elapsed_time(end)
    kb, kf = sb.kernel_timing(False), sf.kernel_timing(False)
    stats1 = [sb.stats(), sf.stats()]
    delta = {k: sum(stats1[i][k] - stats0[i][k] for i in range(2)) for k in stats0[0]}
    max_ms = ranks.max(elapsed_ms)
    value = whole_job_rate(ranks.world, FRAMES, args.steps, max_ms)

    # end to end through the C ABI with pinned host buffers
    h_noisy = torch.from_numpy(noisy).pin_memory()
    h_basic = torch.empty_like(h_noisy).pin_memory()
    h_final = torch.empty_like(h_noisy).pin_memory()

    def e2e_step():
        # Final's clip does not depend on Basic: its copy is issued first and
        # runs while Basic computes (each session copies its own inputs)
        sb.set_clip_ptr(lib.SOURCE_CLIP, h_noisy.data_ptr())
        sf.set_clip_ptr(lib.SOURCE_CLIP, h_noisy.data_ptr())
        sb.render_clip_into(h_basic.data_ptr())
        sf.set_clip_ptr(lib.SOURCE_REF, h_basic.data_ptr())
        sf.render_clip_into(h_final.data_ptr())

    e2e_step()
    ranks.barrier()
    torch.cuda.synchronize()
    e2e_steps = max(1, min(args.steps, 5))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        e2e_step()
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_value = whole_job_rate(ranks.world, FRAMES, e2e_steps, ranks.max(e0.elapsed_time(e1)))
    # bit-equal for the exact form; the chosen forms add filtered rows into
    # the stacks with atomics, whose order (and so the last bits of a Basic
    # frame) varies from run to run, which can change a Final selection:
    # there the two Final outputs' PSNR must agree within 1e-3 dB
    if form == "plain":
        same = bool(torch.equal(h_final, d_final.cpu()))
    else:
        same = bool(abs(synth.psnr(h_final.numpy(), clean) - synth.psnr(final_out, clean)) <= 1e-3)

    # the chained render (vnlbgpu_render_chain_device), device-resident
    chain_step()
    torch.cuda.synchronize()
    c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    c0.record(stream)
    for _ in range(args.steps):
        chain_step()
    c1.record(stream)
    torch.cuda.synchronize()
    chain_value = whole_job_rate(ranks.world, FRAMES, args.steps, ranks.max(c0.elapsed_time(c1)))
    # bit-equal for the exact form; the chosen forms' Basic frames differ in
    # their last bits from run to run (atomic additions), which can change a
    # Final selection: there the chained output's PSNR must equal the
    # sequential one's within 1e-3 dB
    chained = d_final.cpu().numpy()
    chain_same = bool(np.array_equal(chained, final_out)) if form == "plain" else \
        bool(abs(synth.psnr(chained, clean) - synth.psnr(final_out, clean)) <= 1e-3)

    # One more device-resident step with one pipeline lane per session: the
    # anchor frames' kernels then run one after another, so each launch's
    # event-timed duration is that of the kernel alone (the roofline's
    # denominator); the timed steps above overlap up to eight lanes.
    for s in (sb, sf):
        s.set_lanes(1)
    step()
    torch.cuda.synchronize()
    stats1 = [sb.stats(), sf.stats()]
    sb.kernel_timing(True)
    sf.kernel_timing(True)
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    step()
    s1.record(stream)
    torch.cuda.synchronize()
    kb1, kf1 = sb.kernel_timing(False), sf.kernel_timing(False)
    stats2 = [sb.stats(), sf.stats()]
    serial_stats = {k: sum(stats2[i][k] - stats1[i][k] for i in range(2)) for k in stats0[0]}
    for s in (sb, sf):
        s.set_lanes(0)
    sb.close()
    sf.close()
    kernels = {k: (kb[k][0] + kf[k][0], kb[k][1] + kf[k][1]) for k in kb}
    serial = {"kernels": {k: (kb1[k][0] + kf1[k][0], kb1[k][1] + kf1[k][1]) for k in kb1},
              "basic": kb1, "final": kf1, "ms_per_step": s0.elapsed_time(s1), "stats": serial_stats,
              "basic_stats": {k: stats2[0][k] - stats1[0][k] for k in stats0[0]},
              "final_stats": {k: stats2[1][k] - stats1[1][k] for k in stats0[0]}}
    return {"form": form, "value": value, "max_ms": max_ms, "e2e": e2e_value, "same": same, "psnr": psnr,
            "kernels": kernels, "stats": delta, "lanes": lanes, "bp": bp,
            "serial": serial, "chain": {"value": chain_value, "output_matches_sequential": chain_same},
            "tuning": tuning,
            "outputs": (basic_out, final_out)}


def measure_frame_path(form, args, ranks, noisy, local, threads=8):
    """End to end through the per-frame drop-in path, as a VapourSynth script
    runs vnlbcu.Basic into vnlbcu.Final: `threads` frame threads per stage
    call vnlbgpu_render_frame_window with pageable host frames (one array per
    plane) and pageable outputs.  The clip is the workload's 16 frames played
    back and forth, (warmup + steps) * 16 frames per rank, so that every step
    is 16 new output frames of a long clip (the sessions' source stores and
    stack caches are bounded; frames already on the device are not copied
    again).  Under torchrun the ranks split this one clip by
    vnlbgpu_shard_plan: each renders its block of Final frames, the Basic
    frames they read and nothing else, with no exchange between ranks.  A
    Final frame starts once the Basic frames of its source window are out.

    Two phases on the same sessions: the first warmup * 16 Final frames (and
    the Basic frames they read), untimed; then the timed phase, every
    remaining Basic and Final frame, from a synchronised start with all
    threads idle to the last Final frame on the host: wall time, max over
    ranks.  The timed phase therefore holds all the work of its frames,
    including the ramp at its start."""
    import torch
    import vnlbgpu_lib as lib

    warm = max(1, args.warmup)
    per_rank = FRAMES * (warm + args.steps)
    total = per_rank * ranks.world
    frames = [[noisy[(f % FRAMES) if (f // FRAMES) % 2 == 0 else FRAMES - 1 - f % FRAMES][c] for c in range(PLANES)]
              for f in range(FRAMES * 2)]

    def src(f):
        return frames[f % (2 * FRAMES)]

    bp, fp = stage_params(lib.STAGE_BASIC, form), stage_params(lib.STAGE_FINAL, form)
    for p in (bp, fp):
        p.device_id = local
        p.num_streams = threads
    plan = lib.shard_plan(total, ranks.world, ranks.rank, (bp.search_bwd, bp.search_fwd, bp.patch_time),
                          (fp.search_bwd, fp.search_fwd, fp.patch_time))
    (o0, o1), (b0, b1) = plan["out"], plan["basic"]
    sb = lib.Session(bp, WIDTH, HEIGHT, total, PLANES)
    sf = lib.Session(fp, WIDTH, HEIGHT, total, PLANES)
    ring = 48  # Basic outputs kept for Final; Basic runs at most ring - 16 frames ahead
    basic_out = [np.empty((PLANES, HEIGHT, WIDTH), np.float32) for _ in range(ring)]
    final_out = [np.empty((PLANES, HEIGHT, WIDTH), np.float32) for _ in range(threads)]
    cond = threading.Condition()
    basic_done = set()
    state = {"final_done": o0}  # Final frames below this index are all out

    def run_phase(f_first, f_last):
        """Final frames f_first..f_last and the Basic frames they read that
        are not out yet."""
        need0 = sf.required_source_range(f_first)[0]
        need1 = sf.required_source_range(f_last)[1]
        todo_b = [m for m in range(max(b0, need0), min(b1, need1) + 1) if m not in basic_done]
        st = {"b": 0, "f": f_first, "error": None, "finished": set()}

        def basic_worker():
            try:
                while True:
                    with cond:
                        if st["b"] >= len(todo_b) or st["error"]:
                            return
                        n = todo_b[st["b"]]
                        st["b"] += 1
                        while n - state["final_done"] >= ring - 16 and not st["error"]:
                            cond.wait()
                    first, last = sb.required_source_range(n)
                    sb.render_frame_window(n, [src(f) for f in range(first, last + 1)], first=first,
                                           out=basic_out[n % ring])
                    with cond:
                        basic_done.add(n)
                        cond.notify_all()
            except Exception as e:  # noqa: BLE001 - re-raised below
                with cond:
                    st["error"] = e
                    cond.notify_all()

        def final_worker(slot):
            try:
                while True:
                    with cond:
                        n = st["f"]
                        if n > f_last or st["error"]:
                            return
                        st["f"] += 1
                    first, last = sf.required_source_range(n)
                    with cond:
                        while not all(f in basic_done for f in range(first, last + 1)) and not st["error"]:
                            cond.wait()
                    refs = [[basic_out[f % ring][c] for c in range(PLANES)] for f in range(first, last + 1)]
                    sf.render_frame_window(n, [src(f) for f in range(first, last + 1)], refs, first=first,
                                           out=final_out[slot])
                    with cond:
                        st["finished"].add(n)
                        while state["final_done"] in st["finished"]:
                            state["final_done"] += 1
                        cond.notify_all()
            except Exception as e:  # noqa: BLE001
                with cond:
                    st["error"] = e
                    cond.notify_all()

        pool = [threading.Thread(target=basic_worker) for _ in range(threads)]
        pool += [threading.Thread(target=final_worker, args=(i,)) for i in range(threads)]
        for t in pool:
            t.start()
        for t in pool:
            t.join()
        if st["error"]:
            raise st["error"]
        return len(todo_b)

    warm_last = min(o1, o0 + FRAMES * warm - 1)
    run_phase(o0, warm_last)
    torch.cuda.synchronize()
    ranks.barrier()
    t0 = time.perf_counter()
    basic_frames = run_phase(warm_last + 1, o1)
    torch.cuda.synchronize()
    seconds = ranks.max(time.perf_counter() - t0)
    timed = o1 - warm_last
    st_b, st_f = sb.stats(), sf.stats()
    sb.close()
    sf.close()
    return {"value": ranks.world * timed / seconds,
            "threads_per_stage": threads, "clip_frames": total, "timed_final_frames_per_rank": timed,
            "timed_basic_frames_per_rank": basic_frames,
            "shard": {"out": plan["out"], "basic": plan["basic"], "source": plan["source"]},
            "source_slots": {"basic": st_b["source_slots"], "final": st_f["source_slots"]},
            "anchor_frames": {"basic": st_b["anchor_frames"], "final": st_f["anchor_frames"]},
            "source_uploads": {"basic": st_b["source_uploads"], "final": st_f["source_uploads"]},
            "pipeline_lanes": {"basic": st_b["pipeline_lanes"], "final": st_f["pipeline_lanes"]}}


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per launch of each
# kernel class, from one ncu capture of the profile case at the workload's
# frame size (python bench.py --profile-case: one Basic and one Final anchor
# frame of a 3-frame 1920x1080 YUV444PS clip, CPU-default parameters), mean of
# the Basic and Final launches; the filter class sums prepare, Jacobi and
# apply.  None where no capture of the current kernels exists.
TRAFFIC_PER_LAUNCH = {
    ("cpu", "match/plain"): 57.4e6,        # match_kernel<8,0,0>: Basic 31.8 MB, Final 83.0 MB
    ("cpu", "match/chosen_tc"): 342.7e6,   # strip offsets + tc_distance + tc_select: 286.9 / 398.5 MB
    ("cpu", "filter/plain"): 492.8e6,      # prepare + jacobi + apply: Basic 402.0 MB, Final 583.6 MB
    ("cpu", "filter/chosen"): 503.9e6,     # the same, apply adding rows into pixel-interleaved stacks:
    ("cpu", "filter/chosen_tc"): 503.9e6,  # 415.3 / 592.5 MB
}
TRAFFIC_SOURCE = ("ncu --metrics gpu__time_duration.sum,dram__bytes_read.sum,dram__bytes_write.sum "
                  "--clock-control none python bench.py --profile-case --form chosen_tc (and --form plain)")


def roofline_of(r, steps, which=None):
    """Roofline of the dominant kernel class of one measured form (or of the
    class `which`), from the one-lane step: algorithmic work per launch over
    the mean event-timed duration of a launch running alone."""
    serial = r["serial"]
    kernels, st, bp = serial["kernels"], serial["stats"], r["bp"]
    dominant = which or max(("match", "filter"), key=lambda k: kernels[k][0])
    ms, launches = kernels[dominant]
    launches = max(1, launches)
    ms_launch = ms / launches
    anchor_frames = max(1, st["anchor_frames"])  # one match and one filter call per anchor frame and stage
    groups_per_frame = st["groups"] / anchor_frames
    window, temporal = bp.search_window, min(3, bp.search_bwd + bp.search_fwd + 1)
    dm_basic = bp.patch_size ** 2 * bp.patch_time
    dm_final = dm_basic * PLANES
    # per launch: a launch is one anchor frame of one stage; Basic and Final
    # launches alternate, so a mean launch has the mean match dimension
    dm_mean = 0.5 * (dm_basic + dm_final)
    common = {"ms_per_launch": ms_launch, "launches": launches,
              "timing": "CUDA events around each launch in a step with one pipeline lane per session (kernels "
                        "serialised), mean over the launches of the step",
              "serial_step_ms": serial["ms_per_step"]}
    traffic = TRAFFIC_PER_LAUNCH.get((PARAMS, dominant + "/" + r["form"]))
    if traffic is not None:
        common.update(traffic=traffic, traffic_unit="DRAM bytes per launch (ncu, one capture of the profile case)",
                      traffic_source=TRAFFIC_SOURCE)
    else:
        common.update(traffic=None)
    if dominant == "match" and r["form"] == "plain":
        ops = 3.0 * groups_per_frame * window * window * temporal * dm_mean
        return dict(common, kernel="match (exact FP32 SSD + selection replay)", bound="fp32",
                    achieved=ops / (ms_launch / 1e3) / 1e12, peak=FP32_LANE_OPS / 1e12, unit="TFLOP/s",
                    frac=ops / (ms_launch / 1e3) / FP32_LANE_OPS,
                    peak_source="nominal FP32 lane-op rate 148 SM x 128 x 1.965 GHz (MEASURED_PEAKS.json has no "
                                "FP32 figure)",
                    work="3 FP32 ops (sub, mul, add; no FMA, the CPU's order) per candidate element: G x W^2 x T x "
                         "d_m per launch (one anchor frame of one stage)")
    if dominant == "match" and r["form"] == "chosen":
        flops = 2.0 * groups_per_frame * window * window * temporal * dm_mean
        return dict(common, kernel="match, chosen form (FP32 dot-product distances + exact re-rank)", bound="fp32",
                    achieved=flops / (ms_launch / 1e3) / 1e12, peak=2 * FP32_LANE_OPS / 1e12, unit="TFLOP/s",
                    frac=flops / (ms_launch / 1e3) / (2 * FP32_LANE_OPS),
                    peak_source="nominal FP32 FMA rate x 2 (MEASURED_PEAKS.json has no FP32 figure)",
                    work="2 G C d_m (multiply-adds of all candidate dot products) per launch")
    if dominant == "match":
        flops = 2.0 * groups_per_frame * window * window * temporal * dm_mean
        peak = measured_peak("bf16_tflops", 1590.0)  # the kernel is timed alone: the burst figure
        return dict(common, kernel="match, chosen_tc form (tcgen05 BF16 distances into tensor memory, selection on "
                                   "them, exact FP32 re-rank)",
                    bound="tensor", achieved=flops / (ms_launch / 1e3) / 1e12, peak=peak, unit="TFLOP/s",
                    frac=flops / (ms_launch / 1e3) / 1e12 / peak,
                    peak_source="MEASURED_PEAKS.json bf16_tflops, burst (of measured)" if peak != 1590.0
                                else "fallback 1.59 PFLOP/s (of fallback)",
                    work="2 G C d_m (algorithmic multiply-adds of all candidate distances) per launch")
    # filter: Gram, basis, projections and reconstruction (FP32, exact)
    D, B, rk = dm_final, bp.similar, bp.rank
    act, rows = st["active_groups"] / anchor_frames, st["rows"] / anchor_frames
    flops = act * (B * (B + 1) * D + 2 * rk * B * D) + rows * 2 * rk * D * 2.5
    return dict(common, kernel="group filter (prepare + Jacobi + apply), one call per anchor frame and stage",
                bound="fp32", achieved=flops / (ms_launch / 1e3) / 1e12, peak=2 * FP32_LANE_OPS / 1e12,
                unit="TFLOP/s", frac=flops / (ms_launch / 1e3) / (2 * FP32_LANE_OPS),
                peak_source="nominal FP32 FMA rate x 2 (MEASURED_PEAKS.json has no FP32 figure)",
                work="Gram B(B+1)D + basis 2rBD per active group, projection and reconstruction 5rD per "
                     "retained row, per call")


def json_scalar(o):
    """numpy scalars (a comparison's bool, a PSNR) in the JSON line as Python values."""
    if isinstance(o, np.generic):
        return o.item()
    raise TypeError(f"{type(o).__name__} is not JSON serializable")


def measured_peak(key: str, fallback: float) -> float:
    try:
        with open(ROOT / "MEASURED_PEAKS.json") as f:
            v = json.load(f).get(key)
        return float(v) if v else fallback
    except (OSError, ValueError, TypeError):
        return fallback


# The other configurations of the workload list, measured beside the
# headline (device-resident, Basic then Final, in each listed form): frames/s
# with the same clock, PSNR against the clean clip.
EXTRA_WORKLOADS = {
    "gray_256x256x8_sigma10_cpu_defaults": dict(
        forms=["plain"], width=256, height=256, frames=8, planes=1, sigma=10.0, steps=20, warmup=3,
        basic=dict(CPU_DEFAULTS), final=dict(CPU_DEFAULTS, tau=400.0, variance_threshold=1.7)),
    "gray_1920x1080x32_sigma25_tau400_groups64": dict(
        forms=["plain", "chosen_tc"], width=1920, height=1080, frames=32, planes=1, sigma=25.0, steps=2, warmup=1,
        basic=dict(block_size=8, block_step=4, group_size=16, bm_range=9, radius=2, patch_time=2, rank=16,
                   cap_factor=4.0, tau=400.0),
        final=dict(block_size=8, block_step=4, group_size=16, bm_range=9, radius=2, patch_time=2, rank=16,
                   cap_factor=4.0, tau=400.0, variance_threshold=1.7)),
}


# the mixed stream: 4 GrayS 1280x720 + 2 YUV444PS 1920x1080 + 1 GrayS
# 3840x2160, 24 frames each, sigma cycling 5 / 15 / 30, tau 200, cap 4,
# patch_time 2, rank by noise level (24 at sigma 5, 16 at 15, 8 at 30) with a
# group of the same size (the rank is at most the group)
MIXED_STREAM = dict(
    clips=[(1280, 720, 1, 5.0), (1280, 720, 1, 15.0), (1280, 720, 1, 30.0), (1280, 720, 1, 5.0),
           (1920, 1080, 3, 15.0), (1920, 1080, 3, 30.0), (3840, 2160, 1, 15.0)],
    frames=24, steps=2, warmup=3, rank={5.0: 24, 15.0: 16, 30.0: 8},
    stage=dict(block_size=8, block_step=8, bm_range=9, radius=1, patch_time=2, cap_factor=4.0, tau=200.0))


def measure_mixed_stream(form, args, ranks, local):
    """Frames/s of the mixed stream in one form: every clip has its own Basic
    and Final sessions on its own CUDA stream, driven by its own host thread,
    all clips in flight at once; the step is the whole batch of clips, timed
    with events from one start event that every clip stream waits on to an
    end event that waits on every clip stream.  Chosen forms are autotuned
    per session before the timed steps."""
    import threading

    import torch
    import vnlbcu
    import vnlbgpu_lib as lib

    spec = MIXED_STREAM
    n = spec["frames"]
    clips = []
    for i, (w, h, c, sigma) in enumerate(spec["clips"]):
        clean, noisy = synth.make_clip(w, h, n, c, sigma, seed=100 * ranks.rank + i)
        shape = np.empty((n, c, h, w), np.float32)
        kw = dict(spec["stage"], rank=spec["rank"][sigma], group_size=spec["rank"][sigma], form=form)
        bp = vnlbcu.parse_parameters(lib.STAGE_BASIC, shape, sigma, dict(kw))
        fp = vnlbcu.parse_parameters(lib.STAGE_FINAL, shape, sigma, dict(kw, variance_threshold=None))
        bp.device_id = fp.device_id = local
        st = torch.cuda.Stream()
        d_noisy = torch.from_numpy(noisy).cuda()
        clip = dict(size=f"{w}x{h}x{c}", sigma=sigma, clean=clean, noisy=noisy, stream=st, d_noisy=d_noisy,
                    d_basic=torch.empty_like(d_noisy), d_final=torch.empty_like(d_noisy),
                    sb=lib.Session(bp, w, h, n, c), sf=lib.Session(fp, w, h, n, c), done=torch.cuda.Event())
        for s in (clip["sb"], clip["sf"]):
            s.set_stream(st.cuda_stream)
        clips.append(clip)

    def run(clip, start):
        if start is not None:
            clip["stream"].wait_event(start)
        sb, sf = clip["sb"], clip["sf"]
        sb.set_clip_device(lib.SOURCE_CLIP, clip["d_noisy"].data_ptr())
        sf.set_clip_device(lib.SOURCE_CLIP, clip["d_noisy"].data_ptr())
        sf.set_clip_device(lib.SOURCE_REF, clip["d_basic"].data_ptr())
        sb.render_clip_device(clip["d_basic"].data_ptr())
        sf.render_clip_device(clip["d_final"].data_ptr())
        clip["done"].record(clip["stream"])

    def step(start=None):
        errors = []

        def body(clip):
            try:
                run(clip, start)
            except Exception as e:  # re-raised on the calling thread
                errors.append(e)
        threads = [threading.Thread(target=body, args=(c,)) for c in clips]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        if errors:
            raise errors[0]

    step()
    torch.cuda.synchronize()
    tuning = []
    if form != "plain":
        for c in clips:
            tuning.append({"clip": c["size"], "basic": c["sb"].autotune(1)["match_warps"],
                           "final": c["sf"].autotune(1)["match_warps"]})
    for _ in range(spec["warmup"]):
        step()
    torch.cuda.synchronize()
    main = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ranks.barrier()
    torch.cuda.synchronize()
    e0.record(main)
    for _ in range(spec["steps"]):
        step(e0)
    for c in clips:
        main.wait_event(c["done"])
    e1.record(main)
    torch.cuda.synchronize()
    ms = ranks.max(e0.elapsed_time(e1))
    per_clip = []
    for c in clips:
        c["sb"].synchronize()
        c["sf"].synchronize()
        out = c["d_final"].cpu().numpy()
        per_clip.append({"clip": c["size"], "sigma": c["sigma"], "psnr_noisy_db": synth.psnr(c["noisy"], c["clean"]),
                         "psnr_final_db": synth.psnr(out, c["clean"]), "final": out})
        c["sb"].close()
        c["sf"].close()
    total = n * len(clips)
    return {"value": whole_job_rate(ranks.world, total, spec["steps"], ms), "unit": UNIT,
            "ms_per_step": ms / spec["steps"], "frames_per_step": total, "form": form, "clips": per_clip,
            "autotune": tuning}


def mixed_stream_line(args, ranks, local):
    """The mixed stream in the plain form and in the chosen_tc form, with each
    clip's PSNR change between the two (the chosen form's bar is 0.05 dB)."""
    plain = measure_mixed_stream("plain", args, ranks, local)
    tc = measure_mixed_stream("chosen_tc", args, ranks, local)
    clips = []
    for a, b in zip(plain["clips"], tc["clips"]):
        clips.append({"clip": a["clip"], "sigma": a["sigma"], "psnr_noisy_db": a["psnr_noisy_db"],
                      "psnr_plain_db": a["psnr_final_db"], "psnr_chosen_tc_db": b["psnr_final_db"],
                      "max_abs_vs_plain": float(np.max(np.abs(a["final"] - b["final"])))})
    return {"frames_per_step": plain["frames_per_step"], "steps": MIXED_STREAM["steps"],
            "warmup": MIXED_STREAM["warmup"], "plain": {"value": plain["value"], "ms_per_step": plain["ms_per_step"]},
            "chosen_tc": {"value": tc["value"], "ms_per_step": tc["ms_per_step"], "autotune": tc["autotune"]},
            "speedup_chosen_tc_vs_plain": tc["value"] / plain["value"],
            "max_psnr_loss_db": max(c["psnr_plain_db"] - c["psnr_chosen_tc_db"] for c in clips), "clips": clips,
            "params": dict(MIXED_STREAM["stage"], rank=MIXED_STREAM["rank"], group_size="= rank"), "unit": UNIT,
            "pipeline": "one host thread and one CUDA stream per clip, all clips in flight; not graph-captured"}


def workload_line(spec, args, ranks, stream, local):
    """One workload in each of its forms; with a chosen form beside the plain
    one, its speed-up and PSNR change against the plain form."""
    runs = {f: measure_workload(spec, args, ranks, stream, local, f) for f in spec["forms"]}
    out = dict(runs["plain"])
    for f, r in runs.items():
        if f == "plain":
            continue
        out[f + "_form"] = dict(r, speedup_vs_plain=r["value"] / out["value"],
                                psnr_loss_vs_plain_db=out["psnr_db"]["final"] - r["psnr_db"]["final"],
                                max_abs_vs_plain=float(np.max(np.abs(r.pop("final_out") - out["final_out"]))))
    out.pop("final_out")
    return out


def measure_workload(spec, args, ranks, stream, local, form="plain"):
    """Device-resident Basic + Final frames/s of one workload in one form
    (a chosen form autotuned per session first)."""
    import torch
    import vnlbcu
    import vnlbgpu_lib as lib

    w, h, n, planes, sigma = spec["width"], spec["height"], spec["frames"], spec["planes"], spec["sigma"]
    clean, noisy = synth.make_clip(w, h, n, planes, sigma, seed=ranks.rank)
    shape = np.empty((n, planes, h, w), np.float32)
    bp = vnlbcu.parse_parameters(lib.STAGE_BASIC, shape, sigma, dict(spec["basic"], form=form))
    fp = vnlbcu.parse_parameters(lib.STAGE_FINAL, shape, sigma, dict(spec["final"], form=form))
    bp.device_id = fp.device_id = local
    d_noisy = torch.from_numpy(noisy).cuda()
    d_basic, d_final = torch.empty_like(d_noisy), torch.empty_like(d_noisy)
    sb, sf = lib.Session(bp, w, h, n, planes), lib.Session(fp, w, h, n, planes)
    for s in (sb, sf):
        s.set_stream(stream.cuda_stream)

    def step():
        sb.set_clip_device(lib.SOURCE_CLIP, d_noisy.data_ptr())
        sf.set_clip_device(lib.SOURCE_CLIP, d_noisy.data_ptr())
        sf.set_clip_device(lib.SOURCE_REF, d_basic.data_ptr())
        sb.render_clip_device(d_basic.data_ptr())
        sf.render_clip_device(d_final.data_ptr())

    tuning = None
    if form != "plain":
        step()
        torch.cuda.synchronize()
        tuning = {"basic": sb.autotune(1)["match_warps"], "final": sf.autotune(1)["match_warps"]}
    for _ in range(spec["warmup"]):
        step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ranks.barrier()
    e0.record(stream)
    for _ in range(spec["steps"]):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    sb.synchronize()
    sf.synchronize()
    ms = ranks.max(e0.elapsed_time(e1))
    out = d_final.cpu().numpy()
    basic = d_basic.cpu().numpy()
    st = [sb.stats(), sf.stats()]
    sb.close()
    sf.close()
    return {"value": whole_job_rate(ranks.world, n, spec["steps"], ms), "unit": UNIT,
            "ms_per_step": ms / spec["steps"], "steps": spec["steps"], "warmup": spec["warmup"],
            "form": form, "autotune": tuning, "final_out": out,
            "params": {"basic": spec["basic"], "final": spec["final"]},
            "psnr_db": {"noisy": synth.psnr(noisy, clean), "basic": synth.psnr(basic, clean),
                        "final": synth.psnr(out, clean)},
            "rows_per_active_group": {"basic": st[0]["rows"] / max(1, st[0]["active_groups"]),
                                      "final": st[1]["rows"] / max(1, st[1]["active_groups"])}}


def reference_cuda_stages(head):
    """The reference's own CUDA stage kernels (src/cuda: block matcher with
    CUB sorts, group filter with cuBLAS and cuSOLVER, scatter aggregation),
    built for sm_100a by baseline/Makefile, timed by the reference's own
    stage benchmarks (tools/benchmark_cuda_*.cpp) at this workload's per
    anchor frame shapes, beside our kernels' one-lane per-launch times of the
    same run.  Their frames are 640x360 synthetic ones (the benchmarks' own);
    what carries over is the work per group: every grid anchor matched over
    19x19x3 candidates (K 8, buffer 32, patch 8), and every active group
    filtered (B 8, D 192, S the measured mean rows, rank 8) and scattered."""
    tools = ROOT / "baseline" / "_ref"
    if not (tools / "bench_block_match").exists():
        return {"unavailable": "baseline/_ref not built (make -C baseline needs the reference sources)"}
    serial = head["serial"]
    out = {"source": "reference src/cuda built for sm_100a (baseline/Makefile), timed by its "
                     "tools/benchmark_cuda_{block_match,group_filter,aggregation}.cpp; ours: one-lane event "
                     "times of this run, per launch (one anchor frame of one stage)"}

    def run(args_):
        try:
            r = subprocess.run([str(a) for a in args_], capture_output=True, text=True, timeout=300)
        except (OSError, subprocess.TimeoutExpired) as e:
            return None, str(e)
        if r.returncode != 0:
            return None, (r.stderr or r.stdout).strip()[-300:]
        for line in r.stdout.splitlines():
            if line.startswith("average batch:") or line.startswith("average clear+scatter:"):
                return float(line.split(":")[1].split()[0]), None
        return None, "no timing line"

    for stage, name in ((serial["basic_stats"], "basic"), (serial["final_stats"], "final")):
        frames = max(1, stage["anchor_frames"])
        groups = int(round(stage["groups"] / frames))
        active = int(round(stage["active_groups"] / frames))
        rows = stage["rows"] / max(1, stage["active_groups"])
        ours = serial[name]
        entry = {"grid_groups": groups, "active_groups": active, "mean_rows": rows}
        ms, err = run([tools / "bench_block_match", 8, groups, 20, name, "topk", 1, "contiguous", "--patch", 8,
                       "--channels", 3, "--window", 19, "--search-bwd", 1, "--search-fwd", 1, "--retained", 32])
        entry["match"] = {"reference_ms": ms, "ours_ms": ours["match"][0] / max(1, ours["match"][1])}
        if err:
            entry["match"]["error"] = err
        # the filter benchmark runs the reference's Basic-stage filter
        ms, err = run([tools / "bench_group_filter", 8, 192, min(32, max(8, int(round(rows)))), active, 20, 8])
        entry["filter"] = {"reference_ms": ms, "ours_ms": ours["filter"][0] / max(1, ours["filter"][1])}
        if err:
            entry["filter"]["error"] = err
        ms, err = run([tools / "bench_aggregation", min(32, max(8, int(round(rows)))), 32, active, 20, 1, "k",
                       "spread"])
        tiles_ms = ours["tiles"][0] / ours["tiles"][1] if ours["tiles"][1] else 0.0
        entry["aggregate"] = {"reference_ms": ms,
                              "ours_ms": tiles_ms + ours["normalize"][0] / max(1, ours["normalize"][1]),
                              "ours_kernels": "stack tiles + normalise" if ours["tiles"][1] else
                              "normalise (the chosen form adds the rows into the stacks inside the filter's apply "
                              "kernel, timed with the filter)"}
        if err:
            entry["aggregate"]["error"] = err
        for k in ("match", "filter", "aggregate"):
            e = entry[k]
            if e.get("reference_ms") and e.get("ours_ms"):
                e["speedup"] = e["reference_ms"] / e["ours_ms"]
        out[name] = entry
    return out


def run_ours(args):
    import torch

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    ranks = RankGroup("nccl", torch.device("cuda", local))
    rank, world = ranks.rank, ranks.world

    clean, noisy = synth.make_clip(WIDTH, HEIGHT, FRAMES, PLANES, SIGMA, seed=rank)
    clip_bytes = noisy.nbytes
    d_noisy = torch.from_numpy(noisy).cuda()
    # one dedicated stream for both stages: Final is ordered after the Basic
    # frames it reads, and the timing events see all of the work
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    forms = ["plain", "chosen", "chosen_tc"] if args.form == "all" else [args.form]
    if PARAMS == "vnlbcu":
        forms = [f for f in forms if f != "chosen"]
    # clocks sampled over every timed measurement below (the GPU is busy from
    # the first warm-up step to the last frame of the per-frame run)
    with ClockSampler(local) as clocks:
        results = {f: measure_form(f, args, ranks, stream, noisy, clean, d_noisy, local) for f in forms}
        head = results[forms[-1]]
        frame_path = None
        if not args.no_frame_path:
            frame_path = measure_frame_path(head["form"], args, ranks, noisy, local)
    reference_cuda = None
    if rank == 0 and not args.no_reference_cuda and PARAMS == "cpu":
        reference_cuda = reference_cuda_stages(head)
    workloads = {}
    if not args.no_workloads and PARAMS == "cpu":
        for name, spec in EXTRA_WORKLOADS.items():
            workloads[name] = workload_line(spec, args, ranks, stream, local)
        workloads["mixed_stream_7_clips_24f"] = mixed_stream_line(args, ranks, local)
    per_kernel = {}
    total_kernel_ms = sum(v[0] for v in head["kernels"].values())
    for k, v in head["kernels"].items():
        per_kernel[k] = {"ms_per_step": v[0] / args.steps, "launches": v[1],
                         "share": v[0] / total_kernel_ms if total_kernel_ms else None}
    roofline = roofline_of(head, args.steps)

    cpu_baseline = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and PARAMS == "cpu":
        _, kind, threads, fraction, cstep, sample = cpu_reference_sample()
        cstep()
        c0 = time.perf_counter()
        cstep()
        cs = time.perf_counter() - c0
        cpu_baseline = {"value": threads * fraction / cs, "unit": UNIT, "cores": threads, "kind": kind,
                        "sample": sample}

    if rank == 0:
        describe = {"plain": "plain (exact, bit-identical to the CPU core)",
                    "chosen": "chosen (selection on FP32 dot-product distances, exact FP32 re-rank)",
                    "chosen_tc": "chosen_tc (selection on BF16 tcgen05 tensor-core distances, exact FP32 re-rank)"}
        config = dict(workload_config(describe[head["form"]]), psnr_db=head["psnr"], kernels=per_kernel,
                      dominant_kernel=roofline["kernel"], e2e_output_matches_device_output=head["same"],
                      e2e_output_check="bit-equal" if head["form"] == "plain" else
                      "Final PSNR within 1e-3 dB (atomic additions' order varies between runs)",
                      pipeline_lanes=head["lanes"])
        if "plain" in results and head["form"] != "plain":
            plain = results["plain"]
            config["plain_form"] = {"value": plain["value"], "e2e": plain["e2e"], "psnr_db": plain["psnr"],
                                    "ms_per_step": plain["max_ms"] / args.steps}
            config["speedup_vs_plain"] = head["value"] / plain["value"]
            config["psnr_loss_db_vs_plain"] = {s: plain["psnr"][s] - head["psnr"][s] for s in ("basic", "final")}
            config["max_abs_vs_plain"] = {
                s: float(np.max(np.abs(a - b))) for s, a, b in
                zip(("basic", "final"), head["outputs"], plain["outputs"])}
        for f, other in results.items():
            if f in ("plain", head["form"]):
                continue
            config[f + "_form"] = {"value": other["value"], "e2e": other["e2e"], "psnr_db": other["psnr"],
                                   "ms_per_step": other["max_ms"] / args.steps,
                                   "match_ms_per_step": other["kernels"]["match"][0] / args.steps}
        if head["form"] != "plain" and not roofline["kernel"].startswith("match"):
            config["match_roofline"] = roofline_of(head, args.steps, which="match")
        e2e_whole = {"value": head["e2e"], "unit": UNIT, "h2d_bytes_per_step": 3 * clip_bytes,
                     "d2h_bytes_per_step": 2 * clip_bytes,
                     "api": "vnlbgpu_set_clip_host + vnlbgpu_render_clip_host per stage (whole clip, pinned host "
                            "buffers), CUDA events on the sessions' stream"}
        config["chain"] = dict(head["chain"], api="vnlbgpu_render_chain_device (Basic into Final, stages "
                                                      "overlapped on the device), device-resident")
        config["autotune"] = head["tuning"]
        if workloads:
            config["workloads"] = workloads
        if reference_cuda is not None:
            config["reference_cuda"] = reference_cuda
        if frame_path is not None:
            e2e = dict(value=frame_path["value"], unit=UNIT, h2d_bytes_per_step=3 * clip_bytes,
                       d2h_bytes_per_step=2 * clip_bytes,
                       api="vnlbgpu_render_frame_window per output frame (the plugin's getFrame), pageable host "
                           "frames, eight frame threads per stage; wall time, synchronised, max over ranks")
            config["e2e_frame_path"] = frame_path
            config["e2e_whole_clip"] = e2e_whole
        else:
            e2e = e2e_whole
        line = {"metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": head["max_ms"] / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "bf16+f32" if head["form"] == "chosen_tc" else "f32",
                "data": "synthetic", "config": config, "roofline": roofline, "cpu_baseline": cpu_baseline,
                "e2e": e2e,
                "gpu_launches": head["stats"]["kernel_launches"], "clocks": clocks.summary()}
        print(json.dumps(line, default=json_scalar), flush=True)
    ranks.close()
    return 0


def run_learned(args):
    """Learned block-match proposals at a 33 x 33 x 5 window (bm_range 16,
    radius 2), 1920x1080 YUV444PS, sigma 20, the CPU defaults otherwise: one
    network per stage, trained by the library's kernels on the full search's
    top-8 offsets of independently seeded clips (every grid anchor of
    `--learned-train-frames` anchor frames per clip, two clips), then the
    clip rendered (device-resident, Basic then Final, 16 frames) by the full
    search and by the learned form at recall thresholds 0.9 (the per-tile
    check decides) and 0 (the learned rows always stand).  Prints one JSON
    line: frames/s, PSNR, held-out recall, share of tiles kept."""
    import torch
    import learned as LR
    import vnlbgpu_lib as lib

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    kw = dict(CPU_DEFAULTS, bm_range=16, radius=2)
    stage_kw = {lib.STAGE_BASIC: dict(kw, variance_threshold=1.1, weight_alpha=0.75, weight_beta=0.35,
                                      weight_gamma=1.0),
                lib.STAGE_FINAL: dict(kw, tau=400.0, variance_threshold=1.7, flat_areas=1, weight_alpha=1.0,
                                      weight_beta=0.5, weight_gamma=1.0)}
    frames_train = args.learned_train_frames
    clips = LR.synthetic_clips(WIDTH, HEIGHT, frames_train, PLANES, SIGMA, seeds=(1001, 1002))
    refs = [LR.session(lib.STAGE_BASIC, c, SIGMA, stage_kw[lib.STAGE_BASIC]).render_clip() for c in clips]
    clean, noisy = synth.make_clip(WIDTH, HEIGHT, FRAMES, PLANES, SIGMA, seed=0)
    nets, train_info = {}, {}
    for stage in (lib.STAGE_BASIC, lib.STAGE_FINAL):
        feats, targets = LR.training_pairs(stage, clips, SIGMA, stage_kw[stage],
                                           refs if stage == lib.STAGE_FINAL else None)
        inputs, outputs = LR.network_shape(stage, PLANES, stage_kw[stage], noisy, SIGMA)
        net = lib.MLP(inputs, 128, 3, outputs, max_batch=4096, seed=7 + stage)
        t0 = time.perf_counter()
        losses = LR.train(net, feats, targets, steps=args.learned_steps, batch=4096, lr=1e-3)
        torch.cuda.synchronize()
        train_s = time.perf_counter() - t0
        nets[stage] = net
        train_info[stage] = {"pairs": int(feats.shape[0]), "steps": args.learned_steps, "batch": 4096,
                             "seconds": train_s, "loss_first": float(np.mean(losses[:10])),
                             "loss_last": float(np.mean(losses[-10:]))}

    def render(form, threshold=None):
        sb = LR.session(lib.STAGE_BASIC, noisy, SIGMA, stage_kw[lib.STAGE_BASIC], form=form)
        if form == "learned":
            sb.set_learned(nets[lib.STAGE_BASIC], 64, threshold, 64)
        basic = sb.render_clip()  # warm-up: grids, buffers
        sf = LR.session(lib.STAGE_FINAL, noisy, SIGMA, stage_kw[lib.STAGE_FINAL], ref=basic, form=form)
        if form == "learned":
            sf.set_learned(nets[lib.STAGE_FINAL], 64, threshold, 64)
        sf.render_clip()
        st0 = [sb.stats(), sf.stats()]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            sb.set_clip(lib.SOURCE_CLIP, noisy)
            basic = sb.render_clip()
            sf.set_clip(lib.SOURCE_CLIP, noisy)
            sf.set_clip(lib.SOURCE_REF, basic)
            final = sf.render_clip()
        seconds = (time.perf_counter() - t0) / args.steps
        st = [sb.stats(), sf.stats()]
        tiles = sum(st[i]["learned_tiles"] - st0[i]["learned_tiles"] for i in range(2))
        fell = sum(st[i]["learned_fallback_tiles"] - st0[i]["learned_fallback_tiles"] for i in range(2))
        sb.close()
        sf.close()
        return {"value": FRAMES / seconds, "ms_per_step": seconds * 1e3,
                "psnr_db": {"basic": synth.psnr(basic, clean), "final": synth.psnr(final, clean)},
                "tiles_checked": tiles, "tiles_kept": tiles - fell}

    hold = {}
    for stage in (lib.STAGE_BASIC, lib.STAGE_FINAL):
        ref = None
        if stage == lib.STAGE_FINAL:
            ref = LR.session(lib.STAGE_BASIC, noisy, SIGMA, stage_kw[lib.STAGE_BASIC]).render_clip()
        f, t = LR.training_pairs(stage, [noisy], SIGMA, stage_kw[stage], [ref] if ref is not None else None)
        hold[stage] = LR.recall(nets[stage], f, t, 64)
    out = {"metric": "learned block-match proposals, 1080p YUV444PS Basic+Final frames/s at bm_range 16, radius 2",
           "unit": UNIT, "steps": args.steps, "timing": "host wall time around whole-clip host renders",
           "full_search": render("plain"), "learned_threshold_0.9": render("learned", 0.9),
           "learned_threshold_0": render("learned", 0.0),
           "held_out_recall_at_64": {"basic": hold[lib.STAGE_BASIC], "final": hold[lib.STAGE_FINAL]},
           "training": {"basic": train_info[lib.STAGE_BASIC], "final": train_info[lib.STAGE_FINAL]}}
    print(json.dumps(out, default=json_scalar), flush=True)
    return 0


def run_profile_case(args):
    """A small case for ncu: one Basic and one Final anchor frame of a
    3-frame YUV444PS clip (the workload's frame size unless --profile-size
    gives a smaller one, and its parameters), each stage launching every
    kernel class once."""
    import vnlbgpu_lib as lib

    width, height = WIDTH, HEIGHT
    if args.profile_size:
        width, height = (int(v) for v in args.profile_size.lower().split("x"))
    if args.learned:
        return run_learned_profile_case(width, height)
    _, noisy = synth.make_clip(width, height, 3, PLANES, SIGMA, seed=0)
    shape = np.empty((3, PLANES, height, width), np.float32)
    out = []
    for stage in (lib.STAGE_BASIC, lib.STAGE_FINAL):
        import vnlbcu
        form = args.form if args.form != "all" else "plain"
        if PARAMS == "vnlbcu":
            kw = dict(form=form)
        else:
            kw = dict(CPU_DEFAULTS, form=form)
            if stage == lib.STAGE_FINAL:
                kw.update(tau=400.0, variance_threshold=1.7)
            else:
                kw.update(variance_threshold=1.1)
        s = lib.Session(vnlbcu.parse_parameters(stage, shape, SIGMA, kw), width, height, 3, PLANES)
        s.set_clip(lib.SOURCE_CLIP, noisy)
        if stage == lib.STAGE_FINAL:
            s.set_clip(lib.SOURCE_REF, noisy)
        out.append(float(s.render_stack(1).sum()))
        s.close()
    print(json.dumps({"profile_case": "ok", "checksums": out}))
    return 0


def run_learned_profile_case(width, height):
    """The learned form's small case for ncu (--learned --profile-case): the
    contribution stack of anchor frame 2 of a 5-frame YUV444PS clip, Basic,
    bm_range 16, radius 2, with an untrained network of the trained one's
    shape and the learned rows always kept (threshold 0), then the same
    anchor frame by the full search; the network's work does not depend on
    its weights."""
    import learned as LR
    import vnlbgpu_lib as lib

    kw = dict(CPU_DEFAULTS, bm_range=16, radius=2, variance_threshold=1.1)
    _, noisy = synth.make_clip(width, height, 5, PLANES, SIGMA, seed=0)
    inputs, outputs = LR.network_shape(lib.STAGE_BASIC, PLANES, kw, noisy, SIGMA)
    net = lib.MLP(inputs, 128, 3, outputs, max_batch=4096, seed=3)
    out = []
    for form in ("learned", "plain"):
        s = LR.session(lib.STAGE_BASIC, noisy, SIGMA, kw, form=form)
        if form == "learned":
            s.set_learned(net, 64, 0.0, 64)
        out.append(float(s.render_stack(2).sum()))
        s.close()
    print(json.dumps({"profile_case": "ok", "form": "learned then plain", "checksums": out}))
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-reference-cuda", action="store_true",
                    help="skip timing the reference's own CUDA stage kernels (baseline/_ref, if built)")
    ap.add_argument("--no-workloads", action="store_true",
                    help="skip the other workload configurations measured beside the headline")
    ap.add_argument("--no-frame-path", action="store_true",
                    help="skip the end-to-end run through the per-frame path (vnlbgpu_render_frame_window)")
    ap.add_argument("--form", choices=("all", "plain", "chosen", "chosen_tc"), default="all",
                    help="matcher form(s) to time; with all, the tensor-core form (chosen_tc) is the headline "
                         "and the plain and FP32 chosen forms are measured beside it for the speed-up and the PSNR "
                         "gate")
    ap.add_argument("--profile-case", action="store_true",
                    help="run only a small case (one anchor frame per stage) for ncu captures")
    ap.add_argument("--profile-size", default=None, metavar="WxH",
                    help="frame size of the profile case (default: the workload's 1920x1080)")
    ap.add_argument("--learned", action="store_true",
                    help="measure the learned block-match proposals at bm_range 16, radius 2 instead")
    ap.add_argument("--learned-train-frames", type=int, default=30,
                    help="frames per training clip (two clips) for --learned; 30 gives about 2e6 (anchor, "
                         "top-8) pairs at 1080p")
    ap.add_argument("--learned-steps", type=int, default=600, help="Adam steps per network for --learned")
    ap.add_argument("--params", choices=("cpu", "vnlbcu"), default="cpu",
                    help="parameter set: the CPU core's defaults (the headline) or vnlbcu's own defaults")
    args = ap.parse_args()
    global PARAMS
    PARAMS = args.params
    if args.profile_case:
        return run_profile_case(args)
    if args.learned:
        return run_learned(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
