"""Regenerates the golden fixtures of tests/golden/ (run in the build container,
where the reference sources and the oracle build exist):

    make -C oracle ref && python tests/golden/make_golden.py

reference_cases.npz
    The reference's own end-to-end fixtures (tests/reference_cases/*/:
    input.npz, basic_ref.npz, final_ref.npz and case.toml), produced by the
    original pariasm/vnlb implementation, repacked into one file with their
    parameters and tolerances.  They pin the oracle at the reference's own
    (loose) tolerance.

ref_outputs.npz
    Small seeded synthetic clips and the Basic/Final outputs of the reference's
    CPU core built out of tree (oracle/_ref/libvnlb_ref.so; the
    Basic -> Aggregate -> Final -> Aggregate chain of the vnlb plugin).  They
    pin the C restatement and the GPU path bit for bit without the reference
    sources being present.

flow_outputs.npz
    The same with the vnlb plugin's mvfw / mvbw MVTools clips: seeded random
    vectors, some frames invalid or marked as scene changes
    (tests/mvtools_blobs.py), and the aggregated Basic and Final outputs of the
    reference's flow-guided search (process_*_anchor_mvtools; the Basic ->
    Aggregate -> Final -> Aggregate chain).  The clips and vectors are
    regenerated from the seeds by tests/mvtools_blobs.flow_case.
"""
from __future__ import annotations

import json
import os
import sys
import tomllib
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT / "vapoursynth-vnlb_b200"))
sys.path.insert(0, str(ROOT / "tests"))

import oracle as O  # noqa: E402
import mvtools_blobs as M  # noqa: E402
import synth  # noqa: E402

REFERENCE = Path(os.environ.get("VNLB_REFERENCE", "/root/reference"))
OUT = Path(__file__).resolve().parent

# (name, width, height, frames, planes, sigma, seed, shared kwargs, basic extra, final extra)
SYNTHETIC_CASES = [
    ("gray_cpu_defaults", 64, 48, 5, 1, 20.0, 11, {}, {}, {}),
    ("yuv_cpu_defaults", 48, 40, 4, 3, 20.0, 12, {}, {}, {}),
    ("yuv_cuda_like", 48, 40, 4, 3, 20.0, 13,
     dict(block_size=7, patch_time=2, bm_range=6, group_size=16, rank=15, block_step=3), {}, {}),
    ("gray_tau_cap_pt2", 64, 48, 6, 1, 25.0, 14,
     dict(block_size=8, patch_time=2, radius=2, block_step=4, group_size=16, rank=16, cap_factor=4.0),
     dict(tau=400.0), {}),
    ("yuv_unwindowed_rank0", 40, 40, 3, 3, 15.0, 15,
     dict(weight_gamma=0.0, rank=0), {}, {}),
]


def reference_cases():
    cases = sorted(p for p in (REFERENCE / "tests" / "reference_cases").iterdir() if p.is_dir())
    arrays, meta = {}, {}
    for case in cases:
        with (case / "case.toml").open("rb") as f:
            info = tomllib.load(f)
        with np.load(case / "input.npz") as d:
            arrays[f"{case.name}/noisy"] = np.asarray(d["noisy"], np.float32)
        with np.load(case / "basic_ref.npz") as d:
            arrays[f"{case.name}/basic"] = np.asarray(d["basic"], np.float32)
        with np.load(case / "final_ref.npz") as d:
            arrays[f"{case.name}/final"] = np.asarray(d["final"], np.float32)
        meta[case.name] = {"noise": info["noise"], "vnlb": info["vnlb"], "tolerance": info["tolerance"],
                           "reference": {"implementation": info["reference"]["implementation"],
                                         "commit": info["reference"]["commit"]}}
    np.savez_compressed(OUT / "reference_cases.npz", meta=json.dumps(meta), **arrays)


def ref_outputs():
    o = O.Oracle("ref")
    arrays, meta = {}, {}
    for name, w, h, f, planes, sigma, seed, shared, b_extra, f_extra in SYNTHETIC_CASES:
        _, noisy = synth.make_clip(w, h, f, planes, sigma, seed=seed)
        bp = O.cpu_params(O.BASIC, sigma, **shared, **b_extra)
        fp = O.cpu_params(O.FINAL, sigma, **shared, **f_extra)
        basic, final = o.chain(noisy, bp, fp)
        arrays[f"{name}/noisy"] = noisy
        arrays[f"{name}/basic"] = basic
        arrays[f"{name}/final"] = final
        meta[name] = {"sigma": sigma, "shared": shared, "basic": b_extra, "final": f_extra}
    np.savez_compressed(OUT / "ref_outputs.npz", meta=json.dumps(meta), **arrays)


def flow_outputs():
    o = O.Oracle("ref")
    arrays, meta = {}, {}
    for case in M.FLOW_CASES:
        name, w, h, f, planes, sigma, seed, kw, fw_spec, bw_spec = case
        noisy, fw, bw = M.flow_case(*case)
        flow = (M.flow_grids(fw), M.flow_grids(bw))
        bp = O.cpu_params(O.BASIC, sigma, **kw)
        fp = O.cpu_params(O.FINAL, sigma, **kw)
        bs = o.stage_stacks(O.BASIC, bp, noisy, flow=flow)
        basic = o.aggregate(bs, noisy, bp.search_bwd, bp.search_fwd, bp.patch_time)
        fs = o.stage_stacks(O.FINAL, fp, noisy, basic, flow=flow)
        final = o.aggregate(fs, noisy, fp.search_bwd, fp.search_fwd, fp.patch_time)
        arrays[f"{name}/basic"] = basic
        arrays[f"{name}/final"] = final
        meta[name] = {"sigma": sigma, "kwargs": kw}
    np.savez_compressed(OUT / "flow_outputs.npz", meta=json.dumps(meta), **arrays)


if __name__ == "__main__":
    reference_cases()
    ref_outputs()
    flow_outputs()
    for p in ("reference_cases.npz", "ref_outputs.npz", "flow_outputs.npz"):
        print(p, (OUT / p).stat().st_size, "bytes")
