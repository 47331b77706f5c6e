"""Builds the native library of the B200 VNLB path in the source tree.

    python vapoursynth-vnlb_b200/build_native.py

compiles csrc/*.cu and csrc/session.cpp for sm_100a into
vapoursynth-vnlb_b200/lib/libvnlbgpu.so.  Floating-point contraction is off
(--fmad=false, -ffp-contract=off): the plain path states every fused
multiply-add explicitly, so that its arithmetic matches the reference CPU core
operation for operation.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB_DIR = PKG / "lib"
LIB = LIB_DIR / "libvnlbgpu.so"
SOURCES = ["match.cu", "match_chosen.cu", "paste.cu", "filter.cu", "aggregate.cu", "aggregate_noalloc.cu",
           "learned.cu", "session.cpp", "mlp.cpp", "mvtools.cpp", "smem_limit.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def build(verbose: bool = False, ptxas_info: bool = False, out: Path | None = None,
          defines: tuple[str, ...] = ()) -> Path:
    """Compiles the library to `out` (default lib/libvnlbgpu.so); `defines`
    are extra -D macros for a variant build."""
    lib = Path(out) if out else LIB
    lib.parent.mkdir(parents=True, exist_ok=True)
    LIB_DIR.mkdir(exist_ok=True)
    objs = []
    common = ARCH + ["-O3", "-lineinfo", "-std=c++17", "--fmad=false", "-Xcompiler", "-fPIC,-ffp-contract=off",
                     "-I", str(PKG.parent / "include")]
    if ptxas_info:
        common += ["-Xptxas", "-v"]
    common += [f"-D{d}" for d in defines]
    build_dir = PKG / "_build" / ("variant_" + lib.stem if out else "default")
    build_dir.mkdir(parents=True, exist_ok=True)
    for src in SOURCES:
        obj = build_dir / (Path(src).stem + ".o")
        cmd = [nvcc(), "-c", str(CSRC / src), "-o", str(obj)] + common
        if src.endswith(".cpp"):
            cmd += ["-x", "cu"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        objs.append(str(obj))
    cmd = [nvcc(), "-shared", "-o", str(lib)] + ARCH + [*objs, "-cudart", "static"]
    subprocess.run(cmd, check=True)
    return lib


if __name__ == "__main__":
    build(verbose=True, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
