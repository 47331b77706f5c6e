"""ctypes access to the CPU oracles of the VNLB hot path.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py, always as the checker.  The product
(vapoursynth-vnlb_b200/) never imports this module.

Two libraries expose the same C interface (oracle/vnlb_oracle.h):
  * "ref"    oracle/_ref/libvnlb_ref.so, the reference's own src/core,
             src/linalg and src/aggregate compiled by oracle/Makefile;
  * "port"   oracle/libvnlb_oracle.so, the plain-C restatement vnlb_oracle.c.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, fields, replace
from pathlib import Path

import numpy as np

ORACLE_DIR = Path(__file__).resolve().parent
REF_LIB = ORACLE_DIR / "_ref" / "libvnlb_ref.so"
REF_GLIBC_LIB = ORACLE_DIR / "_ref" / "libvnlb_ref_glibc.so"
PORT_LIB = ORACLE_DIR / "libvnlb_oracle.so"

BASIC, FINAL = 0, 1
EIGHT_BIT = 255.0


class _CParams(ctypes.Structure):
    _fields_ = [
        ("sigma", ctypes.c_float), ("patch_size", ctypes.c_int),
        ("patch_time", ctypes.c_int), ("search_window", ctypes.c_int),
        ("search_bwd", ctypes.c_int), ("search_fwd", ctypes.c_int),
        ("similar", ctypes.c_int), ("rank", ctypes.c_int),
        ("similar_cap_factor", ctypes.c_float),
        ("model_cap_factor", ctypes.c_float), ("beta", ctypes.c_float),
        ("tau", ctypes.c_float), ("variance_threshold", ctypes.c_float),
        ("sigma_basic", ctypes.c_float), ("gamma", ctypes.c_float),
        ("weight_alpha", ctypes.c_float), ("weight_beta", ctypes.c_float),
        ("weight_gamma", ctypes.c_float), ("weight_epsilon", ctypes.c_float),
        ("membership_noise_floor", ctypes.c_float),
        ("proc_step", ctypes.c_int), ("flat_areas", ctypes.c_int),
        ("couple_channels", ctypes.c_int),
    ]


@dataclass(frozen=True)
class StageParams:
    """vnlb::core::StageParameters (src/core/core.hpp:17-41), core units."""
    sigma: float = 1.0
    patch_size: int = 8
    patch_time: int = 1
    search_window: int = 19
    search_bwd: int = 1
    search_fwd: int = 1
    similar: int = 8
    rank: int = 8
    similar_cap_factor: float = 4.0
    model_cap_factor: float = 1.0
    beta: float = 1.0
    tau: float = 0.0
    variance_threshold: float = 1.1
    sigma_basic: float = 0.0
    gamma: float = 0.95
    weight_alpha: float = 0.75
    weight_beta: float = 0.35
    weight_gamma: float = 1.0
    weight_epsilon: float = 1.0e-6
    membership_noise_floor: float = 0.25
    proc_step: int = 8
    flat_areas: int = 0
    couple_channels: int = 1

    def to_c(self) -> _CParams:
        return _CParams(*[getattr(self, f.name) for f in fields(self)])

    @property
    def slots(self) -> int:
        return self.search_bwd + self.search_fwd + self.patch_time


class _CFlowGrids(ctypes.Structure):
    _fields_ = [("present", ctypes.c_int), ("block_size_x", ctypes.c_int), ("block_size_y", ctypes.c_int),
                ("pel", ctypes.c_int), ("overlap_x", ctypes.c_int), ("overlap_y", ctypes.c_int),
                ("block_count_x", ctypes.c_int), ("block_count_y", ctypes.c_int),
                ("usable", ctypes.POINTER(ctypes.c_ubyte)), ("vectors", ctypes.POINTER(ctypes.c_int))]


class _CFlow(ctypes.Structure):
    _fields_ = [("fw", _CFlowGrids), ("bw", _CFlowGrids)]


@dataclass(frozen=True)
class FlowGrids:
    """One direction of motion vectors (vnlb_flow_grids, oracle/vnlb_oracle.h):
    the MVTools block geometry, a usable flag per frame and the finest-level
    vectors [frames][block_count_y][block_count_x][2] in sub-pel units."""
    block_size_x: int
    block_size_y: int
    pel: int
    overlap_x: int
    overlap_y: int
    usable: np.ndarray
    vectors: np.ndarray


def c_flow(fw: FlowGrids | None, bw: FlowGrids | None):
    """-> (vnlb_flow, the arrays it points into)."""
    keep = []

    def grids(g):
        if g is None:
            return _CFlowGrids()
        usable = np.ascontiguousarray(g.usable, dtype=np.uint8)
        vectors = np.ascontiguousarray(g.vectors, dtype=np.int32)
        keep.extend([usable, vectors])
        return _CFlowGrids(1, g.block_size_x, g.block_size_y, g.pel, g.overlap_x, g.overlap_y, vectors.shape[2],
                           vectors.shape[1], usable.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)),
                           vectors.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))

    return _CFlow(grids(fw), grids(bw)), keep


def cpu_params(stage: int, sigma: float, **kw) -> StageParams:
    """The vnlb.Basic / vnlb.Final argument rules of parse_stage_parameters
    (src/vs/plugin.cpp:372-449): 8-bit sigma and tau, radius, bm_range and the
    Final-stage default overrides."""
    p = StageParams(sigma=np.float32(sigma) / np.float32(EIGHT_BIT))
    if stage == FINAL:
        p = replace(p, tau=float(np.float32(400.0) / np.float32(EIGHT_BIT * EIGHT_BIT)),
                    variance_threshold=1.7, flat_areas=1, weight_alpha=1.0,
                    weight_beta=0.5, weight_gamma=1.0)
    kw = dict(kw)
    mapping = {"block_size": "patch_size", "group_size": "similar",
               "cap_factor": "similar_cap_factor", "block_step": "proc_step",
               "chroma": "couple_channels"}
    if "radius" in kw:
        r = kw.pop("radius")
        p = replace(p, search_bwd=r, search_fwd=r)
    if "bm_range" in kw:
        p = replace(p, search_window=2 * kw.pop("bm_range") + 1)
    if "tau" in kw:
        p = replace(p, tau=float(np.float32(kw.pop("tau")) / np.float32(EIGHT_BIT * EIGHT_BIT)))
    if "sigma_basic" in kw:
        p = replace(p, sigma_basic=float(np.float32(kw.pop("sigma_basic")) / np.float32(EIGHT_BIT)))
    for key, value in kw.items():
        p = replace(p, **{mapping.get(key, key): value})
    return p


class Oracle:
    def __init__(self, kind: str = "port"):
        path = {"ref": REF_LIB, "ref_glibc": REF_GLIBC_LIB, "port": PORT_LIB}[kind]
        if not path.exists():
            raise FileNotFoundError(f"oracle library {path} is not built (make -C oracle)")
        self.kind = kind
        self.prefix = "vnlbref_" if kind.startswith("ref") else "vnlboracle_"
        self.lib = ctypes.CDLL(str(path))
        getattr(self.lib, self.prefix + "last_error").restype = ctypes.c_char_p

    def _fn(self, name):
        return getattr(self.lib, self.prefix + name)

    def _check(self, status: int):
        if status != 0:
            raise ValueError(self._fn("last_error")().decode())

    @staticmethod
    def _ptr(array):
        if array is None:
            return None
        return array.ctypes.data_as(ctypes.POINTER(ctypes.c_float))

    def stage_stacks(self, stage: int, params: StageParams, clip: np.ndarray,
                     basic: np.ndarray | None = None, first_anchor: int = 0,
                     anchor_count: int | None = None, threads: int | None = None,
                     flow: tuple[FlowGrids | None, FlowGrids | None] | None = None):
        clip = np.ascontiguousarray(clip, dtype=np.float32)
        frames, channels, height, width = clip.shape
        if basic is not None:
            basic = np.ascontiguousarray(basic, dtype=np.float32)
        if anchor_count is None:
            anchor_count = frames - first_anchor
        threads = threads or os.cpu_count() or 1
        out = np.zeros((anchor_count, channels, params.slots * 2 * height, width), np.float32)
        cp = params.to_c()
        if flow is not None:
            cf, keep = c_flow(*flow)
            self._check(self._fn("stage_stacks_flow")(
                ctypes.c_int(stage), ctypes.byref(cp), self._ptr(clip), self._ptr(basic),
                width, height, frames, channels, first_anchor, anchor_count, threads,
                ctypes.byref(cf), self._ptr(out)))
            return out
        self._check(self._fn("stage_stacks")(
            ctypes.c_int(stage), ctypes.byref(cp), self._ptr(clip), self._ptr(basic),
            width, height, frames, channels, first_anchor, anchor_count, threads,
            self._ptr(out)))
        return out

    def aggregate(self, stacks: np.ndarray, source: np.ndarray, search_bwd: int,
                  search_fwd: int, patch_time: int) -> np.ndarray:
        stacks = np.ascontiguousarray(stacks, dtype=np.float32)
        source = np.ascontiguousarray(source, dtype=np.float32)
        frames, channels, height, width = source.shape
        out = np.empty_like(source)
        self._check(self._fn("aggregate")(
            self._ptr(stacks), self._ptr(source), width, height, frames, channels,
            search_bwd, search_fwd, patch_time, self._ptr(out)))
        return out

    def chain(self, noisy: np.ndarray, basic_params: StageParams,
              final_params: StageParams, threads: int | None = None):
        """vnlb.Basic -> vnlb.Aggregate -> vnlb.Final(ref=basic) -> Aggregate."""
        bs = self.stage_stacks(BASIC, basic_params, noisy, threads=threads)
        basic = self.aggregate(bs, noisy, basic_params.search_bwd,
                               basic_params.search_fwd, basic_params.patch_time)
        fs = self.stage_stacks(FINAL, final_params, noisy, basic, threads=threads)
        final = self.aggregate(fs, noisy, final_params.search_bwd,
                               final_params.search_fwd, final_params.patch_time)
        return basic, final


class _Group(ctypes.Structure):
    _fields_ = [("anchor_x", ctypes.c_int), ("anchor_y", ctypes.c_int), ("similar", ctypes.c_int),
                ("first_match", ctypes.c_int)]


class _Match(ctypes.Structure):
    _fields_ = [("distance", ctypes.c_float), ("x", ctypes.c_int), ("y", ctypes.c_int),
                ("frame", ctypes.c_int), ("weight", ctypes.c_float)]


ROW_DTYPE = [("distance", "f4"), ("x", "i4"), ("y", "i4"), ("frame", "i4"), ("weight", "f4")]


def anchor_groups(stage: int, params: StageParams, clip: np.ndarray, basic: np.ndarray | None,
                  anchor: int, flow: tuple[FlowGrids | None, FlowGrids | None] | None = None):
    """Restatement only: the processed groups of one anchor frame in raster
    order -> (stack, groups [(x, y, S, first)], rows structured array)."""
    o = Oracle("port")
    clip = np.ascontiguousarray(clip, dtype=np.float32)
    frames, channels, height, width = clip.shape
    if basic is not None:
        basic = np.ascontiguousarray(basic, dtype=np.float32)
    stack = np.zeros((channels, params.slots * 2 * height, width), np.float32)
    cp = params.to_c()
    total = ctypes.c_int()
    cf, keep = c_flow(*flow) if flow is not None else (None, [])
    fref = ctypes.byref(cf) if cf is not None else None
    fn = o.lib.vnlboracle_anchor_groups_flow
    n = fn(ctypes.c_int(stage), ctypes.byref(cp), o._ptr(clip), o._ptr(basic), width, height, frames,
           channels, anchor, fref, o._ptr(stack), None, 0, None, 0, ctypes.byref(total))
    if n < 0:
        o._check(-1)
    groups = (_Group * max(1, n))()
    matches = (_Match * max(1, total.value))()
    fn(ctypes.c_int(stage), ctypes.byref(cp), o._ptr(clip), o._ptr(basic), width, height, frames, channels,
       anchor, fref, o._ptr(stack), groups, n, matches, total.value, ctypes.byref(total))
    g = [(x.anchor_x, x.anchor_y, x.similar, x.first_match) for x in groups[:n]]
    rows = np.array([(m.distance, m.x, m.y, m.frame, m.weight) for m in matches[:total.value]], dtype=ROW_DTYPE)
    return stack, g, rows


def match_anchor(stage: int, params: StageParams, clip: np.ndarray, basic: np.ndarray | None, anchor: int,
                 x: int, y: int):
    """Restatement only: the retained rows of one anchor (no paste mask)."""
    o = Oracle("port")
    clip = np.ascontiguousarray(clip, dtype=np.float32)
    frames, channels, height, width = clip.shape
    if basic is not None:
        basic = np.ascontiguousarray(basic, dtype=np.float32)
    cap = 8192
    out = (_Match * cap)()
    cp = params.to_c()
    n = o.lib.vnlboracle_match_anchor(ctypes.c_int(stage), ctypes.byref(cp), o._ptr(clip), o._ptr(basic),
                                          width, height, frames, channels, anchor, x, y, out, cap)
    if n < 0:
        o._check(-1)
    return np.array([(m.distance, m.x, m.y, m.frame, m.weight) for m in out[:n]], dtype=ROW_DTYPE)
