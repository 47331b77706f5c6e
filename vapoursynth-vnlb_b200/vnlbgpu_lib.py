"""ctypes binding of the C ABI in include/vnlbgpu.h (lib/libvnlbgpu.so).

The library is built in-tree by build_native.py.  There is no CPU fallback:
if the library is missing or no CUDA device is usable, every call raises.
"""
from __future__ import annotations

import ctypes
import os
import threading
from pathlib import Path

import numpy as np

# VNLBGPU_LIBRARY names another build of the same library (a variant built for
# a comparison); unset, the in-tree build is loaded.
LIB_PATH = Path(os.environ.get("VNLBGPU_LIBRARY") or Path(__file__).resolve().parent / "lib" / "libvnlbgpu.so")

STAGE_BASIC, STAGE_FINAL = 0, 1
FORM_PLAIN, FORM_CHOSEN, FORM_CHOSEN_TC, FORM_LEARNED = 0, 1, 2, 3
SOURCE_CLIP, SOURCE_REF = 0, 1


class VNLBError(RuntimeError):
    """Raised with the library's error text (prefixed like the plugin's)."""


class Params(ctypes.Structure):
    _fields_ = [
        ("stage", ctypes.c_int), ("sigma", ctypes.c_float), ("patch_size", ctypes.c_int),
        ("patch_time", ctypes.c_int), ("search_window", ctypes.c_int), ("search_bwd", ctypes.c_int),
        ("search_fwd", ctypes.c_int), ("similar", ctypes.c_int), ("rank", ctypes.c_int),
        ("similar_cap_factor", ctypes.c_float), ("model_cap_factor", ctypes.c_float),
        ("beta", ctypes.c_float), ("tau", ctypes.c_float), ("variance_threshold", ctypes.c_float),
        ("sigma_basic", ctypes.c_float), ("gamma", ctypes.c_float), ("weight_alpha", ctypes.c_float),
        ("weight_beta", ctypes.c_float), ("weight_gamma", ctypes.c_float),
        ("weight_epsilon", ctypes.c_float), ("membership_noise_floor", ctypes.c_float),
        ("proc_step", ctypes.c_int), ("flat_areas", ctypes.c_int), ("couple_channels", ctypes.c_int),
        ("device_id", ctypes.c_int), ("num_streams", ctypes.c_int), ("chunk_size", ctypes.c_int),
        ("form", ctypes.c_int),
    ]


class Stats(ctypes.Structure):
    _fields_ = [(name, ctypes.c_longlong) for name in
                ("anchor_frames", "groups", "active_groups", "rows", "kernel_launches", "pipeline_lanes",
                 "source_slots", "source_uploads", "learned_tiles", "learned_fallback_tiles")]


class MVToolsAnalysis(ctypes.Structure):
    """vnlbgpu_mvtools_analysis: MVToolsAnalysisData (src/flow/flow.hpp:37-55)."""
    _fields_ = [(name, ctypes.c_int) for name in (
        "block_size_x", "block_size_y", "pel", "level_count", "delta_frame", "backwards", "width", "height",
        "overlap_x", "overlap_y", "block_count_x", "block_count_y", "bits_per_sample", "chroma_ratio_x",
        "chroma_ratio_y", "padding_x", "padding_y")]


MVFW, MVBW = 0, 1


class DiagRow(ctypes.Structure):
    _fields_ = [("distance", ctypes.c_float), ("x", ctypes.c_int), ("y", ctypes.c_int),
                ("frame", ctypes.c_int), ("weight", ctypes.c_float)]


EXPORTS = [
    "vnlbgpu_last_error", "vnlbgpu_create", "vnlbgpu_destroy", "vnlbgpu_set_frame",
    "vnlbgpu_set_clip_host", "vnlbgpu_set_clip_device", "vnlbgpu_required_source_range",
    "vnlbgpu_render_frame", "vnlbgpu_render_frame_window",
    "vnlbgpu_render_clip_host", "vnlbgpu_render_clip_device", "vnlbgpu_render_chain_device", "vnlbgpu_synchronize",
    "vnlbgpu_render_stack", "vnlbgpu_aggregate", "vnlbgpu_aggregate_frame_noalloc", "vnlbgpu_get_stats",
    "vnlbgpu_stream",
    "vnlbgpu_set_stream", "vnlbgpu_diag_anchor", "vnlbgpu_diag_kernel_timing", "vnlbgpu_diag_set_lanes",
    "vnlbgpu_diag_filtered", "vnlbgpu_diag_stall_tensor_waits",
    "vnlbgpu_parse_mvtools_analysis", "vnlbgpu_parse_mvtools_vectors", "vnlbgpu_set_mvtools_analysis",
    "vnlbgpu_set_mvtools_frame", "vnlbgpu_shard_plan", "vnlbgpu_mlp_create", "vnlbgpu_mlp_destroy",
    "vnlbgpu_mlp_parameters", "vnlbgpu_mlp_get_weights", "vnlbgpu_mlp_set_weights", "vnlbgpu_mlp_gradients",
    "vnlbgpu_mlp_train_step", "vnlbgpu_mlp_logits", "vnlbgpu_mlp_shortlist", "vnlbgpu_set_learned",
    "vnlbgpu_learned_pairs", "vnlbgpu_autotune",
]
KERNEL_CLASSES = ("match", "paste", "filter", "tiles", "normalize")

_lib = None
_lib_lock = threading.Lock()


def load() -> ctypes.CDLL:
    global _lib
    with _lib_lock:
        if _lib is None:
            if not LIB_PATH.exists():
                raise VNLBError(f"VNLB CUDA: native library {LIB_PATH} is not built "
                                "(run vapoursynth-vnlb_b200/build_native.py)")
            lib = ctypes.CDLL(str(LIB_PATH))
            lib.vnlbgpu_last_error.restype = ctypes.c_char_p
            lib.vnlbgpu_create.argtypes = [ctypes.POINTER(Params), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
            lib.vnlbgpu_destroy.argtypes = [ctypes.c_void_p]
            lib.vnlbgpu_destroy.restype = None
            lib.vnlbgpu_set_clip_host.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
            lib.vnlbgpu_set_clip_device.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
            lib.vnlbgpu_set_frame.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                              ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_ssize_t)]
            lib.vnlbgpu_render_frame.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p),
                                                 ctypes.POINTER(ctypes.c_ssize_t)]
            lib.vnlbgpu_render_stack.argtypes = lib.vnlbgpu_render_frame.argtypes
            lib.vnlbgpu_required_source_range.argtypes = [ctypes.c_void_p, ctypes.c_int,
                                                          ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
            lib.vnlbgpu_render_frame_window.argtypes = [
                ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_ssize_t),
                ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_ssize_t),
                ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_ssize_t)]
            lib.vnlbgpu_render_clip_host.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
            lib.vnlbgpu_render_clip_device.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
            lib.vnlbgpu_render_chain_device.argtypes = [ctypes.c_void_p] * 4
            lib.vnlbgpu_synchronize.argtypes = [ctypes.c_void_p]
            lib.vnlbgpu_get_stats.argtypes = [ctypes.c_void_p, ctypes.POINTER(Stats)]
            lib.vnlbgpu_stream.argtypes = [ctypes.c_void_p]
            lib.vnlbgpu_stream.restype = ctypes.c_void_p
            lib.vnlbgpu_aggregate.argtypes = [ctypes.c_void_p, ctypes.c_void_p] + [ctypes.c_int] * 8 + [ctypes.c_void_p]
            lib.vnlbgpu_aggregate_frame_noalloc.argtypes = ([ctypes.c_void_p, ctypes.c_void_p] + [ctypes.c_int] * 9
                                                            + [ctypes.c_void_p])
            lib.vnlbgpu_diag_anchor.argtypes = [
                ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                ctypes.POINTER(ctypes.c_int)]
            lib.vnlbgpu_set_stream.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
            lib.vnlbgpu_diag_kernel_timing.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                                       ctypes.c_void_p]
            lib.vnlbgpu_diag_set_lanes.argtypes = [ctypes.c_void_p, ctypes.c_int]
            lib.vnlbgpu_diag_stall_tensor_waits.argtypes = [ctypes.c_void_p, ctypes.c_int]
            lib.vnlbgpu_diag_filtered.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                                  ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
            lib.vnlbgpu_parse_mvtools_analysis.argtypes = [ctypes.c_char_p, ctypes.c_size_t,
                                                           ctypes.POINTER(MVToolsAnalysis)]
            lib.vnlbgpu_parse_mvtools_vectors.argtypes = [
                ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(MVToolsAnalysis), ctypes.POINTER(ctypes.c_int),
                ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]
            lib.vnlbgpu_set_mvtools_analysis.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p,
                                                         ctypes.c_size_t]
            lib.vnlbgpu_set_mvtools_frame.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_char_p,
                                                      ctypes.c_size_t, ctypes.c_int]
            lib.vnlbgpu_shard_plan.argtypes = [ctypes.c_int] * 9 + [ctypes.POINTER(ctypes.c_int)] * 3
            lib.vnlbgpu_autotune.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                             ctypes.POINTER(ctypes.c_int), ctypes.c_char_p, ctypes.c_size_t]
            lib.vnlbgpu_mlp_create.argtypes = [ctypes.c_int] * 5 + [ctypes.c_uint, ctypes.c_int,
                                                                   ctypes.POINTER(ctypes.c_void_p)]
            lib.vnlbgpu_mlp_destroy.argtypes = [ctypes.c_void_p]
            lib.vnlbgpu_mlp_destroy.restype = None
            lib.vnlbgpu_mlp_parameters.argtypes = [ctypes.c_void_p]
            lib.vnlbgpu_mlp_parameters.restype = ctypes.c_longlong
            lib.vnlbgpu_mlp_get_weights.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
            lib.vnlbgpu_mlp_set_weights.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
            lib.vnlbgpu_mlp_gradients.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                                  ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_float)]
            lib.vnlbgpu_mlp_train_step.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                                   ctypes.c_int, ctypes.c_float, ctypes.POINTER(ctypes.c_float)]
            lib.vnlbgpu_mlp_logits.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
            lib.vnlbgpu_mlp_shortlist.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                                  ctypes.c_void_p]
            lib.vnlbgpu_set_learned.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_float,
                                                ctypes.c_int]
            lib.vnlbgpu_learned_pairs.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                                  ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                                  ctypes.POINTER(ctypes.c_int)]
            _lib = lib
    return _lib


def _check(status: int):
    if status != 0:
        raise VNLBError(load().vnlbgpu_last_error().decode())


def _f32(a: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def parse_mvtools_analysis(data: bytes) -> MVToolsAnalysis:
    """parse_mvtools_analysis (flow.hpp:193-250) of an MVTools_MVAnalysisData
    property; host only, no device needed."""
    out = MVToolsAnalysis()
    _check(load().vnlbgpu_parse_mvtools_analysis(bytes(data), len(data), ctypes.byref(out)))
    return out


def parse_mvtools_vectors(data: bytes, analysis: MVToolsAnalysis):
    """parse_mvtools_vectors (flow.hpp:252-318) of an MVTools_vectors property:
    (valid, int32 array [count, 2] of the finest level's vectors)."""
    valid, count = ctypes.c_int(), ctypes.c_size_t()
    cap = analysis.block_count_x * analysis.block_count_y
    xy = np.zeros((max(cap, 1), 2), np.int32)
    _check(load().vnlbgpu_parse_mvtools_vectors(bytes(data), len(data), ctypes.byref(analysis), ctypes.byref(valid),
                                                xy.ctypes.data, cap, ctypes.byref(count)))
    return bool(valid.value), xy[:count.value]


class MLP:
    """vnlbgpu_mlp: the learned proposals' network, trained and run by the
    library's CUDA kernels.  x / targets / outputs are device pointers (e.g.
    torch CUDA tensors' data_ptr()); weights and gradients are flat host
    arrays, layer by layer [W_l (fan_out x fan_in)][b_l]."""

    def __init__(self, inputs: int, hidden: int, layers: int, outputs: int, max_batch: int = 4096, seed: int = 0,
                 device_id: int = 0):
        self.lib = load()
        self.shape = (inputs, hidden, layers, outputs)
        handle = ctypes.c_void_p()
        _check(self.lib.vnlbgpu_mlp_create(inputs, hidden, layers, outputs, max_batch, seed, device_id,
                                           ctypes.byref(handle)))
        self.handle = handle

    def close(self):
        if getattr(self, "handle", None):
            self.lib.vnlbgpu_mlp_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def parameters(self) -> int:
        return int(self.lib.vnlbgpu_mlp_parameters(self.handle))

    def get_weights(self) -> np.ndarray:
        out = np.empty(self.parameters(), np.float32)
        _check(self.lib.vnlbgpu_mlp_get_weights(self.handle, out.ctypes.data))
        return out

    def set_weights(self, flat: np.ndarray):
        flat = _f32(flat)
        if flat.size != self.parameters():
            raise VNLBError("VNLB CUDA: weight count does not match the network")
        _check(self.lib.vnlbgpu_mlp_set_weights(self.handle, flat.ctypes.data))

    def gradients(self, x_ptr: int, targets_ptr: int, batch: int, tk: int):
        grads = np.empty(self.parameters(), np.float32)
        loss = ctypes.c_float()
        _check(self.lib.vnlbgpu_mlp_gradients(self.handle, ctypes.c_void_p(x_ptr), ctypes.c_void_p(targets_ptr), batch,
                                              tk, grads.ctypes.data, ctypes.byref(loss)))
        return grads, loss.value

    def train_step(self, x_ptr: int, targets_ptr: int, batch: int, tk: int, lr: float) -> float:
        loss = ctypes.c_float()
        _check(self.lib.vnlbgpu_mlp_train_step(self.handle, ctypes.c_void_p(x_ptr), ctypes.c_void_p(targets_ptr),
                                               batch, tk, lr, ctypes.byref(loss)))
        return loss.value

    def logits(self, x_ptr: int, batch: int, out_ptr: int):
        _check(self.lib.vnlbgpu_mlp_logits(self.handle, ctypes.c_void_p(x_ptr), batch, ctypes.c_void_p(out_ptr)))

    def shortlist(self, x_ptr: int, batch: int, k: int, out_ptr: int):
        _check(self.lib.vnlbgpu_mlp_shortlist(self.handle, ctypes.c_void_p(x_ptr), batch, k,
                                              ctypes.c_void_p(out_ptr)))


def render_chain_device(basic: "Session", final: "Session", basic_out_ptr: int, final_out_ptr: int):
    """vnlbgpu_render_chain_device: Basic into Final over the whole clip on
    the device, the stages overlapped; final's ref must be basic_out_ptr."""
    _check(load().vnlbgpu_render_chain_device(basic.handle, final.handle, ctypes.c_void_p(basic_out_ptr),
                                              ctypes.c_void_p(final_out_ptr)))


def shard_plan(frames: int, world: int, rank: int, basic: tuple[int, int, int], final: tuple[int, int, int]):
    """vnlbgpu_shard_plan: rank's block of Final output frames, the Basic
    frames it reads and the source frames both stages read, each an inclusive
    (first, last) range or None.  basic / final are (search_bwd, search_fwd,
    patch_time) of the two stages.  Host only."""
    out, bas, src = (ctypes.c_int * 2)(), (ctypes.c_int * 2)(), (ctypes.c_int * 2)()
    _check(load().vnlbgpu_shard_plan(frames, world, rank, *basic, *final, out, bas, src))
    pick = lambda r: None if r[0] < 0 else (r[0], r[1])
    return {"out": pick(out), "basic": pick(bas), "source": pick(src)}


class Session:
    """One configured stage (Basic or Final) over one clip geometry."""

    def set_mvtools_analysis(self, direction: int, data: bytes):
        """The mvfw (MVFW) or mvbw (MVBW) clip's MVTools_MVAnalysisData."""
        _check(load().vnlbgpu_set_mvtools_analysis(self.handle, direction, bytes(data), len(data)))

    def set_mvtools_frame(self, direction: int, frame: int, vectors: bytes, scene_change: bool = False):
        """Frame `frame`'s MVTools_vectors of that clip, and whether the source
        clip's frame marks a scene change."""
        _check(load().vnlbgpu_set_mvtools_frame(self.handle, direction, frame, bytes(vectors), len(vectors),
                                                1 if scene_change else 0))

    def __init__(self, params: Params, width: int, height: int, frames: int, channels: int):
        self.lib = load()
        self.shape = (frames, channels, height, width)
        self.params = params
        handle = ctypes.c_void_p()
        _check(self.lib.vnlbgpu_create(ctypes.byref(params), width, height, frames, channels,
                                       ctypes.byref(handle)))
        self.handle = handle
        self._keep = {}

    def close(self):
        if getattr(self, "handle", None):
            self.lib.vnlbgpu_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_clip(self, source: int, clip: np.ndarray):
        clip = _f32(clip)
        if clip.shape != self.shape:
            raise VNLBError(f"VNLB CUDA: clip shape {clip.shape} does not match {self.shape}")
        _check(self.lib.vnlbgpu_set_clip_host(self.handle, source, clip.ctypes.data))

    def set_clip_ptr(self, source: int, host_ptr: int):
        """Uploads a whole clip from a raw host pointer (e.g. pinned memory)."""
        _check(self.lib.vnlbgpu_set_clip_host(self.handle, source, ctypes.c_void_p(host_ptr)))

    def set_clip_device(self, source: int, device_ptr: int, keepalive=None):
        self._keep[source] = keepalive
        _check(self.lib.vnlbgpu_set_clip_device(self.handle, source, ctypes.c_void_p(device_ptr)))

    def render_clip(self) -> np.ndarray:
        out = np.empty(self.shape, np.float32)
        _check(self.lib.vnlbgpu_render_clip_host(self.handle, out.ctypes.data))
        return out

    def render_clip_into(self, out_ptr: int):
        _check(self.lib.vnlbgpu_render_clip_host(self.handle, ctypes.c_void_p(out_ptr)))

    def render_clip_device(self, device_ptr: int):
        _check(self.lib.vnlbgpu_render_clip_device(self.handle, ctypes.c_void_p(device_ptr)))

    def synchronize(self):
        _check(self.lib.vnlbgpu_synchronize(self.handle))

    def _planes(self, arrays):
        ptrs = (ctypes.c_void_p * len(arrays))(*[a.ctypes.data for a in arrays])
        strides = (ctypes.c_ssize_t * len(arrays))(*[a.strides[0] for a in arrays])
        return ptrs, strides

    def render_frame(self, n: int) -> np.ndarray:
        frames, channels, height, width = self.shape
        out = np.empty((channels, height, width), np.float32)
        ptrs, strides = self._planes([out[c] for c in range(channels)])
        _check(self.lib.vnlbgpu_render_frame(self.handle, n, ptrs, strides))
        return out

    def set_frame(self, source: int, frame: int, planes):
        """vnlbgpu_set_frame: one frame from per-plane 2-D arrays (any row
        stride); a frame already on the device is not copied again."""
        ptrs, strides = self._planes(list(planes))
        _check(self.lib.vnlbgpu_set_frame(self.handle, source, frame, ptrs, strides))

    def required_source_range(self, n: int) -> tuple[int, int]:
        first, last = ctypes.c_int(), ctypes.c_int()
        _check(self.lib.vnlbgpu_required_source_range(self.handle, n, ctypes.byref(first), ctypes.byref(last)))
        return first.value, last.value

    def render_frame_window(self, n: int, clip_frames, ref_frames=None, first: int | None = None,
                            out: np.ndarray | None = None) -> np.ndarray:
        """vnlbgpu_render_frame_window: output frame n, giving the source
        frames first .. first + len(clip_frames) - 1 as sequences of per-plane
        2-D arrays (VapourSynth frames: one array per plane, any row stride).
        `first` defaults to the start of the required source range."""
        frames, channels, height, width = self.shape
        if first is None:
            first = self.required_source_range(n)[0]
        count = len(clip_frames)
        clip_planes = [p for f in clip_frames for p in f]
        cp, cs = self._planes(clip_planes)
        rp = rs = None
        if ref_frames is not None:
            rp, rs = self._planes([p for f in ref_frames for p in f])
        if out is None:
            out = np.empty((channels, height, width), np.float32)
        op, os_ = self._planes([out[c] for c in range(channels)])
        _check(self.lib.vnlbgpu_render_frame_window(self.handle, n, first, count, cp, cs, rp, rs, op, os_))
        return out

    def render_stack(self, n: int) -> np.ndarray:
        frames, channels, height, width = self.shape
        slots = self.params.search_bwd + self.params.search_fwd + self.params.patch_time
        out = np.empty((channels, slots * 2 * height, width), np.float32)
        ptrs, strides = self._planes([out[c] for c in range(channels)])
        _check(self.lib.vnlbgpu_render_stack(self.handle, n, ptrs, strides))
        return out

    def stats(self) -> dict:
        s = Stats()
        _check(self.lib.vnlbgpu_get_stats(self.handle, ctypes.byref(s)))
        return {name: getattr(s, name) for name, _ in Stats._fields_}

    def stream(self) -> int:
        return self.lib.vnlbgpu_stream(self.handle) or 0

    def set_stream(self, stream_ptr: int):
        _check(self.lib.vnlbgpu_set_stream(self.handle, ctypes.c_void_p(stream_ptr or None)))

    def kernel_timing(self, enable: bool = True) -> dict:
        """Per-kernel-class device time (ms) and launches since the last call."""
        ms = np.zeros(len(KERNEL_CLASSES), np.float64)
        n = np.zeros(len(KERNEL_CLASSES), np.int64)
        _check(self.lib.vnlbgpu_diag_kernel_timing(self.handle, 1 if enable else 0, ms.ctypes.data, n.ctypes.data))
        return {k: (float(ms[i]), int(n[i])) for i, k in enumerate(KERNEL_CLASSES)}

    def set_learned(self, mlp: MLP, shortlist: int = 64, recall_threshold: float = 0.9, tile: int = 64):
        """vnlbgpu_set_learned: the network of a learned-form session."""
        self._keep["mlp"] = mlp
        _check(self.lib.vnlbgpu_set_learned(self.handle, mlp.handle, shortlist, recall_threshold, tile))

    def learned_pairs(self, anchor: int, k: int = 8):
        """vnlbgpu_learned_pairs: (features [G][inputs], target classes [G][k])
        of anchor frame `anchor`'s grid anchors under the full search."""
        count, inputs = ctypes.c_int(), ctypes.c_int()
        _check(self.lib.vnlbgpu_learned_pairs(self.handle, anchor, None, None, 0, k, ctypes.byref(count),
                                              ctypes.byref(inputs)))
        feats = np.zeros((max(1, count.value), inputs.value), np.float32)
        targets = np.full((max(1, count.value), k), -1, np.int32)
        _check(self.lib.vnlbgpu_learned_pairs(self.handle, anchor, feats.ctypes.data, targets.ctypes.data, count.value,
                                              k, ctypes.byref(count), ctypes.byref(inputs)))
        return feats[:count.value], targets[:count.value]

    def stall_tensor_waits(self, on: bool):
        """vnlbgpu_diag_stall_tensor_waits: the tensor-core matcher's test switch."""
        _check(self.lib.vnlbgpu_diag_stall_tensor_waits(self.handle, 1 if on else 0))

    def autotune(self, anchor: int = 1) -> dict:
        """vnlbgpu_autotune: the fastest bit-identical strip width and apply
        kernel on anchor frame `anchor`."""
        w, rows = ctypes.c_int(), ctypes.c_int()
        buf = ctypes.create_string_buffer(1024)
        _check(self.lib.vnlbgpu_autotune(self.handle, anchor, ctypes.byref(w), ctypes.byref(rows), buf, 1024))
        return {"match_warps": w.value, "apply_rows": bool(rows.value),
                "timings": [line for line in buf.value.decode().splitlines() if line]}

    def set_lanes(self, lanes: int):
        """vnlbgpu_diag_set_lanes: use at most `lanes` pipeline lanes (0: all)."""
        _check(self.lib.vnlbgpu_diag_set_lanes(self.handle, lanes))

    def diag_filtered(self, anchor: int) -> np.ndarray:
        """The filtered rows [rows][row_dim] of anchor frame `anchor`'s
        processed groups, in the order of diag_anchor's active rows."""
        rows, dim = ctypes.c_int(), ctypes.c_int()
        _check(self.lib.vnlbgpu_diag_filtered(self.handle, anchor, None, 0, ctypes.byref(rows), ctypes.byref(dim)))
        out = np.zeros((max(1, rows.value), dim.value), np.float32)
        _check(self.lib.vnlbgpu_diag_filtered(self.handle, anchor, out.ctypes.data, rows.value, ctypes.byref(rows),
                                              ctypes.byref(dim)))
        return out[:rows.value]

    def diag_anchor(self, anchor: int):
        """Runs one anchor frame and returns (grid, active) read-backs."""
        frames, channels, height, width = self.shape
        G = ctypes.c_int()
        A = ctypes.c_int()
        R = ctypes.c_int()
        M = ctypes.c_int()
        # first call with zero capacity to learn the sizes
        _check(self.lib.vnlbgpu_diag_anchor(self.handle, anchor, None, None, None, 0, 0, None, None, 0, 0,
                                            ctypes.byref(G), ctypes.byref(A), ctypes.byref(R), ctypes.byref(M)))
        g, a, r, m = G.value, A.value, R.value, M.value
        xy = np.zeros((g, 2), np.int32)
        counts = np.zeros(g, np.int32)
        grid_rows = (DiagRow * max(1, g * m))()
        active = np.zeros(max(1, a), np.int32)
        active_rows = (DiagRow * max(1, r))()
        _check(self.lib.vnlbgpu_diag_anchor(self.handle, anchor, xy.ctypes.data, counts.ctypes.data, grid_rows,
                                            g, g * m, active.ctypes.data, active_rows, a, r,
                                            ctypes.byref(G), ctypes.byref(A), ctypes.byref(R), ctypes.byref(M)))
        to_np = lambda rows, n: np.array([(x.distance, x.x, x.y, x.frame, x.weight) for x in rows[:n]],
                                         dtype=[("distance", "f4"), ("x", "i4"), ("y", "i4"), ("frame", "i4"),
                                                ("weight", "f4")])
        return {"xy": xy, "counts": counts, "grid_rows": to_np(grid_rows, g * m).reshape(g, m) if g else None,
                "max_rows": m, "active": active[:a], "active_rows": to_np(active_rows, r)}


def aggregate(stacks: np.ndarray, source: np.ndarray, search_bwd: int, search_fwd: int, patch_time: int,
              device_id: int = 0) -> np.ndarray:
    lib = load()
    stacks = _f32(stacks)
    source = _f32(source)
    frames, channels, height, width = source.shape
    out = np.empty_like(source)
    _check(lib.vnlbgpu_aggregate(stacks.ctypes.data, source.ctypes.data, width, height, frames, channels,
                                 search_bwd, search_fwd, patch_time, device_id, out.ctypes.data))
    return out


def aggregate_frame_noalloc(stacks: np.ndarray, source: np.ndarray, n: int, search_bwd: int, search_fwd: int,
                            patch_time: int, device_id: int = 0) -> np.ndarray:
    """vnlb.Aggregate of output frame n alone, through the library's fixed
    device scratch (no device allocation): [planes][H][W]."""
    lib = load()
    stacks = _f32(stacks)
    source = _f32(source)
    frames, channels, height, width = source.shape
    out = np.empty((channels, height, width), np.float32)
    _check(lib.vnlbgpu_aggregate_frame_noalloc(stacks.ctypes.data, source.ctypes.data, width, height, frames,
                                               channels, search_bwd, search_fwd, patch_time, device_id, n,
                                               out.ctypes.data))
    return out
