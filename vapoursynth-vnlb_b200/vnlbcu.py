"""vnlbcu.Basic / vnlbcu.Final on the B200 path.

Mirrors the reference's CUDA VapourSynth plugin surface (namespace vnlbcu,
registered at src/vs/cuda_plugin.cpp:2147-2181): the same argument names, the
same defaults and default clamps (parse_parameters, cuda_plugin.cpp:370-536),
the same validation messages (validate_parameters, :545-626, and
derive_geometry, :691-807), and aggregated output frames of the input's format.

A clip is a float32 array [frames, planes, height, width] with 1 plane
(GrayS) or 3 planes (YUV444PS).  The computation runs through the C ABI of
include/vnlbgpu.h; there is no CPU fallback.
"""
from __future__ import annotations

import math

import numpy as np

import vnlbgpu_lib as lib
from vnlbgpu_lib import VNLBError

EIGHT_BIT = np.float32(255.0)
EIGHT_BIT_DISTANCE = np.float32(255.0) * np.float32(255.0)
DEFAULT_GROUP = 16
DEFAULT_RANK = 15
DEFAULT_CHUNK = 768
INT_MAX = 2**31 - 1


def _err(message: str):
    raise VNLBError("VNLB CUDA: " + message)


def _check_clip(clip, name="clip"):
    if not isinstance(clip, np.ndarray) or clip.ndim != 4 or clip.shape[1] not in (1, 3) or \
            clip.dtype != np.float32 or min(clip.shape) <= 0:
        _err("only constant GrayS and YUV444PS clips are supported")
    return clip


def _int(name, value):
    if isinstance(value, (bool, np.bool_)) or not isinstance(value, (int, np.integer)):
        _err(f"{name} must be an integer")
    if value < -2**31 or value > INT_MAX:
        _err(f"{name} is outside the supported int range")
    return int(value)


def _float(name, value):
    if not isinstance(value, (int, float, np.integer, np.floating)) or isinstance(value, bool):
        _err(f"{name} must be a float")
    return np.float32(value)


def parse_parameters(stage: int, clip: np.ndarray, sigma, args: dict) -> lib.Params:
    """parse_parameters (src/vs/cuda_plugin.cpp:370-536)."""
    frames, planes, height, width = clip.shape
    if sigma is None:
        _err("missing required argument: sigma")
    sigma8 = _float("sigma", sigma)
    gray = planes == 1
    final = stage == lib.STAGE_FINAL
    p = dict(sigma=sigma8 / EIGHT_BIT, patch_size=10 if gray else 7, patch_time=2 if frames > 1 else 1,
             search_window=27, similar=DEFAULT_GROUP, rank=DEFAULT_RANK, similar_cap_factor=np.float32(4.0),
             model_cap_factor=np.float32(1.0), beta=np.float32(1.0), tau=np.float32(0.0),
             sigma_basic=np.float32(0.0), gamma=np.float32(0.95), weight_alpha=np.float32(0.75),
             weight_beta=np.float32(0.35), weight_gamma=np.float32(1.0), weight_epsilon=np.float32(1.0e-6),
             membership_noise_floor=np.float32(0.25), proc_step=0, flat_areas=0, couple_channels=1,
             device_id=0, num_streams=1, chunk_size=DEFAULT_CHUNK)
    if gray:
        vt = np.float32(3.7) if not final else max(np.float32(0.0), np.float32(1.87) - np.float32(0.028) * sigma8)
    else:
        vt = np.float32(2.7) if not final else max(
            np.float32(0.2), np.float32(1.7) + (np.float32(1.2) - np.float32(1.7)) * (sigma8 - np.float32(10.0))
            / np.float32(10.0))
    p["variance_threshold"] = np.float32(vt)
    if final:
        p.update(tau=np.float32(400.0) / EIGHT_BIT_DISTANCE, flat_areas=1, weight_alpha=np.float32(1.0),
                 weight_beta=np.float32(0.5), weight_gamma=np.float32(1.0))
    given = {k for k, v in args.items() if v is not None}
    g = lambda k: args.get(k)
    if "block_size" in given:
        p["patch_size"] = _int("block_size", g("block_size"))
    if "patch_time" in given:
        p["patch_time"] = _int("patch_time", g("patch_time"))
    radius_default = 1 if frames > p["patch_time"] else 0
    p["search_bwd"] = p["search_fwd"] = radius_default
    if "radius" in given:
        r = _int("radius", g("radius"))
        if r < 0:
            _err("radius must be non-negative")
        p["search_bwd"] = p["search_fwd"] = r
    if "search_bwd" in given:
        p["search_bwd"] = _int("search_bwd", g("search_bwd"))
    if "search_fwd" in given:
        p["search_fwd"] = _int("search_fwd", g("search_fwd"))
    if "bm_range" in given:
        r = _int("bm_range", g("bm_range"))
        if r < 0 or r > (INT_MAX - 1) // 2:
            _err("bm_range must be non-negative")
        p["search_window"] = 2 * r + 1
    for key, field in (("group_size", "similar"), ("rank", "rank"), ("block_step", "proc_step")):
        if key in given:
            p[field] = _int(key, g(key))
    for key, field in (("cap_factor", "similar_cap_factor"), ("model_cap_factor", "model_cap_factor"),
                       ("beta", "beta"), ("variance_threshold", "variance_threshold"),
                       ("weight_alpha", "weight_alpha"), ("weight_beta", "weight_beta"),
                       ("weight_gamma", "weight_gamma"), ("weight_epsilon", "weight_epsilon"),
                       ("membership_noise_floor", "membership_noise_floor")):
        if key in given:
            p[field] = _float(key, g(key))
    if "tau" in given:
        p["tau"] = _float("tau", g("tau")) / EIGHT_BIT_DISTANCE
    if final:
        if "sigma_basic" in given:
            p["sigma_basic"] = _float("sigma_basic", g("sigma_basic")) / EIGHT_BIT
        if "gamma" in given:
            p["gamma"] = _float("gamma", g("gamma"))
        if "flat_areas" in given:
            p["flat_areas"] = 1 if _int("flat_areas", g("flat_areas")) != 0 else 0
    p["couple_channels"] = 1 if (_int("chroma", g("chroma")) if "chroma" in given else 1) != 0 else 0
    for key, field in (("device_id", "device_id"), ("num_streams", "num_streams"), ("chunk_size", "chunk_size")):
        if key in given:
            p[field] = _int(key, g(key))
    # matcher form (no reference counterpart): "plain" reproduces the CPU core
    # bit for bit; "chosen" selects on approximate distances and re-ranks the
    # retained candidates exactly; "chosen_tc" computes the approximate
    # distances on BF16 tensor cores (tcgen05, FP32 accumulation)
    p["form"] = lib.FORM_PLAIN
    if "form" in given:
        forms = {"plain": lib.FORM_PLAIN, "chosen": lib.FORM_CHOSEN, "chosen_tc": lib.FORM_CHOSEN_TC,
                 "learned": lib.FORM_LEARNED}
        if g("form") not in forms:
            _err('form must be "plain", "chosen", "chosen_tc" or "learned"')
        p["form"] = forms[g("form")]
    # default group/rank clamps (cuda_plugin.cpp:482-534)
    default_group = "group_size" not in given
    default_rank = "rank" not in given
    P, Pt, W = p["patch_size"], p["patch_time"], p["search_window"]
    if default_group and P > 0 and Pt > 0:
        sample_dim = P * P * Pt * planes
        if sample_dim <= INT_MAX and sample_dim > 1:
            p["similar"] = min(p["similar"], sample_dim - 1)
    candidates = 0
    if (default_group or default_rank) and 0 < P <= width and P <= height and 0 < Pt <= frames and W > 0 \
            and p["search_bwd"] >= 0 and p["search_fwd"] >= 0:
        temporal = min(p["search_bwd"] + p["search_fwd"] + 1, frames - Pt + 1)
        spatial = min(W, width - P + 1) * min(W, height - P + 1)
        if temporal > 0 and spatial > 0 and spatial * temporal <= INT_MAX:
            candidates = spatial * temporal
    if default_group and candidates > 0:
        p["similar"] = min(p["similar"], candidates)
    if default_rank and candidates > 0:
        p["rank"] = min(p["rank"], min(p["similar"], candidates))
    validate_parameters(p, clip)
    derive_geometry(p, clip)
    if p["proc_step"] == 0:  # vnlbcu's automatic step is half the block (cuda_plugin.cpp:775-777)
        p["proc_step"] = max(1, p["patch_size"] // 2)
    return lib.Params(stage=stage, **{k: (float(v) if isinstance(v, np.floating) else v) for k, v in p.items()})


def validate_parameters(p: dict, clip: np.ndarray):
    """validate_parameters (src/vs/cuda_plugin.cpp:545-626)."""
    frames, planes, height, width = clip.shape
    fin = lambda v: math.isfinite(float(v))
    if not fin(p["sigma"]) or p["sigma"] <= 0:
        _err("sigma must be finite and positive")
    if p["patch_size"] <= 0 or p["patch_size"] > width or p["patch_size"] > height:
        _err("block_size must fit inside the frame")
    if p["patch_time"] <= 0 or p["patch_time"] > frames:
        _err("patch_time must fit inside the clip")
    if p["search_window"] <= 0 or p["search_window"] % 2 == 0:
        _err("bm_range must describe a positive odd search window")
    if p["search_bwd"] < 0 or p["search_fwd"] < 0:
        _err("search_bwd and search_fwd must be non-negative")
    if p["search_bwd"] + p["search_fwd"] + 1 > INT_MAX:
        _err("temporal search span overflows int")
    if p["similar"] <= 0:
        _err("group_size must be positive")
    if p["rank"] < 0:
        _err("rank must be non-negative")
    if not fin(p["similar_cap_factor"]) or (p["similar_cap_factor"] != 0 and p["similar_cap_factor"] < 1):
        _err("cap_factor must be zero or at least 1.0")
    if not fin(p["model_cap_factor"]) or p["model_cap_factor"] != 1:
        _err("the CUDA backend currently requires model_cap_factor=1")
    if not fin(p["beta"]) or p["beta"] <= 0:
        _err("beta must be finite and positive")
    for key in ("tau",):
        if not fin(p[key]) or p[key] < 0:
            _err(f"{key} must be finite and non-negative")
    if not fin(p["variance_threshold"]):
        _err("variance_threshold must be finite")
    if not fin(p["sigma_basic"]) or p["sigma_basic"] < 0:
        _err("sigma_basic must be finite and non-negative")
    if not fin(p["gamma"]) or p["gamma"] <= 0:
        _err("gamma must be finite and positive")
    for key in ("weight_alpha", "weight_beta", "weight_gamma"):
        if not fin(p[key]) or p[key] < 0:
            _err(f"{key} must be finite and non-negative")
    if not fin(p["weight_epsilon"]) or p["weight_epsilon"] <= 0:
        _err("weight_epsilon must be finite and positive")
    if not fin(p["membership_noise_floor"]) or p["membership_noise_floor"] <= 0:
        _err("membership_noise_floor must be finite and positive")
    if p["proc_step"] < 0:
        _err("block_step must be non-negative; use 0 for auto")
    if not p["couple_channels"]:
        _err("the CUDA backend currently requires chroma=1 (coupled channels)")
    if p["device_id"] < 0:
        _err("device_id must be non-negative")
    if p["num_streams"] < 1 or p["num_streams"] > 32:
        _err("num_streams must be in the range 1..32")
    if p["chunk_size"] <= 0:
        _err("chunk_size must be positive")


def derive_geometry(p: dict, clip: np.ndarray):
    """The constraints of derive_geometry (src/vs/cuda_plugin.cpp:691-807)."""
    frames, planes, height, width = clip.shape
    valid = frames - p["patch_time"] + 1
    temporal = min(p["search_bwd"] + p["search_fwd"] + 1, valid)
    candidates = min(p["search_window"], width - p["patch_size"] + 1) * \
        min(p["search_window"], height - p["patch_size"] + 1) * temporal
    basis = min(p["similar"], candidates)
    if basis > 128:
        _err("the CUDA dual-PCA filter supports at most 128 model samples")
    if p["rank"] > basis:
        _err("rank must not exceed min(group_size, candidate_count)")
    sample_dim = p["patch_size"] ** 2 * p["patch_time"] * planes
    if basis >= sample_dim:
        _err("the CUDA backend currently requires the dual-PCA path (min(group_size, candidate_count) must be "
             "smaller than the coupled patch dimension)")


class _Filter:
    """A configured filter: frames are computed on request (getFrame)."""

    def __init__(self, stage: int, clip: np.ndarray, ref, sigma, args):
        self.clip = _check_clip(clip)
        self.params = parse_parameters(stage, self.clip, sigma, args)
        frames, planes, height, width = self.clip.shape
        self.session = lib.Session(self.params, width, height, frames, planes)
        self.session.set_clip(lib.SOURCE_CLIP, self.clip)
        if stage == lib.STAGE_FINAL:
            self.session.set_clip(lib.SOURCE_REF, ref)

    @property
    def num_frames(self) -> int:
        return self.clip.shape[0]

    def get_frame(self, n: int) -> np.ndarray:
        return self.session.render_frame(n)

    def render(self) -> np.ndarray:
        return self.session.render_clip()


_BASIC_ARGS = ("block_size", "block_step", "group_size", "bm_range", "patch_time", "radius", "search_bwd",
               "search_fwd", "rank", "cap_factor", "model_cap_factor", "beta", "tau", "variance_threshold",
               "weight_alpha", "weight_beta", "weight_gamma", "weight_epsilon", "membership_noise_floor", "chroma",
               "device_id", "num_streams", "chunk_size", "form")
_FINAL_ARGS = _BASIC_ARGS + ("sigma_basic", "gamma", "flat_areas")


def _collect(kwargs, allowed):
    unknown = set(kwargs) - set(allowed)
    if unknown:
        raise TypeError(f"unexpected argument(s): {', '.join(sorted(unknown))}")
    return kwargs


def Basic(clip: np.ndarray, sigma=None, **kwargs) -> np.ndarray:
    """vnlbcu.Basic: returns the aggregated Basic estimate of every frame."""
    return _Filter(lib.STAGE_BASIC, clip, None, sigma, _collect(kwargs, _BASIC_ARGS)).render()


def Final(clip: np.ndarray, ref: np.ndarray = None, sigma=None, **kwargs) -> np.ndarray:
    """vnlbcu.Final: returns the aggregated Final estimate of every frame."""
    clip = _check_clip(clip)
    if not isinstance(ref, np.ndarray):
        _err("ref must be a video node")
    if ref.shape != clip.shape or ref.dtype != np.float32:
        _err("ref clip properties must match input clip")
    return _Filter(lib.STAGE_FINAL, clip, ref, sigma, _collect(kwargs, _FINAL_ARGS)).render()


def BasicFilter(clip, sigma=None, **kwargs) -> _Filter:
    """vnlbcu.Basic as a frame server: get_frame(n) renders one frame."""
    return _Filter(lib.STAGE_BASIC, clip, None, sigma, _collect(kwargs, _BASIC_ARGS))


def FinalFilter(clip, ref=None, sigma=None, **kwargs) -> _Filter:
    """vnlbcu.Final as a frame server."""
    clip = _check_clip(clip)
    if not isinstance(ref, np.ndarray) or ref.shape != clip.shape:
        _err("ref clip properties must match input clip")
    return _Filter(lib.STAGE_FINAL, clip, ref, sigma, _collect(kwargs, _FINAL_ARGS))
