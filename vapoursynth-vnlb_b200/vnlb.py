"""vnlb.Basic / vnlb.Final / vnlb.Aggregate with contribution-stack semantics,
computed on the B200 path.

Mirrors the reference's CPU VapourSynth plugin surface (namespace vnlb,
registered at src/vs/plugin.cpp:1155-1194): argument names and defaults of
parse_stage_parameters (plugin.cpp:372-449) and parse_temporal_parameters
(:236-260), the validation of validate_stage_configuration
(src/core/core.cpp:1948-2024), and the output layout of render_stage_frame:
per anchor frame a stack frame of height H * 2 * slots per plane, numerator
rows slot*2H + y and weight rows slot*2H + H + y, the weight repeated in every
plane.  vnlb.Aggregate divides the summed stacks (render_aggregate_frame,
plugin.cpp:966-1045).  The GPU path implements the CPU core's stage for
coupled and uncoupled planes, the dual-PCA and the covariance models, any
model cap and the MVTools-guided search centres (mvfw / mvbw); eigen problems
above 96 x 96 raise.

MVTools clips: VapourSynth hands the plugin frames whose properties carry the
vectors; here `mvfw` and `mvbw` are sequences of those property mappings, one
per frame ("MVTools_MVAnalysisData", "MVTools_vectors" as bytes), and
`clip_props` the source clip's per-frame property mappings, of which the
scene-change flags are read (_SceneChangePrev or Scenechange for mvfw,
_SceneChangeNext for mvbw; src/vs/plugin.cpp:476-485).
"""
from __future__ import annotations

import math

import numpy as np

import vnlbgpu_lib as lib
from vnlbgpu_lib import VNLBError

EIGHT_BIT = np.float32(255.0)
EIGHT_BIT_DISTANCE = np.float32(255.0) * np.float32(255.0)
INT_MAX = 2**31 - 1


def _err(message: str):
    raise VNLBError("VNLB: " + message)


def _clip(clip):
    if not isinstance(clip, np.ndarray) or clip.ndim != 4 or clip.shape[1] not in (1, 3) or \
            clip.dtype != np.float32:
        _err("only constant GrayS and YUV444PS clips are supported")
    return clip


def parse_temporal(args: dict, patch_time=1, search_bwd=1, search_fwd=1):
    """parse_temporal_parameters (src/vs/plugin.cpp:236-260)."""
    if args.get("patch_time") is not None:
        patch_time = int(args["patch_time"])
    if args.get("radius") is not None:
        radius = int(args["radius"])
        if radius < 0:
            _err("radius must be non-negative")
        search_bwd = search_fwd = radius
    if args.get("search_bwd") is not None:
        search_bwd = int(args["search_bwd"])
    if args.get("search_fwd") is not None:
        search_fwd = int(args["search_fwd"])
    if patch_time <= 0 or search_bwd < 0 or search_fwd < 0:
        _err("patch_time must be positive and search_bwd/search_fwd must be non-negative")
    return patch_time, search_bwd, search_fwd


def parse_stage_parameters(stage: int, sigma, args: dict) -> dict:
    """parse_stage_parameters (src/vs/plugin.cpp:372-449), core units."""
    if sigma is None:
        _err("missing required argument: sigma")
    p = dict(sigma=np.float32(sigma) / EIGHT_BIT, patch_size=8, patch_time=1, search_window=19, search_bwd=1,
             search_fwd=1, similar=8, rank=8, similar_cap_factor=np.float32(4.0),
             model_cap_factor=np.float32(1.0), beta=np.float32(1.0), tau=np.float32(0.0),
             variance_threshold=np.float32(1.1), sigma_basic=np.float32(0.0), gamma=np.float32(0.95),
             weight_alpha=np.float32(0.75), weight_beta=np.float32(0.35), weight_gamma=np.float32(1.0),
             weight_epsilon=np.float32(1.0e-6), membership_noise_floor=np.float32(0.25), proc_step=8,
             flat_areas=0, couple_channels=1)
    if stage == lib.STAGE_FINAL:
        p.update(tau=np.float32(400.0) / EIGHT_BIT_DISTANCE, variance_threshold=np.float32(1.7), flat_areas=1,
                 weight_alpha=np.float32(1.0), weight_beta=np.float32(0.5), weight_gamma=np.float32(1.0))
    g = lambda k: args.get(k)
    if g("block_size") is not None:
        p["patch_size"] = int(g("block_size"))
    p["patch_time"], p["search_bwd"], p["search_fwd"] = parse_temporal(args, p["patch_time"], p["search_bwd"],
                                                                     p["search_fwd"])
    if g("bm_range") is not None:
        r = int(g("bm_range"))
        if r < 0 or r > (INT_MAX - 1) // 2:
            _err("bm_range must be non-negative")
        p["search_window"] = 2 * r + 1
    for key, field in (("group_size", "similar"), ("rank", "rank"), ("block_step", "proc_step")):
        if g(key) is not None:
            p[field] = int(g(key))
    for key, field in (("cap_factor", "similar_cap_factor"), ("model_cap_factor", "model_cap_factor"),
                       ("beta", "beta"), ("variance_threshold", "variance_threshold"),
                       ("weight_alpha", "weight_alpha"), ("weight_beta", "weight_beta"),
                       ("weight_gamma", "weight_gamma"), ("weight_epsilon", "weight_epsilon"),
                       ("membership_noise_floor", "membership_noise_floor")):
        if g(key) is not None:
            p[field] = np.float32(g(key))
    if g("tau") is not None:
        p["tau"] = np.float32(g("tau")) / EIGHT_BIT_DISTANCE
    if stage == lib.STAGE_FINAL:
        if g("sigma_basic") is not None:
            p["sigma_basic"] = np.float32(g("sigma_basic")) / EIGHT_BIT
        if g("gamma") is not None:
            p["gamma"] = np.float32(g("gamma"))
        if g("flat_areas") is not None:
            p["flat_areas"] = 1 if int(g("flat_areas")) != 0 else 0
    if g("chroma") is not None:
        p["couple_channels"] = 1 if int(g("chroma")) != 0 else 0
    return p


def validate_stage_configuration(p: dict, clip: np.ndarray):
    """validate_stage_parameters / validate_stage_configuration (core.cpp:1948-2024)."""
    frames, planes, height, width = clip.shape
    fin = lambda v: math.isfinite(float(v))
    checks = [
        (fin(p["sigma"]) and p["sigma"] > 0, "sigma must be finite and positive"),
        (p["patch_size"] > 0, "block_size must be positive"),
        (p["patch_time"] > 0, "patch_time must be positive"),
        (p["search_window"] > 0 and p["search_window"] % 2 == 1, "bm_range must describe a positive odd search window"),
        (p["search_bwd"] >= 0 and p["search_fwd"] >= 0, "search_bwd and search_fwd must be non-negative"),
        (p["similar"] > 0, "group_size must be positive"),
        (p["rank"] >= 0, "rank must be non-negative"),
        (fin(p["similar_cap_factor"]) and (p["similar_cap_factor"] == 0 or p["similar_cap_factor"] >= 1),
         "cap_factor must be zero or at least 1.0"),
        (fin(p["model_cap_factor"]) and (p["model_cap_factor"] == 0 or p["model_cap_factor"] >= 1),
         "model_cap_factor must be zero or at least 1.0"),
        (fin(p["beta"]) and p["beta"] > 0, "beta must be finite and positive"),
        (fin(p["tau"]) and p["tau"] >= 0, "tau must be finite and non-negative"),
        (fin(p["variance_threshold"]), "variance_threshold must be finite"),
        (fin(p["sigma_basic"]) and p["sigma_basic"] >= 0, "sigma_basic must be finite and non-negative"),
        (fin(p["gamma"]) and p["gamma"] > 0, "gamma must be finite and positive"),
        (fin(p["weight_alpha"]) and p["weight_alpha"] >= 0, "weight_alpha must be finite and non-negative"),
        (fin(p["weight_beta"]) and p["weight_beta"] >= 0, "weight_beta must be finite and non-negative"),
        (fin(p["weight_gamma"]) and p["weight_gamma"] >= 0, "weight_gamma must be finite and non-negative"),
        (fin(p["weight_epsilon"]) and p["weight_epsilon"] > 0, "weight_epsilon must be finite and positive"),
        (fin(p["membership_noise_floor"]) and p["membership_noise_floor"] > 0,
         "membership_noise_floor must be finite and positive"),
        (p["proc_step"] >= 0, "block_step must be non-negative; use 0 for auto"),
        (p["patch_size"] <= width and p["patch_size"] <= height, "block_size must fit inside the frame"),
        (p["patch_time"] <= frames, "patch_time must fit inside the clip"),
    ]
    for ok, message in checks:
        if not ok:
            _err(message)
    estimator_dim = p["patch_size"] ** 2 * p["patch_time"] * (planes if p["couple_channels"] else 1)
    if p["rank"] > estimator_dim:
        _err("rank must not exceed the effective patch dimension")
    if p["similar"] < min(estimator_dim, p["rank"]):
        _err("group_size must cover the effective VNLB rank")


_STAGE_ARGS = ("block_size", "block_step", "group_size", "bm_range", "patch_time", "radius", "search_bwd",
               "search_fwd", "rank", "cap_factor", "model_cap_factor", "beta", "tau", "variance_threshold",
               "weight_alpha", "weight_beta", "weight_gamma", "weight_epsilon", "membership_noise_floor", "chroma")


def _set_flow(session, clip, mvfw, mvbw, clip_props):
    """read_mvtools_analysis_from_node + validate_mvtools_clip (plugin.cpp:
    429-474, 881-899) and cache_mvtools_grid (:507-525) for every frame."""
    frames = clip.shape[0]
    props = list(clip_props) if clip_props is not None else [{}] * frames
    if len(props) != frames:
        _err("clip_props must hold one property mapping per frame")
    for direction, name, vectors in ((lib.MVFW, "mvfw", mvfw), (lib.MVBW, "mvbw", mvbw)):
        if vectors is None:
            continue
        vectors = list(vectors)
        if len(vectors) != frames:
            _err(f"{name} frame count must match clip")
        try:
            session.set_mvtools_analysis(direction, vectors[0]["MVTools_MVAnalysisData"])
        except KeyError:
            _err(f"{name} frames carry no MVTools_MVAnalysisData")
        for n in range(frames):
            if direction == lib.MVBW:
                scene = bool(props[n].get("_SceneChangeNext", 0))
            else:
                scene = bool(props[n].get("_SceneChangePrev", 0)) or bool(props[n].get("Scenechange", 0))
            try:
                data = vectors[n]["MVTools_vectors"]
            except KeyError:
                _err(f"{name} frame {n} carries no MVTools_vectors")
            session.set_mvtools_frame(direction, n, data, scene)


class _StageFilter:
    def __init__(self, stage, clip, ref, sigma, kwargs, allowed, mvfw=None, mvbw=None, clip_props=None):
        unknown = set(kwargs) - set(allowed)
        if unknown:
            raise TypeError(f"unexpected argument(s): {', '.join(sorted(unknown))}")
        self.clip = _clip(clip)
        self.p = parse_stage_parameters(stage, sigma, kwargs)
        validate_stage_configuration(self.p, self.clip)
        frames, planes, height, width = self.clip.shape
        params = lib.Params(stage=stage, device_id=0, num_streams=1, chunk_size=768,
                            **{k: (float(v) if isinstance(v, np.floating) else v) for k, v in self.p.items()})
        try:
            self.session = lib.Session(params, width, height, frames, planes)
        except VNLBError as error:
            raise VNLBError(str(error).replace("VNLB CUDA: ", "VNLB: ", 1)) from None
        self.session.set_clip(lib.SOURCE_CLIP, self.clip)
        if stage == lib.STAGE_FINAL:
            self.session.set_clip(lib.SOURCE_REF, ref)
        if mvfw is not None or mvbw is not None:
            _set_flow(self.session, self.clip, mvfw, mvbw, clip_props)
        self.slots = self.p["search_bwd"] + self.p["search_fwd"] + self.p["patch_time"]

    def get_frame(self, n: int) -> np.ndarray:
        return self.session.render_stack(n)

    def render(self) -> np.ndarray:
        return np.stack([self.get_frame(n) for n in range(self.clip.shape[0])])


def Basic(clip, sigma=None, mvfw=None, mvbw=None, clip_props=None, **kwargs) -> np.ndarray:
    """vnlb.Basic: contribution stacks [frames, planes, slots*2*H, W]."""
    return _StageFilter(lib.STAGE_BASIC, clip, None, sigma, kwargs, _STAGE_ARGS, mvfw, mvbw, clip_props).render()


def Final(clip, ref=None, sigma=None, mvfw=None, mvbw=None, clip_props=None, **kwargs) -> np.ndarray:
    """vnlb.Final: contribution stacks of the Final stage matched on `ref`."""
    clip = _clip(clip)
    if not isinstance(ref, np.ndarray) or ref.shape != clip.shape or ref.dtype != np.float32:
        _err("ref clip properties must match input clip")
    return _StageFilter(lib.STAGE_FINAL, clip, ref, sigma, kwargs,
                        _STAGE_ARGS + ("sigma_basic", "gamma", "flat_areas"), mvfw, mvbw, clip_props).render()


def Aggregate(clip, src=None, patch_time=None, radius=None, search_bwd=None, search_fwd=None) -> np.ndarray:
    """vnlb.Aggregate: normalises the stacks of the contributing anchors."""
    if not isinstance(clip, np.ndarray) or not isinstance(src, np.ndarray) or clip.dtype != np.float32 or \
            src.dtype != np.float32 or clip.ndim != 4 or src.ndim != 4 or clip.shape[1] != src.shape[1] or \
            src.shape[1] not in (1, 3):
        _err("Aggregate requires matching constant GrayS or YUV444PS clips")
    pt, sb, sf = parse_temporal(dict(patch_time=patch_time, radius=radius, search_bwd=search_bwd,
                                     search_fwd=search_fwd))
    slots = sb + sf + pt
    frames, planes, height, width = src.shape
    if clip.shape != (frames, planes, height * 2 * slots, width):
        _err("contribution stack layout does not match src and parameters")
    return lib.aggregate(clip, src, sb, sf, pt)
