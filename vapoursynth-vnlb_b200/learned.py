"""Learned block-match proposals: training pairs, training and evaluation.

The network (vnlbgpu_lib.MLP, hand-written CUDA forward and backward kernels)
reads, for every anchor, the coarse features the learned form computes (3 x 3
cells of 16 x 16 box means around the patch centre, in every scheduled frame
and search plane, minus the anchor frame's centre cell) and scores every
offset of the search window (class = scheduled frame, window row, window
column).  Its targets are the offsets of the K nearest rows of the full exact
search on synthetic clips (vnlbgpu_learned_pairs), so the plain matcher
teaches it.  A session of form "learned" then runs exact SSD on the top
`shortlist` offsets only, with the full search as the check and fallback per
tile.

Device buffers come from torch (plumbing only); every computation is the
library's own kernels.
"""
from __future__ import annotations

import numpy as np

import synth
import vnlbcu
import vnlbgpu_lib as lib


def session(stage: int, clip: np.ndarray, sigma: float, kw: dict, ref: np.ndarray | None = None,
            form: str = "plain") -> lib.Session:
    params = vnlbcu.parse_parameters(stage, clip, sigma, dict(kw, form=form))
    frames, planes, h, w = clip.shape
    s = lib.Session(params, w, h, frames, planes)
    s.set_clip(lib.SOURCE_CLIP, clip)
    if stage == lib.STAGE_FINAL:
        s.set_clip(lib.SOURCE_REF, ref)
    return s


def network_shape(stage: int, planes: int, kw: dict, clip: np.ndarray, sigma: float):
    """(inputs, outputs) of the learned form's network for these parameters."""
    p = vnlbcu.parse_parameters(stage, clip, sigma, dict(kw))
    slots = p.search_bwd + p.search_fwd + 1
    search_planes = planes if stage == lib.STAGE_FINAL else 1
    return slots * search_planes * 9, slots * p.search_window * p.search_window


def training_pairs(stage: int, clips, sigma: float, kw: dict, refs=None, k: int = 8):
    """Features and target classes of every grid anchor of every anchor frame
    of `clips` (full exact search), stacked."""
    feats, targets = [], []
    for i, clip in enumerate(clips):
        s = session(stage, clip, sigma, kw, refs[i] if refs is not None else None)
        p = s.params
        for anchor in range(clip.shape[0] - p.patch_time + 1):
            f, t = s.learned_pairs(anchor, k)
            feats.append(f)
            targets.append(t)
        s.close()
    return np.concatenate(feats), np.concatenate(targets)


def train(mlp: lib.MLP, features: np.ndarray, targets: np.ndarray, steps: int, batch: int = 1024,
          lr: float = 1e-3, seed: int = 0) -> list[float]:
    """Adam steps on random batches; returns the batch losses."""
    import torch

    x = torch.from_numpy(np.ascontiguousarray(features, np.float32)).cuda()
    t = torch.from_numpy(np.ascontiguousarray(targets, np.int32)).cuda()
    rng = np.random.default_rng(seed)
    n, tk = t.shape
    losses = []
    xb = torch.empty((batch, x.shape[1]), dtype=torch.float32, device="cuda")
    tb = torch.empty((batch, tk), dtype=torch.int32, device="cuda")
    for _ in range(steps):
        idx = torch.from_numpy(rng.integers(0, n, batch)).cuda()
        torch.index_select(x, 0, idx, out=xb)
        torch.index_select(t, 0, idx, out=tb)
        torch.cuda.synchronize()
        losses.append(mlp.train_step(xb.data_ptr(), tb.data_ptr(), batch, tk, lr))
    return losses


def recall(mlp: lib.MLP, features: np.ndarray, targets: np.ndarray, shortlist: int = 64) -> float:
    """Mean over anchors of the share of their target classes in the
    network's `shortlist` best-scored offsets."""
    import torch

    x = torch.from_numpy(np.ascontiguousarray(features, np.float32)).cuda()
    out = torch.empty((x.shape[0], shortlist), dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    mlp.shortlist(x.data_ptr(), x.shape[0], shortlist, out.data_ptr())
    got = out.cpu().numpy()
    hits, total = 0, 0
    for row, t in zip(got, targets):
        valid = t[t >= 0]
        total += valid.size
        hits += np.isin(valid, row).sum()
    return hits / max(total, 1)


def synthetic_clips(w: int, h: int, frames: int, planes: int, sigma: float, seeds):
    return [synth.make_clip(w, h, frames, planes, sigma, seed=s)[1] for s in seeds]
