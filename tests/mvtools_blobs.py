"""Synthetic MVTools frame properties for the flow-guided search tests.

MVTools attaches two binary properties to every frame of a vector clip:
MVTools_MVAnalysisData (21 little-endian 32-bit fields; the reference reads
fields 2-7 and 10-20, src/flow/flow.hpp:193-250) and MVTools_vectors (u32
total size, u32 valid flag, then one block per search level, each a u32 byte
size followed by 16-byte vectors i32 x, i32 y, u64 SAD, coarsest first; the
reference uses the last, finest level, flow.hpp:252-318).  These builders
write both from arrays, and `flow_grids` gives the same vectors in the oracle's
FlowGrids form.
"""
from __future__ import annotations

import struct
from dataclasses import dataclass

import numpy as np


@dataclass
class Direction:
    block_size: int
    overlap: int
    pel: int
    backwards: bool
    vectors: np.ndarray  # int32 [frames, block_count_y, block_count_x, 2], sub-pel units
    valid: np.ndarray    # bool [frames]: the MVTools_vectors valid flag
    scene: np.ndarray    # bool [frames]: scene change flag of the source clip's frame


def analysis_blob(d: Direction, width: int, height: int, delta: int = 1, levels: int = 2) -> bytes:
    bcy, bcx = d.vectors.shape[1:3]
    f = [0] * 21
    f[2], f[3], f[4], f[5] = d.block_size, d.block_size, d.pel, levels
    f[6] = delta & 0xFFFFFFFF
    f[7] = 1 if d.backwards else 0
    f[10], f[11] = width, height
    f[12], f[13] = d.overlap, d.overlap
    f[14], f[15] = bcx, bcy
    f[16], f[17], f[18], f[19], f[20] = 8, 1, 1, 16, 16
    return struct.pack("<21I", *f)


def vectors_blob(vectors: np.ndarray, valid: bool = True, coarse: int = 1) -> bytes:
    """One frame's MVTools_vectors: `coarse` coarse levels of 4 vectors, then
    the finest level holding `vectors` [block_count_y, block_count_x, 2]."""
    body = b""
    for level in range(coarse):
        data = b"".join(struct.pack("<iiQ", 7 * level, -3, 99) for _ in range(4))
        body += struct.pack("<I", 4 + len(data)) + data
    flat = vectors.reshape(-1, 2)
    data = b"".join(struct.pack("<iiQ", int(x), int(y), 1234) for x, y in flat)
    body += struct.pack("<I", 4 + len(data)) + data
    return struct.pack("<II", 8 + len(body), 1 if valid else 0) + body


def random_direction(rng, frames: int, width: int, height: int, block_size: int, overlap: int, pel: int,
                     backwards: bool, reach: int, unusable: float = 0.2) -> Direction:
    """Random vectors of up to +-reach whole pixels; a share of the frames
    invalid or marked as scene changes."""
    step = block_size - overlap
    bcx, bcy = -(-width // step), -(-height // step)
    vectors = rng.integers(-reach * pel, reach * pel + 1, (frames, bcy, bcx, 2)).astype(np.int32)
    bad = rng.random(frames) < unusable
    valid = ~(bad & (rng.random(frames) < 0.5))
    scene = bad & valid
    return Direction(block_size, overlap, pel, backwards, vectors, valid, scene)


def props(d: Direction, width: int, height: int):
    """The vector clip's per-frame property mappings."""
    a = analysis_blob(d, width, height)
    return [{"MVTools_MVAnalysisData": a, "MVTools_vectors": vectors_blob(d.vectors[n], bool(d.valid[n]))}
            for n in range(d.vectors.shape[0])]


def clip_props(fw: Direction | None, bw: Direction | None, frames: int):
    """The source clip's per-frame scene-change properties."""
    out = [{} for _ in range(frames)]
    for n in range(frames):
        if fw is not None and fw.scene[n]:
            out[n]["_SceneChangePrev"] = 1
        if bw is not None and bw.scene[n]:
            out[n]["_SceneChangeNext"] = 1
    return out


def flow_grids(d: Direction | None):
    """The oracle's FlowGrids of one direction (usable = valid and no scene
    change, cache_mvtools_grid, src/vs/plugin.cpp:507-525)."""
    if d is None:
        return None
    import oracle as O
    return O.FlowGrids(d.block_size, d.block_size, d.pel, d.overlap, d.overlap,
                       (d.valid & ~d.scene).astype(np.uint8), d.vectors)


# (name, width, height, frames, planes, sigma, seed, kwargs, fw (block, overlap, pel, reach) or None, bw)
FLOW_CASES = [
    ("gray_fw_bw_pel2", 48, 40, 6, 1, 20.0, 21, dict(radius=2, block_step=4, bm_range=5), (8, 4, 2, 5),
     (8, 4, 2, 5)),
    ("yuv_fw_pel4_overlap0", 40, 32, 5, 3, 20.0, 22, dict(radius=2, block_step=4, bm_range=4), (16, 0, 4, 9),
     None),
    ("gray_bw_pel1_far", 48, 40, 5, 1, 15.0, 23, dict(radius=1, bm_range=3, block_step=4), None, (8, 2, 1, 12)),
    ("yuv_fw_bw_patch_time2", 40, 32, 5, 3, 20.0, 24,
     dict(radius=1, block_size=7, patch_time=2, block_step=3, bm_range=4), (8, 4, 2, 3), (8, 4, 2, 3)),
]


def flow_case(name, w, h, f, planes, sigma, seed, kw, fw_spec, bw_spec):
    """The clip and the two directions of one flow case (deterministic)."""
    import synth
    _, noisy = synth.make_clip(w, h, f, planes, sigma, seed=seed)
    rng = np.random.default_rng(seed)
    fw = random_direction(rng, f, w, h, *fw_spec[:3], False, fw_spec[3]) if fw_spec else None
    bw = random_direction(rng, f, w, h, *bw_spec[:3], True, bw_spec[3]) if bw_spec else None
    return noisy, fw, bw
