"""Seeded synthetic clips that stand in for real video in tests and the bench.

No public dataset is named for the VNLB path, so every workload here is
generated.  A clean plane is a sum of six sinusoids of random orientation
(period 4-64 px, amplitude 0.05-0.15) plus a linear gradient plus ten constant
rectangles, clipped to [0, 1].  Each frame is the same scene moved by a random
integer step (dx, dy) in [-2, 2]^2 from the previous frame (global motion).
YUV planes use independent scene seeds, with chroma deviations scaled by 0.3.
Noise is i.i.d. N(0, (sigma/255)^2), drawn per plane from its own seed.

Layout of every clip: float32 array [frames, channels, height, width].
"""
from __future__ import annotations

import numpy as np


def _scene(rng: np.random.Generator):
    waves = []
    for _ in range(6):
        theta = rng.uniform(0.0, np.pi)
        period = rng.uniform(4.0, 64.0)
        amp = rng.uniform(0.05, 0.15)
        phase = rng.uniform(0.0, 2.0 * np.pi)
        waves.append((np.cos(theta) * 2 * np.pi / period,
                      np.sin(theta) * 2 * np.pi / period, amp, phase))
    gradient = rng.uniform(-0.15, 0.15, size=2)
    rects = []
    for _ in range(10):
        w, h = rng.uniform(0.05, 0.25, size=2)
        x0, y0 = rng.uniform(0.0, 1.0, size=2)
        rects.append((x0, y0, w, h, rng.uniform(0.1, 0.9)))
    return waves, gradient, rects


def _render(scene, xs: np.ndarray, ys: np.ndarray, width: int, height: int,
            chroma_scale: float) -> np.ndarray:
    waves, gradient, rects = scene
    value = np.zeros(np.broadcast(xs, ys).shape, dtype=np.float64)
    for kx, ky, amp, phase in waves:
        value += amp * np.sin(kx * xs + ky * ys + phase)
    value += gradient[0] * (xs / width - 0.5) + gradient[1] * (ys / height - 0.5)
    for x0, y0, w, h, level in rects:
        inside = ((xs >= x0 * width) & (xs < (x0 + w) * width) &
                  (ys >= y0 * height) & (ys < (y0 + h) * height))
        value = np.where(inside, level - 0.5, value)
    return np.clip(0.5 + chroma_scale * value, 0.0, 1.0)


def make_clip(width: int, height: int, frames: int, channels: int,
              sigma: float, seed: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """Returns (clean, noisy), both float32 [frames, channels, height, width].

    sigma is on the 8-bit scale (the plugin's sigma argument)."""
    if channels not in (1, 3):
        raise ValueError("channels must be 1 (GrayS) or 3 (YUV444PS)")
    motion_rng = np.random.default_rng([seed, 0x6d6f74])
    steps = motion_rng.integers(-2, 3, size=(frames, 2))
    steps[0] = 0
    offsets = np.cumsum(steps, axis=0)
    clean = np.empty((frames, channels, height, width), dtype=np.float32)
    noisy = np.empty_like(clean)
    yy, xx = np.mgrid[0:height, 0:width].astype(np.float64)
    for c in range(channels):
        scene = _scene(np.random.default_rng([seed, 0x736365, c]))
        noise_rng = np.random.default_rng([seed, 0x6e6f69, c])
        scale = 1.0 if c == 0 else 0.3
        for f in range(frames):
            ox, oy = offsets[f]
            plane = _render(scene, xx + ox, yy + oy, width, height, scale)
            clean[f, c] = plane
            noisy[f, c] = plane + noise_rng.normal(
                0.0, sigma / 255.0, size=(height, width))
    return clean, noisy.astype(np.float32)


def psnr(a: np.ndarray, b: np.ndarray) -> float:
    """PSNR in dB for signals on the [0, 1] scale."""
    mse = float(np.mean((np.asarray(a, np.float64) - np.asarray(b, np.float64)) ** 2))
    return float("inf") if mse == 0.0 else 10.0 * np.log10(1.0 / mse)
