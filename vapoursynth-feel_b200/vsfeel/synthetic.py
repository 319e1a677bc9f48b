"""Seeded synthetic clips for benchmarks and tests.

The reference's own test clip (tests/noise_24f.mkv) is not distributed, and
the reference benchmark denoises a blank clip (benchmark/bench.py:30-52), so
inputs are generated here with a fixed recipe:

* clean canvas: 20 axis-aligned rectangles of constant level U[0.1, 0.9]
  painted over a 0.5 background, plus 6 plane sinusoids (period U[8, 128] px,
  amplitude U[0.05, 0.15], orientation and phase uniform), clipped to [0, 1];
* frame f is the canvas translated by an integer offset drawn uniformly from
  [-shift, shift] in x and y;
* i.i.d. Gaussian noise of standard deviation sigma/255 is added per frame.

Geometry is drawn from ``numpy.random.default_rng(seed)`` and noise from
``numpy.random.default_rng([seed, 1])``, so a clean clip (``noise=False``)
lines up with its noisy twin frame for frame.
"""

from __future__ import annotations

import numpy as np


def clean_canvas(rng: np.random.Generator, height: int, width: int) -> np.ndarray:
    img = np.full((height, width), 0.5, dtype=np.float64)
    for _ in range(20):
        rw = int(rng.integers(max(1, width // 16), max(2, width // 3) + 1))
        rh = int(rng.integers(max(1, height // 16), max(2, height // 3) + 1))
        x0 = int(rng.integers(0, max(1, width - rw + 1)))
        y0 = int(rng.integers(0, max(1, height - rh + 1)))
        img[y0:y0 + rh, x0:x0 + rw] = rng.uniform(0.1, 0.9)
    yy, xx = np.meshgrid(np.arange(height, dtype=np.float64), np.arange(width, dtype=np.float64),
                         indexing="ij")
    for _ in range(6):
        period = rng.uniform(8.0, 128.0)
        amp = rng.uniform(0.05, 0.15)
        theta = rng.uniform(0.0, np.pi)
        phase = rng.uniform(0.0, 2.0 * np.pi)
        img += amp * np.sin(2.0 * np.pi * (xx * np.cos(theta) + yy * np.sin(theta)) / period + phase)
    return np.clip(img, 0.0, 1.0)


def make_clip(nframes: int, height: int, width: int, sigma: float = 3.0, shift: int = 3,
              seed: int = 0, noise: bool = True) -> np.ndarray:
    """Returns float32 frames of shape (nframes, height, width) in about [0, 1]."""
    rng = np.random.default_rng(seed)
    nrng = np.random.default_rng([seed, 1])
    canvas = clean_canvas(rng, height + 2 * shift, width + 2 * shift).astype(np.float32)
    out = np.empty((nframes, height, width), dtype=np.float32)
    for f in range(nframes):
        dx, dy = (int(v) for v in rng.integers(-shift, shift + 1, size=2))
        out[f] = canvas[shift + dy:shift + dy + height, shift + dx:shift + dx + width]
        if noise and sigma > 0:
            out[f] += nrng.standard_normal((height, width), dtype=np.float32) * np.float32(sigma / 255.0)
    return out


def make_clip_range(total: int, first: int, count: int, height: int, width: int,
                    sigma: float = 3.0, shift: int = 3, seed: int = 0) -> np.ndarray:
    """Frames first..first+count-1 of a `total`-frame clip, built without the
    others: make_clip's canvas and per-frame offsets (the same numpy draws),
    with each frame's noise from its own stream ``default_rng([seed, 2, f])``
    so that any range of a long clip -- one rank's shard -- can be generated
    alone. Returns float32 (count, height, width)."""
    if not (0 <= first and count >= 0 and first + count <= total):
        raise ValueError("frame range outside the clip")
    rng = np.random.default_rng(seed)
    canvas = clean_canvas(rng, height + 2 * shift, width + 2 * shift).astype(np.float32)
    offsets = rng.integers(-shift, shift + 1, size=(total, 2))
    out = np.empty((count, height, width), dtype=np.float32)
    for i in range(count):
        f = first + i
        dx, dy = (int(v) for v in offsets[f])
        out[i] = canvas[shift + dy:shift + dy + height, shift + dx:shift + dx + width]
        if sigma > 0:
            nrng = np.random.default_rng([seed, 2, f])
            out[i] += nrng.standard_normal((height, width), dtype=np.float32) * np.float32(sigma / 255.0)
    return out


def make_chroma(nframes: int, height: int, width: int, seed: int = 0) -> np.ndarray:
    """A smooth random sinusoid field in [0, 1] for pass-through chroma planes."""
    rng = np.random.default_rng(seed + 7919)
    yy, xx = np.meshgrid(np.arange(height, dtype=np.float32), np.arange(width, dtype=np.float32),
                         indexing="ij")
    out = np.empty((nframes, height, width), dtype=np.float32)
    for f in range(nframes):
        period = rng.uniform(32.0, 256.0)
        theta = rng.uniform(0.0, np.pi)
        phase = rng.uniform(0.0, 2.0 * np.pi)
        out[f] = 0.5 + 0.4 * np.sin(
            2.0 * np.pi * (xx * np.cos(theta) + yy * np.sin(theta)) / period + phase)
    return out


def make_clip_device(nframes: int, height: int, width: int, sigma: float = 3.0, shift: int = 3,
                     seed: int = 0, device="cuda"):
    """make_clip's recipe with the frames built on the GPU (for large
    benchmark batches): the canvas and the per-frame offsets come from the
    same numpy draws as make_clip; the noise comes from torch's generator
    seeded with `seed`, so the noise values differ from make_clip's."""
    import torch

    rng = np.random.default_rng(seed)
    canvas = torch.from_numpy(
        clean_canvas(rng, height + 2 * shift, width + 2 * shift).astype(np.float32)).to(device)
    gen = torch.Generator(device=device).manual_seed(int(seed))
    out = torch.empty((nframes, height, width), dtype=torch.float32, device=device)
    for f in range(nframes):
        dx, dy = (int(v) for v in rng.integers(-shift, shift + 1, size=2))
        out[f] = canvas[shift + dy:shift + dy + height, shift + dx:shift + dx + width]
        if sigma > 0:
            out[f] += torch.randn((height, width), generator=gen, device=device) * (sigma / 255.0)
    return out
