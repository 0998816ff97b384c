"""Seeded synthetic clips with the shapes and statistics of the benchmark
workloads (no external dataset exists for this path; all inputs are made
here from a seed).

* piecewise_clip: 40 random axis-aligned rectangles of uniform[0,1]
  intensity over a linear gradient, plus AWGN (BM3D basic 640x360 workload).
* texture_clip: band-limited texture (uniform noise, Gaussian blur of
  sigma 2 px) translated per frame by random integer motion in [-3, 3] px,
  plus AWGN (V-BM3D 1920x1080 workload).
* chroma_clip: Y as piecewise_clip, U/V = 0.3 * smooth(Y) + independent
  AWGN (CBM3D YUV444 workload).
"""
from __future__ import annotations

import numpy as np


def _gaussian(img: np.ndarray, sigma: float) -> np.ndarray:
    from scipy.ndimage import gaussian_filter
    return gaussian_filter(img, sigma, mode="reflect")


def piecewise_image(rng: np.random.Generator, height: int, width: int, rects: int = 40) -> np.ndarray:
    gx = np.linspace(0.0, 1.0, width, dtype=np.float64)[None, :]
    gy = np.linspace(0.0, 1.0, height, dtype=np.float64)[:, None]
    a, b = rng.uniform(-0.5, 0.5, size=2)
    img = 0.5 + a * (gx - 0.5) + b * (gy - 0.5)
    img = np.broadcast_to(img, (height, width)).copy()
    for _ in range(rects):
        x0, x1 = np.sort(rng.integers(0, width, size=2))
        y0, y1 = np.sort(rng.integers(0, height, size=2))
        img[y0:y1 + 1, x0:x1 + 1] = rng.uniform(0.0, 1.0)
    return img


def piecewise_clip(frames: int, height: int, width: int, noise: float = 10 / 255,
                   seed: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """Returns (noisy, clean), each [frames, height, width] float32."""
    rng = np.random.default_rng(seed)
    clean = np.stack([piecewise_image(rng, height, width) for _ in range(frames)])
    noisy = clean + rng.normal(0.0, noise, size=clean.shape)
    return noisy.astype(np.float32), clean.astype(np.float32)


def moving_piecewise_clip(frames: int, height: int, width: int, noise: float = 10 / 255,
                          max_motion: int = 3, seed: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """A piecewise image (as piecewise_clip) translated per frame by random
    integer motion in [-max_motion, max_motion] px, plus AWGN: the training
    clips of the learned match proposer. Returns (noisy, clean)."""
    rng = np.random.default_rng(seed)
    steps = rng.integers(-max_motion, max_motion + 1, size=(frames, 2))
    steps[0] = 0
    path = np.cumsum(steps, axis=0)
    pad_y = int(np.abs(path[:, 0]).max()) + 8
    pad_x = int(np.abs(path[:, 1]).max()) + 8
    img = piecewise_image(rng, height + 2 * pad_y, width + 2 * pad_x)
    clean = np.stack([img[pad_y + dy:pad_y + dy + height, pad_x + dx:pad_x + dx + width]
                      for dy, dx in path])
    noisy = clean + rng.normal(0.0, noise, size=clean.shape)
    return noisy.astype(np.float32), clean.astype(np.float32)


def texture_clip(frames: int, height: int, width: int, noise: float = 5 / 255,
                 blur: float = 2.0, max_motion: int = 3, seed: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """Returns (noisy, clean), each [frames, height, width] float32."""
    rng = np.random.default_rng(seed)
    steps = rng.integers(-max_motion, max_motion + 1, size=(frames, 2))
    steps[0] = 0
    path = np.cumsum(steps, axis=0)
    pad_y = int(np.abs(path[:, 0]).max()) + 8
    pad_x = int(np.abs(path[:, 1]).max()) + 8
    base = rng.uniform(0.0, 1.0, size=(height + 2 * pad_y, width + 2 * pad_x))
    tex = _gaussian(base, blur)
    tex = (tex - tex.mean()) / (tex.std() + 1e-12) * 0.15 + 0.5
    clean = np.stack([tex[pad_y + dy:pad_y + dy + height, pad_x + dx:pad_x + dx + width]
                      for dy, dx in path])
    noisy = clean + rng.normal(0.0, noise, size=clean.shape)
    return noisy.astype(np.float32), clean.astype(np.float32)


def chroma_clip(frames: int, height: int, width: int, noise=(10 / 255, 7 / 255, 7 / 255),
                seed: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """Returns (noisy, clean), each [frames, 3, height, width] float32 (YUV444)."""
    rng = np.random.default_rng(seed)
    y = np.stack([piecewise_image(rng, height, width) for _ in range(frames)])
    u = np.stack([0.3 * _gaussian(f, 2.0) for f in y])
    v = np.stack([0.3 * _gaussian(f, 3.0) for f in y])
    clean = np.stack([y, u, v], axis=1)
    noisy = clean.copy()
    for i, s in enumerate(noise):
        noisy[:, i] += rng.normal(0.0, s, size=y.shape)
    return noisy.astype(np.float32), clean.astype(np.float32)


def psnr(a: np.ndarray, b: np.ndarray, peak: float = 1.0) -> float:
    mse = float(np.mean((np.asarray(a, np.float64) - np.asarray(b, np.float64)) ** 2))
    return float("inf") if mse == 0 else 10.0 * np.log10(peak * peak / mse)
