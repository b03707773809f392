"""Seeded synthetic planes for the BM3D workloads.

Clean plane: piecewise-smooth in [0, 1] -- 40 random axis-aligned rectangles
and discs, each filled with a linear intensity gradient, over a random flat
background, plus one sinusoidal texture of amplitude 0.1 and a random
frequency of 0.02-0.2 cycles/pixel, clipped to [0, 1].
Noisy plane: clean + i.i.d. N(0, sigma^2) from an independent seed, not clipped.

The reference scales sigma by the OPP luma norm 1/sqrt(3) even for a single
plane (include/BM3D.h:246-253); ``sigma_param`` gives the parameter value whose
effective noise level equals the injected one.
"""
from __future__ import annotations

import math

import numpy as np

OPP_NORM = (1.0 / math.sqrt(3.0), math.sqrt(0.5), math.sqrt(0.375))


def sigma_param(sigma_255: float, plane: int = 0) -> float:
    """Parameter sigma (0-255 scale) for true noise std sigma_255/255 on `plane`."""
    return sigma_255 / OPP_NORM[plane]


def clean_plane(height: int, width: int, seed: int, shapes: int = 40) -> np.ndarray:
    rng = np.random.default_rng(seed)
    img = np.full((height, width), rng.uniform(0.2, 0.8), np.float64)
    scale = float(max(height, width))
    for _ in range(shapes):
        disc = rng.random() < 0.5
        size = rng.uniform(0.05, 0.35) * scale
        cy, cx = rng.uniform(0, height), rng.uniform(0, width)
        base = rng.uniform(0.0, 1.0)
        gy, gx = rng.uniform(-0.6, 0.6, 2) / scale
        if disc:
            r = size / 2
            y0, y1 = int(max(0, cy - r)), int(min(height, cy + r + 1))
            x0, x1 = int(max(0, cx - r)), int(min(width, cx + r + 1))
        else:
            hh, hw = size * rng.uniform(0.3, 1.0) / 2, size * rng.uniform(0.3, 1.0) / 2
            y0, y1 = int(max(0, cy - hh)), int(min(height, cy + hh + 1))
            x0, x1 = int(max(0, cx - hw)), int(min(width, cx + hw + 1))
        if y1 <= y0 or x1 <= x0:
            continue
        yy, xx = np.mgrid[y0:y1, x0:x1].astype(np.float64)
        val = base + gy * (yy - cy) + gx * (xx - cx)
        if disc:
            mask = (yy - cy) ** 2 + (xx - cx) ** 2 <= (size / 2) ** 2
            sub = img[y0:y1, x0:x1]
            sub[mask] = val[mask]
        else:
            img[y0:y1, x0:x1] = val
    f = rng.uniform(0.02, 0.2)
    theta = rng.uniform(0, math.pi)
    phase = rng.uniform(0, 2 * math.pi)
    yy, xx = np.mgrid[0:height, 0:width].astype(np.float64)
    img += 0.1 * np.sin(2 * math.pi * f * (xx * math.cos(theta) + yy * math.sin(theta)) + phase)
    return np.clip(img, 0.0, 1.0).astype(np.float32)


def noisy_plane(clean: np.ndarray, sigma_255: float, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    noise = rng.standard_normal(clean.shape) * (sigma_255 / 255.0)
    return (clean.astype(np.float64) + noise).astype(np.float32)


def pair(height: int, width: int, sigma_255: float, seed: int):
    """(clean, noisy) with seeds `seed` (image) and `seed + 1_000_003` (noise)."""
    clean = clean_plane(height, width, seed)
    return clean, noisy_plane(clean, sigma_255, seed + 1_000_003)


def psnr(a: np.ndarray, b: np.ndarray, peak: float = 1.0) -> float:
    mse = float(np.mean((np.asarray(a, np.float64) - np.asarray(b, np.float64)) ** 2))
    return float("inf") if mse == 0 else 10.0 * math.log10(peak * peak / mse)


def int_planes(h: int, w: int, s255: float, seed: int, lo: int, hi: int, n: int):
    """n seeded int32 planes: smooth content spanning [lo, hi] plus Gaussian
    noise of sigma s255 / 255 of the range, rounded and clipped to [lo, hi]."""
    rng = np.random.default_rng(seed)
    out = []
    for c in range(n):
        clean = clean_plane(h, w, seed * 7 + c)
        v = lo + clean * (hi - lo) + rng.normal(0.0, s255 / 255.0 * (hi - lo), (h, w))
        out.append(np.clip(np.round(v), lo, hi).astype(np.int32))
    return out
