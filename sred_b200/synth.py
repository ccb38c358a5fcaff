"""Seeded synthetic microscopy-like images for benchmarks and tests.

Spots are Gaussian blobs on a background, placed on a jittered square lattice
(optionally plus randomly placed and elongated spots), then shot noise
(Poisson) and Gaussian read noise are applied. All randomness comes from
``numpy.random.default_rng(seed)``; no external dataset is involved.
"""
from __future__ import annotations

import numpy as np


def spot_image(width: int, height: int, lattice: int, *, seed: int = 0, background: float = 100.0,
               sigma: float = 2.0, amp_range=(50.0, 200.0), jitter: float = 1.5,
               random_fraction: float = 0.0, elongated_fraction: float = 0.0,
               elongated_sigma=(4.0, 1.5), read_noise: float = 10.0) -> np.ndarray:
    """float32 [height, width] image.

    ``lattice`` spots per side are placed on a square lattice spanning the
    image, each jittered by U(-jitter, jitter) px; ``random_fraction`` adds that
    fraction of extra spots at uniform positions; ``elongated_fraction`` of all
    spots get anisotropic widths ``elongated_sigma`` at a uniform angle."""
    rng = np.random.default_rng(seed)
    img = np.full((height, width), background, np.float64)
    sx, sy = width / lattice, height / lattice
    gy, gx = np.mgrid[0:lattice, 0:lattice]
    cx = (gx.ravel() + 0.5) * sx + rng.uniform(-jitter, jitter, lattice * lattice)
    cy = (gy.ravel() + 0.5) * sy + rng.uniform(-jitter, jitter, lattice * lattice)
    n_rand = int(round(random_fraction * lattice * lattice))
    if n_rand:
        cx = np.concatenate([cx, rng.uniform(0, width, n_rand)])
        cy = np.concatenate([cy, rng.uniform(0, height, n_rand)])
    n = cx.size
    amp = rng.uniform(amp_range[0], amp_range[1], n)
    elong = rng.uniform(0, 1, n) < elongated_fraction
    theta = rng.uniform(0, np.pi, n)
    for i in range(n):
        if elong[i]:
            s1, s2 = elongated_sigma
        else:
            s1 = s2 = sigma
        r = int(np.ceil(4 * max(s1, s2)))
        x0, x1 = max(int(cx[i]) - r, 0), min(int(cx[i]) + r + 1, width)
        y0, y1 = max(int(cy[i]) - r, 0), min(int(cy[i]) + r + 1, height)
        if x0 >= x1 or y0 >= y1:
            continue
        yy, xx = np.mgrid[y0:y1, x0:x1]
        dx, dy = xx - cx[i], yy - cy[i]
        c, s = np.cos(theta[i]), np.sin(theta[i])
        u, v = c * dx + s * dy, -s * dx + c * dy
        img[y0:y1, x0:x1] += amp[i] * np.exp(-0.5 * ((u / s1) ** 2 + (v / s2) ** 2))
    img = rng.poisson(img).astype(np.float64) + rng.normal(0.0, read_noise, img.shape)
    return img.astype(np.float32)


def spot_volume(width: int, height: int, depth: int, lattice: int, lattice_z: int, *, seed: int = 0,
                background: float = 100.0, sigma: float = 2.0, sigma_z: float = 1.5, amp_range=(50.0, 200.0),
                jitter: float = 1.5, read_noise: float = 10.0) -> np.ndarray:
    """float32 [depth, height, width] volume: isotropic-in-xy Gaussian spots
    (width ``sigma``, ``sigma_z`` along z) on a jittered lattice of
    ``lattice`` x ``lattice`` x ``lattice_z`` sites, Poisson shot noise and
    Gaussian read noise."""
    rng = np.random.default_rng(seed)
    vol = np.full((depth, height, width), background, np.float64)
    sx, sy, sz = width / lattice, height / lattice, depth / lattice_z
    gz, gy, gx = np.mgrid[0:lattice_z, 0:lattice, 0:lattice]
    n = gx.size
    cx = (gx.ravel() + 0.5) * sx + rng.uniform(-jitter, jitter, n)
    cy = (gy.ravel() + 0.5) * sy + rng.uniform(-jitter, jitter, n)
    cz = (gz.ravel() + 0.5) * sz + rng.uniform(-jitter / 2, jitter / 2, n)
    amp = rng.uniform(amp_range[0], amp_range[1], n)
    r, rz = int(np.ceil(4 * sigma)), int(np.ceil(4 * sigma_z))
    for i in range(n):
        x0, x1 = max(int(cx[i]) - r, 0), min(int(cx[i]) + r + 1, width)
        y0, y1 = max(int(cy[i]) - r, 0), min(int(cy[i]) + r + 1, height)
        z0, z1 = max(int(cz[i]) - rz, 0), min(int(cz[i]) + rz + 1, depth)
        if x0 >= x1 or y0 >= y1 or z0 >= z1:
            continue
        zz, yy, xx = np.mgrid[z0:z1, y0:y1, x0:x1]
        d2 = ((xx - cx[i]) ** 2 + (yy - cy[i]) ** 2) / sigma ** 2 + (zz - cz[i]) ** 2 / sigma_z ** 2
        vol[z0:z1, y0:y1, x0:x1] += amp[i] * np.exp(-0.5 * d2)
    vol = rng.poisson(vol).astype(np.float64) + rng.normal(0.0, read_noise, vol.shape)
    return vol.astype(np.float32)


def normalize_input(img: np.ndarray) -> np.ndarray:
    """Min-max to [0, 1] with the reference's epsilon, in FP32 (java/Utils.java:707-722)."""
    a = np.ascontiguousarray(img, dtype=np.float32)
    mn, mx = np.float32(a.min()), np.float32(a.max())
    return ((a - mn) / (mx - mn + np.float32(1e-7))).astype(np.float32)


# Workloads named by what they are (image side, block, spot layout).
def image_256_spots(seed: int = 0) -> np.ndarray:
    """256x256, 400 spots on a jittered 20x20 lattice."""
    return spot_image(256, 256, 20, seed=seed)


def image_1024_spots(seed: int = 0) -> np.ndarray:
    """1024x1024, 6,400 spots on a jittered 80x80 lattice."""
    return spot_image(1024, 1024, 80, seed=seed)


def image_1024_spots_random(seed: int = 0) -> np.ndarray:
    """1024x1024, 80x80 lattice plus 30% randomly placed spots."""
    return spot_image(1024, 1024, 80, seed=seed, random_fraction=0.3)


def image_2048_elongated(seed: int = 0) -> np.ndarray:
    """2048x2048, 25,600 spots on a 160x160 lattice, 10% elongated."""
    return spot_image(2048, 2048, 160, seed=seed, elongated_fraction=0.1)


def volume_512_spots(seed: int = 0) -> np.ndarray:
    """512x512x128 volume (134 MB as float32), 25,600 spots on a jittered
    40x40x16 lattice."""
    return spot_volume(512, 512, 128, 40, 16, seed=seed)
