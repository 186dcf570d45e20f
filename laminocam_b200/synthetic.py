"""Seeded synthetic inputs (no datasets are available offline).

Ellipse (2D) and ellipsoid (3D) phantoms with the distributions of the
benchmark configurations: centres uniform in the unit disk / ball, semi-axes
uniform in [0.05, 0.4] of the normalised half-extent per axis, rotations
uniform, densities uniform in [0, 1], summed where they overlap.  Noise is
Gaussian with sigma = a fraction of the noise-free maximum.
"""
from __future__ import annotations

import numpy as np


def _grid(n: int) -> np.ndarray:
    """Pixel-centre coordinates in [-1, 1]."""
    return (2.0 * np.arange(n) + 1.0) / n - 1.0


def ellipse_phantom(n: int, count: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    y, x = np.meshgrid(_grid(n), _grid(n), indexing="ij")
    img = np.zeros((n, n), dtype=np.float64)
    for _ in range(count):
        r = np.sqrt(rng.uniform())
        phi = 2 * np.pi * rng.uniform()
        cx, cy = r * np.cos(phi), r * np.sin(phi)
        a, b = rng.uniform(0.05, 0.4, size=2)
        rot = rng.uniform(0, np.pi)
        dens = rng.uniform(0, 1)
        c, s = np.cos(rot), np.sin(rot)
        xr = (x - cx) * c + (y - cy) * s
        yr = -(x - cx) * s + (y - cy) * c
        img += dens * (((xr / a) ** 2 + (yr / b) ** 2) <= 1.0)
    return img.astype(np.float32)


def _euler(a, b, c):
    ca, sa, cb, sb, cc, sc = np.cos(a), np.sin(a), np.cos(b), np.sin(b), np.cos(c), np.sin(c)
    Rz1 = np.array([[ca, -sa, 0], [sa, ca, 0], [0, 0, 1]])
    Ry = np.array([[cb, 0, sb], [0, 1, 0], [-sb, 0, cb]])
    Rz2 = np.array([[cc, -sc, 0], [sc, cc, 0], [0, 0, 1]])
    return Rz1 @ Ry @ Rz2


def ellipsoid_phantom(dims, count: int, seed: int) -> np.ndarray:
    """dims = (n1, n2, n3) = (thickness, y, x); each axis normalised to [-1, 1]."""
    rng = np.random.default_rng(seed)
    n1, n2, n3 = dims
    vol = np.zeros(dims, dtype=np.float32)
    z = _grid(n1).astype(np.float32)
    y = _grid(n2).astype(np.float32)
    x = _grid(n3).astype(np.float32)
    for _ in range(count):
        while True:
            c = rng.uniform(-1, 1, size=3)
            if np.dot(c, c) <= 1.0:
                break
        axes = rng.uniform(0.05, 0.4, size=3)
        R = _euler(*rng.uniform(0, 2 * np.pi, size=3)).astype(np.float32)
        dens = np.float32(rng.uniform(0, 1))
        # bounding box in normalised coordinates
        ext = np.abs(R) @ axes
        lo = c - ext
        hi = c + ext
        iz = np.nonzero((z >= lo[0]) & (z <= hi[0]))[0]
        iy = np.nonzero((y >= lo[1]) & (y <= hi[1]))[0]
        ix = np.nonzero((x >= lo[2]) & (x <= hi[2]))[0]
        if len(iz) == 0 or len(iy) == 0 or len(ix) == 0:
            continue
        Z, Y, X = np.meshgrid(z[iz] - c[0], y[iy] - c[1], x[ix] - c[2], indexing="ij")
        P = np.stack([Z, Y, X], axis=-1) @ R  # rotate into the ellipsoid frame
        inside = ((P / axes.astype(np.float32)) ** 2).sum(-1) <= 1.0
        vol[np.ix_(iz, iy, ix)] += dens * inside
    return vol


def add_noise(data: np.ndarray, frac: float, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    sigma = frac * float(np.max(data))
    return (data + rng.normal(0.0, sigma, size=data.shape)).astype(np.float32)
