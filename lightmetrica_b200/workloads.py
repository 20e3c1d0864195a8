"""Seeded synthetic inputs with the shapes and distributions of the
benchmark configurations (the reference publishes no scenes or datasets).

* ``random_soup``: triangle soup, centres uniform in [-1,1]^3, edge vectors
  Gaussian (sigma 0.01 by default), one primitive, world space.
* ``random_rays``: origins uniform in [-2,2]^3, directions uniform on the
  sphere (z = 1 - 2u, phi = 2 pi u'), minT 0, maxT FLT_MAX.
"""
from __future__ import annotations

import numpy as np

FLT_MAX = float(np.finfo(np.float32).max)


def random_soup(num_tris: int, seed: int = 1, sigma: float = 0.01):
    """Returns (positions (3n,3) float32, faces (n,3) uint32); every triangle
    owns its three vertices. The centroid of triangle i is its centre."""
    rng = np.random.default_rng(seed)
    c = rng.uniform(-1.0, 1.0, size=(num_tris, 3))
    e1 = rng.normal(0.0, sigma, size=(num_tris, 3))
    e2 = rng.normal(0.0, sigma, size=(num_tris, 3))
    v0 = c - (e1 + e2) / 3.0
    pos = np.stack([v0, v0 + e1, v0 + e2], axis=1).astype(np.float32).reshape(-1, 3)
    faces = np.arange(3 * num_tris, dtype=np.uint32).reshape(-1, 3)
    return pos, faces


def random_rays(num_rays: int, seed: int = 2, extent: float = 2.0):
    """Returns (num_rays, 8) float32 AoS rays: o.xyz, d.xyz, minT, maxT."""
    rng = np.random.default_rng(seed)
    o = rng.uniform(-extent, extent, size=(num_rays, 3))
    u = rng.random(num_rays)
    w = rng.random(num_rays)
    z = 1.0 - 2.0 * u
    r = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    phi = 2.0 * np.pi * w
    d = np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=1)
    rays = np.empty((num_rays, 8), np.float32)
    rays[:, 0:3] = o
    rays[:, 3:6] = d
    rays[:, 6] = 0.0
    rays[:, 7] = FLT_MAX
    return rays


def rays_soa(rays):
    """AoS (n, 8) -> dict of contiguous SoA float32 arrays."""
    rays = np.asarray(rays, np.float32)
    names = ("ox", "oy", "oz", "dx", "dy", "dz", "tmin", "tmax")
    return {k: np.ascontiguousarray(rays[:, i]) for i, k in enumerate(names)}
