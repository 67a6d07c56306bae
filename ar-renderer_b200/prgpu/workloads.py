"""Seeded synthetic workloads.

Traversal microbenchmark (the 1,048,576-triangle soup): triangle centroids uniform in the unit
cube, each vertex = centroid + a offset uniform in [-0.01, 0.01]^3; rays with origins uniform in
[-0.5, 1.5]^3 and directions uniform on the sphere (the warp of pbrt's SampleUniformSphere,
src/core/sampling.h:31-37); closest-hit queries use tMax = inf, any-hit queries tMax uniform in
[0, 2]. Geometry uses seed 1 and rays seed 2 by default.
"""

from __future__ import annotations

import numpy as np

from . import abi


def triangle_soup(n: int, seed: int = 1, edge: float = 0.01) -> np.ndarray:
    """(n, 3, 3) float32 vertices."""
    rng = np.random.default_rng(seed)
    c = rng.random((n, 1, 3), dtype=np.float32)
    e = rng.uniform(-edge, edge, (n, 3, 3)).astype(np.float32)
    return np.ascontiguousarray((c + e).astype(np.float32))


def sphere_directions(u: np.ndarray) -> np.ndarray:
    z = 1.0 - 2.0 * u[:, 0]
    r = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    phi = 2.0 * np.pi * u[:, 1]
    return np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=1).astype(np.float32)


def soup_rays(n: int, seed: int = 2, any_hit: bool = False) -> np.ndarray:
    """Structured array of prgpu::Ray (32 bytes each)."""
    rng = np.random.default_rng(seed)
    o = rng.uniform(-0.5, 1.5, (n, 3)).astype(np.float32)
    d = sphere_directions(rng.random((n, 2), dtype=np.float32))
    r = np.zeros(n, dtype=abi.RAY)
    r["o"] = o
    r["d"] = d
    r["tMax"] = rng.uniform(0.0, 2.0, n).astype(np.float32) if any_hit else np.float32(np.inf)
    return r


def rays_as_f8(rays: np.ndarray) -> np.ndarray:
    """The same rays as an (n, 8) float32 view: o, d, tMax, pad (the oracle's layout)."""
    out = np.zeros((rays.shape[0], 8), dtype=np.float32)
    out[:, 0:3] = rays["o"]
    out[:, 3:6] = rays["d"]
    out[:, 6] = rays["tMax"]
    return out
