"""Heterogeneous (voxel grid) media for prgpu_render_ex: Mitsuba 0.5 binary .vol files as
pr::VoxelGridField::LoadVol reads them (src/media/medium.cpp:130-166: "VOL", version 3, encoding
1 = float32, nx ny nz channels, a float bounding box, then x-fastest voxels with the channels
averaged), and the GridMediumDesc records that hand a grid to the device.

A grid medium is referenced from Primitive::mediumInside/Outside and SceneDesc::cameraMedium by
the index mediumCount + k, k its position in SceneExt::gridMedia.
"""

from __future__ import annotations

import ctypes as C
import struct

import numpy as np

from . import abi

_HEADER = struct.Struct("<3sBiiiii6f")


def write_vol(path: str, density: np.ndarray, bounds) -> str:
    """density: (nz, ny, nx) float32 (x fastest in memory); bounds: ((x0, y0, z0), (x1, y1, z1))."""
    d = np.ascontiguousarray(density, dtype=np.float32)
    if d.ndim != 3:
        raise ValueError("density must be (nz, ny, nx)")
    nz, ny, nx = d.shape
    b = np.asarray(bounds, dtype=np.float32).reshape(6)
    with open(path, "wb") as f:
        f.write(_HEADER.pack(b"VOL", 3, 1, nx, ny, nz, 1, *[float(x) for x in b]))
        f.write(d.tobytes())
    return path


def read_vol(path: str):
    """(density (nz, ny, nx) float32 with the channels averaged, bounds (2, 3) float32).
    Raises ValueError on anything pr::VoxelGridField::LoadVol rejects."""
    with open(path, "rb") as f:
        head = f.read(_HEADER.size)
        if len(head) != _HEADER.size:
            raise ValueError(path + ": not a float32 Mitsuba .vol (version 3) file")
        magic, version, enc, nx, ny, nz, ch, *bb = _HEADER.unpack(head)
        if (magic != b"VOL" or version != 3 or enc != 1 or nx <= 0 or ny <= 0 or nz <= 0 or ch <= 0
                or nx * ny * nz > (1 << 31)):
            raise ValueError(path + ": not a float32 Mitsuba .vol (version 3) file")
        n = nx * ny * nz * ch
        raw = np.frombuffer(f.read(4 * n), dtype="<f4")
        if raw.size != n:
            raise ValueError(path + ": truncated voxel data")
    data = raw.reshape(nz * ny * nx, ch).astype(np.float64).sum(1) / ch
    return data.astype(np.float32).reshape(nz, ny, nx), np.array(bb, dtype=np.float32).reshape(2, 3)


def affine_inverse(medium_to_world: np.ndarray) -> np.ndarray:
    """Row-major 3x4 world-to-medium matrix of a 4x4 (or 3x4) affine medium-to-world matrix."""
    m = np.eye(4)
    m[:3, :] = np.asarray(medium_to_world, dtype=np.float64).reshape(-1, 4)[:3]
    return np.linalg.inv(m)[:3, :].astype(np.float32)


def grid_desc(sigma_a: int, sigma_s: int, density: np.ndarray, bounds, scale: float = 1.0, g: float = 0.0,
              world_to_medium: np.ndarray | None = None, max_density: float = 0.0) -> abi.GridMediumDesc:
    """A GridMediumDesc over `density` ((nz, ny, nx) float32, kept alive by the record).
    sigma_a / sigma_s: spectrum indices into SceneDesc::spectra; world_to_medium: row-major 3x4
    (identity when None); bounds: medium-space box of the grid."""
    d = np.ascontiguousarray(density, dtype=np.float32)
    if d.ndim != 3:
        raise ValueError("density must be (nz, ny, nx)")
    r = abi.GridMediumDesc()
    r.sigmaA, r.sigmaS, r.scale, r.g = sigma_a, sigma_s, scale, g
    w = np.eye(4, dtype=np.float32)[:3] if world_to_medium is None else np.asarray(world_to_medium, np.float32)
    for i, v in enumerate(w.reshape(12)):
        r.worldToMedium[i] = float(v)
    b = np.asarray(bounds, dtype=np.float32).reshape(2, 3)
    for i in range(3):
        r.boundsMin[i] = float(b[0, i])
        r.boundsMax[i] = float(b[1, i])
    r.nz, r.ny, r.nx = d.shape
    r.maxDensity = max_density
    r.density = d.ctypes.data
    r._keep = d
    return r


def noise_desc(sigma_a: int, sigma_s: int, bounds, scale: float = 1.0, g: float = 0.0,
               world_to_medium: np.ndarray | None = None, frequency: float = 1.5, octaves: int = 5,
               threshold: float = 0.45, sharpness: float = 4.0, falloff: bool = True,
               offset=(0.0, 0.0, 0.0)) -> abi.GridMediumDesc:
    """A GridMediumDesc of a procedural noise field (pr::NoiseField; the defaults are the reference
    loader's) over the medium-space box `bounds`."""
    r = abi.GridMediumDesc()
    r.sigmaA, r.sigmaS, r.scale, r.g = sigma_a, sigma_s, scale, g
    w = np.eye(4, dtype=np.float32)[:3] if world_to_medium is None else np.asarray(world_to_medium, np.float32)
    for i, v in enumerate(w.reshape(12)):
        r.worldToMedium[i] = float(v)
    b = np.asarray(bounds, dtype=np.float32).reshape(2, 3)
    for i in range(3):
        r.boundsMin[i] = float(b[0, i])
        r.boundsMax[i] = float(b[1, i])
    r.field = abi.GRID_NOISE
    r.noiseOctaves, r.noiseFrequency = octaves, frequency
    r.noiseThreshold, r.noiseSharpness, r.noiseFalloff = threshold, sharpness, 1 if falloff else 0
    r.noiseOffset[:] = [float(v) for v in offset]
    return r


def indexed_desc(sigma_a: int, sigma_s: int, density: np.ndarray, index_origin, index_bounds, scale: float = 1.0,
                 g: float = 0.0, world_to_index: np.ndarray | None = None) -> abi.GridMediumDesc:
    """A GridMediumDesc of an index-space grid (a densified NanoVDB float grid): density
    ((nz, ny, nx) float32, kept alive by the record) holds the voxels at integer index coordinates
    index_origin + (x, y, z); index_bounds: the clip box in index space; world_to_index: row-major
    3x4 (world -> the grid's index space, through the medium's transform)."""
    d = np.ascontiguousarray(density, dtype=np.float32)
    if d.ndim != 3:
        raise ValueError("density must be (nz, ny, nx)")
    r = grid_desc(sigma_a, sigma_s, d, index_bounds, scale=scale, g=g, world_to_medium=world_to_index)
    r.field = abi.GRID_INDEXED
    r.indexOrigin[:] = [int(v) for v in index_origin]
    return r


def grid_array(descs) -> C.Array:
    """A contiguous GridMediumDesc array for SceneExt::gridMedia (keeps the densities alive)."""
    arr = (abi.GridMediumDesc * len(descs))(*descs)
    arr._keep = [getattr(x, "_keep", None) for x in descs]
    return arr
