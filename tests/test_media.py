"""Host side of grid media (no GPU): .vol files as pr::VoxelGridField::LoadVol reads them
(src/media/medium.cpp:130-166), the GridMediumDesc record, and the reference loader reading the
files this package writes."""

import ctypes as C
import struct

import numpy as np
import pytest

from prgpu import abi, media, render, scenes


def test_vol_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    d = rng.uniform(0, 2, (5, 6, 7)).astype(np.float32)
    p = media.write_vol(str(tmp_path / "a.vol"), d, [[-1, -2, -3], [1, 2, 3]])
    r, b = media.read_vol(p)
    assert r.shape == (5, 6, 7) and np.array_equal(r, d)
    assert np.array_equal(b, np.array([[-1, -2, -3], [1, 2, 3]], np.float32))


def test_vol_channels_are_averaged(tmp_path):
    p = tmp_path / "c.vol"
    vox = np.array([[1, 3], [2, 6], [0, 0], [5, 5]], np.float32)  # 4 voxels x 2 channels
    with open(p, "wb") as f:
        f.write(struct.pack("<3sBiiiii6f", b"VOL", 3, 1, 2, 2, 1, 2, 0, 0, 0, 1, 1, 1))
        f.write(vox.tobytes())
    r, _ = media.read_vol(str(p))
    assert np.array_equal(r.ravel(), np.array([2, 4, 0, 5], np.float32))


@pytest.mark.parametrize("mutate", ["magic", "version", "encoding", "dims", "truncated"])
def test_vol_rejects_what_the_reference_rejects(tmp_path, mutate):
    head = dict(magic=b"VOL", version=3, enc=1, nx=2, ny=2, nz=2)
    if mutate == "magic":
        head["magic"] = b"VOX"
    elif mutate == "version":
        head["version"] = 2
    elif mutate == "encoding":
        head["enc"] = 3
    elif mutate == "dims":
        head["ny"] = 0
    p = tmp_path / "bad.vol"
    n = 8 if mutate != "truncated" else 5
    with open(p, "wb") as f:
        f.write(struct.pack("<3sBiiiii6f", head["magic"], head["version"], head["enc"], head["nx"], head["ny"],
                            head["nz"], 1, 0, 0, 0, 1, 1, 1))
        f.write(np.zeros(n, np.float32).tobytes())
    with pytest.raises(ValueError):
        media.read_vol(str(p))


def test_affine_inverse():
    m = np.array([[0, 0, 2, 1], [0, 3, 0, 2], [-1, 0, 0, 3], [0, 0, 0, 1]], np.float64)
    w = media.affine_inverse(m)
    p = np.array([0.3, -0.2, 0.7, 1.0])
    q = m @ p
    assert np.allclose(w @ q, p[:3], atol=1e-6)


def test_grid_desc_layout_and_ext():
    d = np.arange(24, dtype=np.float32).reshape(2, 3, 4)
    g = media.grid_desc(3, 4, d, [[0, 0, 0], [1, 2, 3]], scale=2.0, g=0.3)
    assert (g.nx, g.ny, g.nz) == (4, 3, 2) and g.sigmaA == 3 and g.sigmaS == 4
    assert list(g.worldToMedium) == [1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0]
    assert g.density == d.ctypes.data
    e = render.make_ext(grid_media=[g, g])
    assert e.gridMediumCount == 2 and e.structSize == C.sizeof(abi.SceneExt) == 144
    arr = (abi.GridMediumDesc * 2).from_address(e.gridMedia)
    assert arr[1].nx == 4 and arr[1].density == d.ctypes.data
    assert abi.GridMediumDesc.density.offset == 104 and abi.SceneExt.gridMedia.offset == 40


def test_reference_loader_reads_the_written_grid(oracle, tmp_path):
    """The oracle's exporter numbers the grid after the homogeneous media and reports the bounds
    the loader fitted; the camera sits in the smoke."""
    s = scenes.grid_box_scene(seed=0, width=8, height=8)
    path = scenes.write_reference_json(s, str(tmp_path / "smoke.prscene.json"))
    rs = oracle.RefScene(path)
    desc = abi.SceneDesc.from_address(rs.export())
    grids = rs.grid_media()
    assert [g[0] for g in grids] == ["smoke"]
    assert np.array_equal(grids[0][1], s.grid["bounds"])
    assert desc.cameraMedium == desc.mediumCount + 0


def _trilinear_index(dens, org, p):
    """Trilinear between voxel centres at integer index coordinates org + (x, y, z), 0 beyond the
    array, clamped at 0 (the index-space grid the device samples)."""
    q = p - org
    f = np.floor(q)
    i0 = f.astype(int)
    d = q - f
    nz, ny, nx = dens.shape

    def v(dx, dy, dz):
        x, y, z = i0[:, 0] + dx, i0[:, 1] + dy, i0[:, 2] + dz
        ok = (x >= 0) & (y >= 0) & (z >= 0) & (x < nx) & (y < ny) & (z < nz)
        out = np.zeros(len(p))
        out[ok] = dens[z[ok], y[ok], x[ok]]
        return out

    lx = lambda a, b: (1 - d[:, 0]) * a + d[:, 0] * b
    c00, c10 = lx(v(0, 0, 0), v(1, 0, 0)), lx(v(0, 1, 0), v(1, 1, 0))
    c01, c11 = lx(v(0, 0, 1), v(1, 0, 1)), lx(v(0, 1, 1), v(1, 1, 1))
    ly = lambda a, b: (1 - d[:, 1]) * a + d[:, 1] * b
    return np.maximum(0.0, (1 - d[:, 2]) * ly(c00, c10) + d[:, 2] * ly(c01, c11))


def test_nanovdb_fog_sphere_and_its_index_space_voxels(oracle):
    """A NanoVDB fog sphere written with NanoVDB's tools and loaded by the reference (as its
    tests/test_media.cpp:134-148 does): density 1 at the centre (2 %), 0 outside; and the grid
    densified at its voxel centres (the form the device takes) reproduces the reference field's
    trilinear lookups at random points to 1e-5."""
    import render_util as ru

    vs = 0.05
    path, s = ru.nvdb_scene_file("nvdb_pin", radius=1.0, voxel_size=vs, seed=0, width=8, height=8)
    rs = oracle.RefScene(path)
    (name, b), = rs.grid_media()
    assert name == "smoke" and np.all(b[0] <= -0.9) and np.all(b[1] >= 0.9)
    d0, d1 = rs.grid_density(0, np.array([[0, 0, 0], [1.5, 0, 0]], np.float32))
    assert abs(d0 - 1.0) <= 0.02 and d1 == 0.0
    dens, org, ib = ru.densify_index_grid(rs, 0, vs)
    assert dens.max() <= 1.0 + 1e-6 and dens.min() >= 0.0
    rng = np.random.default_rng(7)
    p = rng.uniform(b[0] * 0.98, b[1] * 0.98, size=(20000, 3)).astype(np.float32)
    want = rs.grid_density(0, p)
    got = _trilinear_index(dens, org, p.astype(np.float64) / vs)
    assert np.abs(got - want).max() <= 1e-5, np.abs(got - want).max()
