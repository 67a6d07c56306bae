"""Shared helpers for the render parity tests: scene files of the box-and-spheres family, the
reference CPU renders (the oracle) and the per-pixel z statistic of two sets of independent
renders (the pattern of the reference's variance test, tests/test_quality.cpp:146-173: per-pixel
variance from independent seeds, since the film stores no second moments)."""

import os
import tempfile

import numpy as np

from prgpu import scenes

_DIR = os.path.join(tempfile.gettempdir(), "prb_scenes")


def scene_file(name: str, **kw) -> str:
    s = scenes.box_scene(**kw)
    return scenes.write_reference_json(s, os.path.join(_DIR, name + ".prscene.json"))


def grid_scene_file(name: str, **kw):
    """(path, BoxScene) of the heterogeneous-smoke variant (writes the .vol beside the JSON)."""
    s = scenes.grid_box_scene(**kw)
    return scenes.write_reference_json(s, os.path.join(_DIR, name + ".prscene.json")), s


def nvdb_scene_file(name: str, radius: float = 0.8, voxel_size: float = 0.04, **kw):
    """(path, BoxScene) of the smoke room with a NanoVDB fog sphere (written by the oracle with
    NanoVDB's tools) in place of the voxel smoke: the same medium transform, spectra and scale, no
    "bounds" key, so the field's own world box clips."""
    import json

    import ref as oracle_ref

    path, s = grid_scene_file(name + "_src", **kw)
    with open(path) as f:
        doc = json.load(f)
    nvdb = oracle_ref.write_fog_sphere(os.path.join(_DIR, name + ".nvdb"), radius, voxel_size)
    smoke = doc["media"]["smoke"]
    smoke.pop("bounds")
    smoke.update(file=nvdb, grid="density")
    path = os.path.join(_DIR, name + ".prscene.json")
    with open(path, "w") as f:
        json.dump(doc, f)
    return path, s


def densify_index_grid(rs, k: int, voxel_size: float):
    """The grid medium k of a loaded scene as index-space voxels: the field sampled at the voxel
    centres (integer index coordinates, medium point = index x voxel_size) over its world box plus
    one voxel on every side. Returns (density (nz, ny, nx), index origin, index-space bounds)."""
    b = rs.grid_media()[k][1].astype(np.float64)
    lo = np.floor(b[0] / voxel_size).astype(int) - 1
    hi = np.ceil(b[1] / voxel_size).astype(int) + 1
    zs, ys, xs = [np.arange(lo[a], hi[a] + 1) for a in (2, 1, 0)]
    z, y, x = np.meshgrid(zs, ys, xs, indexing="ij")
    pts = (np.stack([x, y, z], -1).reshape(-1, 3) * voxel_size).astype(np.float32)
    dens = rs.grid_density(k, pts).reshape(len(zs), len(ys), len(xs))
    return dens, lo, (b / voxel_size).astype(np.float32)


def grid_scene_inputs(rs, s, noise=None, indexed_voxel=None):
    """The GPU-side inputs of a grid scene loaded by the reference: the exported SceneDesc with the
    smoke's sigma_a / sigma_s tables appended (RGB-unbounded spectra, evaluated by the reference
    at the 95 table wavelengths), and a SceneExt carrying the grid as medium mediumCount + 0.
    noise: media.noise_desc keyword arguments, for the scene's noise-field variant; indexed_voxel:
    the voxel size of the NanoVDB variant's grid, handed over densified in its index space."""
    import ctypes as C

    import ref as oracle_ref
    from prgpu import abi, media, render, spectra

    base = abi.SceneDesc.from_address(rs.export())
    sd = abi.SceneDesc()
    C.memmove(C.addressof(sd), C.addressof(base), C.sizeof(sd))
    old = np.ctypeslib.as_array((C.c_float * (95 * base.spectrumCount)).from_address(base.spectra))
    lam = spectra.LAMBDA.astype(np.float32)
    rows = []
    for key in ("sigma_a", "sigma_s"):
        out = np.zeros(95, dtype=np.float32)
        rgb = s.grid[key]
        assert oracle_ref.ref_lib().prref_spectrum(1, rgb[0], rgb[1], rgb[2], None, 95, oracle_ref._p(lam),
                                                   oracle_ref._p(out)) == 0
        rows.append(out)
    table = np.ascontiguousarray(np.concatenate([old.reshape(-1, 95)] + [r[None] for r in rows]), dtype=np.float32)
    sd.spectra = table.ctypes.data
    sd.spectrumCount = table.shape[0]
    grids = rs.grid_media()
    assert [g[0] for g in grids] == ["smoke"], grids
    na = base.spectrumCount
    if indexed_voxel is not None:
        dens, org, ib = densify_index_grid(rs, 0, indexed_voxel)
        w2i = media.affine_inverse(s.grid["matrix"]).astype(np.float64) / indexed_voxel
        desc = media.indexed_desc(na, na + 1, dens, org, ib, scale=s.grid["scale"], g=s.grid["g"], world_to_index=w2i)
    elif noise is not None:
        desc = media.noise_desc(na, na + 1, grids[0][1], scale=s.grid["scale"], g=s.grid["g"],
                                world_to_medium=media.affine_inverse(s.grid["matrix"]), **noise)
    else:
        desc = media.grid_desc(na, na + 1, s.grid["density"], grids[0][1], scale=s.grid["scale"], g=s.grid["g"],
                               world_to_medium=media.affine_inverse(s.grid["matrix"]))
    ext = render.make_ext(grid_media=[desc])
    sd._keep = table
    return sd, ext


def outdoor_scene_file(name: str, **kw) -> str:
    import json

    from prgpu import scenes as sc

    path = os.path.join(_DIR, name + ".prscene.json")
    os.makedirs(_DIR, exist_ok=True)
    with open(path, "w") as f:
        json.dump(sc.outdoor_scene_json(**kw), f)
    return path


def sun_sky_inputs(rs, elevation, azimuth, turbidity, sky_resolution, intensity=0.03):
    """The GPU-side inputs of a sun_sky scene loaded by the reference: the exported SceneDesc with
    D65 and the sun's radiance appended to its spectra, and a SceneExt carrying the Preetham sky
    (uplifted to sigmoid-polynomial texels by the reference's table) and the sun, with the pmfs the
    reference's light sampler gives them (scene_loader.cpp:977-996)."""
    import ctypes as C
    import math

    import ref as oracle_ref
    from prgpu import abi, render, scenes, spectra

    base = abi.SceneDesc.from_address(rs.export())
    sd = abi.SceneDesc()
    C.memmove(C.addressof(sd), C.addressof(base), C.sizeof(sd))
    old = np.ctypeslib.as_array((C.c_float * (95 * base.spectrumCount)).from_address(base.spectra)).reshape(-1, 95)
    lam = spectra.LAMBDA.astype(np.float32)
    d65 = np.zeros(95, np.float32)
    assert oracle_ref.ref_lib().prref_spectrum(2, 1.0, 1.0, 1.0, None, 95, oracle_ref._p(lam), oracle_ref._p(d65)) == 0
    sun_dir = scenes.sun_direction(elevation, azimuth)
    radius = 0.2665
    sun_spec = oracle_ref.sun_radiance(sun_dir, turbidity, radius, lam)
    table = np.ascontiguousarray(np.concatenate([old, d65[None], sun_spec[None]]), np.float32)
    sd.spectra = table.ctypes.data
    sd.spectrumCount = table.shape[0]
    pmfs = dict(rs.infinite_lights())
    sky = oracle_ref.preetham_sky(sun_dir, turbidity, 0.3, sky_resolution, sky_resolution // 2)
    texels = np.ascontiguousarray(oracle_ref.rgb_uplift(sky.reshape(-1, 3)), np.float32)
    env = abi.EnvMapDesc()
    env.width, env.height = sky_resolution, sky_resolution // 2
    env.texels = texels.ctypes.data
    env.illuminant = base.spectrumCount
    env.scale = intensity
    env.rotationDeg = 0.0
    env.pmf = pmfs.get(2, 0.0)
    sun = abi.SunDesc()
    for i in range(3):
        sun.direction[i] = float(sun_dir[i])
    sun.cosThetaMax = math.cos(math.radians(radius))
    sun.spectrum = base.spectrumCount + 1
    sun.scale = intensity
    sun.pmf = pmfs.get(3, 0.0)
    ext = render.make_ext()
    ext.envMap = C.addressof(env)
    ext.sun = C.addressof(sun)
    ext._keep += [env, sun, texels]
    sd._keep = table
    return sd, ext


def large_scene_inputs(rs, path, turbidity=3.0, sky_resolution=64):
    """The GPU-side inputs of the large outdoor scene loaded by the reference: the sun and sky of
    sun_sky_inputs plus the cloud's sigma_a / sigma_s tables appended to the spectra and the cloud
    grid (read back from the .vol the scene names) as grid medium 0."""
    import ctypes as C

    import ref as oracle_ref
    from prgpu import abi, hostscene, media, spectra

    sd, ext = sun_sky_inputs(rs, hostscene.SUN_ELEVATION, hostscene.SUN_AZIMUTH, turbidity, sky_resolution)
    old = np.ctypeslib.as_array((C.c_float * (95 * sd.spectrumCount)).from_address(sd.spectra)).reshape(-1, 95)
    lam = spectra.LAMBDA.astype(np.float32)
    rows = []
    for v in (0.05, 0.95):
        out = np.zeros(95, dtype=np.float32)
        assert oracle_ref.ref_lib().prref_spectrum(1, v, v, v, None, 95, oracle_ref._p(lam), oracle_ref._p(out)) == 0
        rows.append(out)
    table = np.ascontiguousarray(np.concatenate([old, np.stack(rows)]), np.float32)
    na = sd.spectrumCount
    sd.spectra = table.ctypes.data
    sd.spectrumCount = table.shape[0]
    sd._keep = (sd._keep, table)
    grids = rs.grid_media()
    assert [g[0] for g in grids] == ["cloud"], grids
    import json

    with open(path) as f:
        doc = json.load(f)
    density, _ = media.read_vol(doc["media"]["cloud"]["file"])
    desc = media.grid_desc(na, na + 1, density, grids[0][1], scale=1.0, g=0.8,
                           world_to_medium=media.affine_inverse(hostscene.CLOUD_TO_WORLD))
    from prgpu.media import grid_array

    arr = grid_array([desc])
    ext.gridMediumCount = 1
    ext.gridMedia = C.cast(arr, C.c_void_p)
    ext._keep += [desc, arr, density]
    return sd, ext


def luminance_y(img: np.ndarray) -> np.ndarray:
    return img[..., 1]


def z_scores(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """a, b: (seeds, h, w, 3) per-seed mean images. Returns the per-value z statistic."""
    ma, mb = a.mean(0), b.mean(0)
    va = a.var(0, ddof=1) / a.shape[0]
    vb = b.var(0, ddof=1) / b.shape[0]
    den = np.sqrt(va + vb)
    z = np.where(den > 0, (ma - mb) / np.where(den > 0, den, 1), np.where(ma == mb, 0.0, np.inf))
    return z
