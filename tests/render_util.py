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


def grid_scene_inputs(rs, s):
    """The GPU-side inputs of a grid scene loaded by the reference: the exported SceneDesc with the
    smoke's sigma_a / sigma_s tables appended (RGB-unbounded spectra, evaluated by the reference
    at the 95 table wavelengths), and a SceneExt carrying the grid as medium mediumCount + 0."""
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
    desc = media.grid_desc(na, na + 1, s.grid["density"], grids[0][1], scale=s.grid["scale"], g=s.grid["g"],
                           world_to_medium=media.affine_inverse(s.grid["matrix"]))
    ext = render.make_ext(grid_media=[desc])
    sd._keep = table
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
