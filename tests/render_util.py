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
