"""Sun and sky on the GPU against the oracle: the reference PathIntegrator lighting an outdoor
scene with its Preetham sun_sky light (a SunLight cone, src/lights/sky.cpp:84-109, plus an
EnvironmentLight over the sky image MakePreethamSky builds, sky.cpp:146-205, light.cpp:217-297),
rendered from the same scene file."""

import numpy as np
import pytest

import render_util as ru
from prgpu import render

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("elevation,azimuth", [(30.0, 40.0), (8.0, -120.0)])
def test_sun_and_sky_agree_with_reference(gpu, oracle, elevation, azimuth):
    """32 x 32, depth 8: per-pixel z of the mean over 16 renders each side, |z| < 4 on >= 99.5% of
    values; the mean luminance agrees within 4 standard errors of the per-render means (sun
    caustics through the glass sphere make the image mean heavy-tailed on both sides)."""
    w = h = 32
    path = ru.outdoor_scene_file(f"sky_{int(elevation)}", width=w, height=h, elevation=elevation, azimuth=azimuth,
                                 sky_resolution=64)
    rs = oracle.RefScene(path)
    sd, ext = ru.sun_sky_inputs(rs, elevation, azimuth, 3.0, 64)
    assert sorted(t for t, _ in rs.infinite_lights()) == [2, 3]
    g = np.stack([render.render_ex(sd, w, h, 256, seed=1000 + k, max_depth=8, ext=ext) / 256 for k in range(16)])
    c = np.stack([rs.render(256, 2000 + k, 8)[0].astype(np.float64) / 256 for k in range(16)])
    z = ru.z_scores(g, c)
    frac = np.mean(np.abs(z) < 4)
    mg, mc = g[..., 1].mean(axis=(1, 2)), c[..., 1].mean(axis=(1, 2))
    se = np.sqrt(mg.var(ddof=1) / len(mg) + mc.var(ddof=1) / len(mc))
    assert frac >= 0.995, f"only {frac:.4f} of values within |z| < 4"
    assert abs(mg.mean() - mc.mean()) < 4 * se, f"mean Y gpu {mg.mean()} cpu {mc.mean()} (se {se})"
