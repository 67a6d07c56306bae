"""The host library's daylight (prhost_preetham_sky, prhost_sun_radiance) against the reference's
own pr::MakePreethamSky and pr::MakeSunRadiance (src/lights/sky.cpp:146-233) run by the oracle, and
its RGB -> sigmoid-polynomial texel fit against the reference's uplift of the same colours."""

import numpy as np
import pytest

from prgpu import scenes, spectra


@pytest.mark.parametrize("elev,az,turb", [(20.0, 34.4, 3.0), (45.0, 0.0, 2.0), (5.0, 120.0, 6.5), (-3.0, 10.0, 3.0)])
def test_preetham_sky_matches_reference(oracle, elev, az, turb):
    d = scenes.sun_direction(elev, az).astype(np.float32)
    w, h = 128, 64
    mine = spectra.preetham_sky(d, turb, 0.3, w, h)
    ref = oracle.preetham_sky(d, turb, 0.3, w, h).reshape(h, w, 3)
    scale = max(float(np.abs(ref).max()), 1e-30)
    np.testing.assert_allclose(mine, ref, rtol=1e-5, atol=1e-6 * scale)
    if elev > 0:
        assert ref.max() > 0


@pytest.mark.parametrize("elev,turb,radius", [(20.0, 3.0, 0.2665), (60.0, 2.0, 0.5), (0.5, 8.0, 0.2665)])
def test_sun_radiance_matches_reference(oracle, elev, turb, radius):
    d = scenes.sun_direction(elev, 10.0).astype(np.float32)
    lam = np.ascontiguousarray(np.concatenate([spectra.LAMBDA, [362.5, 401.25, 777.7]]), np.float32)
    mine = spectra.sun_radiance(d, turb, radius, lam)
    ref = oracle.sun_radiance(d, turb, radius, lam)
    np.testing.assert_allclose(mine, ref, rtol=1e-5)


def test_texel_fit_reproduces_the_reference_uplift(oracle):
    """Sky colours: the fitted texel spectra under the reference's D65 and the reference's own uplift
    (its 64^3 table of fits) give the same XYZ to within 1 %."""
    rng = np.random.default_rng(3)
    d = scenes.sun_direction(20.0, 34.4).astype(np.float32)
    sky = spectra.preetham_sky(d, 3.0, 0.3, 64, 32).reshape(-1, 3)
    rgb = np.concatenate([sky[sky.max(1) > 0][::7], rng.uniform(0.02, 1.0, (64, 3)).astype(np.float32)])
    lam = spectra.LAMBDA.astype(np.float32)
    d65 = np.zeros(95, np.float32)
    lib = oracle.ref_lib()
    assert lib.prref_spectrum(2, 1.0, 1.0, 1.0, None, 95, oracle._p(lam), oracle._p(d65)) == 0
    mine = spectra.rgb_to_sigmoid(rgb, d65)
    ref = oracle.rgb_uplift(rgb)
    np.testing.assert_allclose(mine[:, 3], ref[:, 3], rtol=1e-6)

    def spec(t):
        x = (t[:, 0:1] * lam + t[:, 1:2]) * lam + t[:, 2:3]
        return t[:, 3:4] * (0.5 + x / (2 * np.sqrt(1 + x * x))) * d65

    cmf = spectra.cie_xyz(spectra.LAMBDA)
    xm, xr = spec(mine.astype(np.float64)) @ cmf.T, spec(ref.astype(np.float64)) @ cmf.T
    rel = np.abs(xm - xr).max(1) / np.abs(xr).max(1)
    assert np.percentile(rel, 99) < 0.01 and rel.max() < 0.03, (np.percentile(rel, 99), rel.max())
