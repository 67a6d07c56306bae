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


def _write_pfm(path, img):
    """Little-endian RGB PFM; file rows run bottom to top (the reference's ReadPFM flips them)."""
    h, w, _ = img.shape
    with open(path, "wb") as f:
        f.write(f"PF\n{w} {h}\n-1.0\n".encode())
        f.write(np.ascontiguousarray(img[::-1], dtype="<f4").tobytes())


def test_image_environment_map_agrees_with_reference(gpu, oracle, tmp_path):
    """An image environment (a warm bright spot and a blue gradient, 48 x 24, turned 70 degrees
    about +y) lighting the outdoor scene: same z-statistics as above."""
    import ctypes as C

    import ref as oracle_ref
    from prgpu import abi, spectra

    hh, ww = 24, 48
    v, u = np.meshgrid((np.arange(hh) + 0.5) / hh, (np.arange(ww) + 0.5) / ww, indexing="ij")
    img = np.zeros((hh, ww, 3), np.float32)
    img[..., 2] = 0.3 + 0.5 * (1 - v)
    img[..., 1] = 0.2 + 0.3 * (1 - v)
    img[..., 0] = 0.1
    spot = np.exp(-(((u - 0.3) / 0.05) ** 2 + ((v - 0.3) / 0.08) ** 2))
    img += (spot * 20.0)[..., None] * np.array([1.0, 0.8, 0.5], np.float32)
    pfm = str(tmp_path / "env.pfm")
    _write_pfm(pfm, img)
    w = h = 32
    path = ru.outdoor_scene_file("envmap", width=w, height=h, env_file=pfm, env_rotation=70.0)
    rs = oracle.RefScene(path)
    base = abi.SceneDesc.from_address(rs.export())
    sd = abi.SceneDesc()
    C.memmove(C.addressof(sd), C.addressof(base), C.sizeof(sd))
    old = np.ctypeslib.as_array((C.c_float * (95 * base.spectrumCount)).from_address(base.spectra)).reshape(-1, 95)
    lam = spectra.LAMBDA.astype(np.float32)
    d65 = np.zeros(95, np.float32)
    assert oracle_ref.ref_lib().prref_spectrum(2, 1.0, 1.0, 1.0, None, 95, oracle_ref._p(lam), oracle_ref._p(d65)) == 0
    table = np.ascontiguousarray(np.concatenate([old, d65[None]]), np.float32)
    sd.spectra, sd.spectrumCount = table.ctypes.data, table.shape[0]
    texels = np.ascontiguousarray(oracle_ref.rgb_uplift(img.reshape(-1, 3)), np.float32)
    env = abi.EnvMapDesc()
    env.width, env.height, env.texels = ww, hh, texels.ctypes.data
    env.illuminant, env.scale, env.rotationDeg = base.spectrumCount, 1.0, 70.0
    env.pmf = dict(rs.infinite_lights())[2]
    ext = render.make_ext()
    ext.envMap = C.addressof(env)
    g = np.stack([render.render_ex(sd, w, h, 256, seed=1000 + k, max_depth=8, ext=ext) / 256 for k in range(16)])
    c = np.stack([rs.render(256, 2000 + k, 8)[0].astype(np.float64) / 256 for k in range(16)])
    z = ru.z_scores(g, c)
    frac = np.mean(np.abs(z) < 4)
    mg, mc = g[..., 1].mean(axis=(1, 2)), c[..., 1].mean(axis=(1, 2))
    se = np.sqrt(mg.var(ddof=1) / len(mg) + mc.var(ddof=1) / len(mc))
    assert frac >= 0.995, f"only {frac:.4f} of values within |z| < 4"
    assert abs(mg.mean() - mc.mean()) < 4 * se, f"mean Y gpu {mg.mean()} cpu {mc.mean()} (se {se})"
