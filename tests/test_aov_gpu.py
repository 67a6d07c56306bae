"""Denoiser guide buffers on the GPU against pr::RenderAOV (src/integrators/aov.cpp:83-196): albedo,
shading normal, depth and position of the first visible surface, with and without following
specular chains, on the box scene (Lambertian, gold and BK7 spheres) and its fog variant (a chain
through glass into a scattering medium takes the medium's albedo). Both sides jitter their
samples independently, so the comparisons are statistical: per-pixel differences below a
tolerance on nearly every pixel and equal image means."""

import ctypes as C

import numpy as np
import pytest

import render_util as ru
from prgpu import abi, render, spectra

pytestmark = pytest.mark.gpu


def _inputs(rs):
    """The exported scene with D65 appended to its spectra, and the reference's colour matrices."""
    import ref as oracle_ref

    base = abi.SceneDesc.from_address(rs.export())
    sd = abi.SceneDesc()
    C.memmove(C.addressof(sd), C.addressof(base), C.sizeof(sd))
    old = np.ctypeslib.as_array((C.c_float * (95 * base.spectrumCount)).from_address(base.spectra)).reshape(-1, 95)
    lam = spectra.LAMBDA.astype(np.float32)
    d65 = np.zeros(95, np.float32)
    assert oracle_ref.ref_lib().prref_spectrum(2, 1.0, 1.0, 1.0, None, 95, oracle_ref._p(lam), oracle_ref._p(d65)) == 0
    table = np.ascontiguousarray(np.concatenate([old, d65[None]]), np.float32)
    sd.spectra = table.ctypes.data
    sd.spectrumCount = table.shape[0]
    sd._keep = table
    adapt, to_rgb = np.zeros(9, np.float32), np.zeros(9, np.float32)
    oracle_ref.ref_lib().prref_aov_matrices(oracle_ref._p(adapt), oracle_ref._p(to_rgb))
    return sd, base.spectrumCount, adapt, to_rgb


@pytest.mark.parametrize("medium", [False, True])
@pytest.mark.parametrize("through", [False, True])
def test_aov_buffers_agree_with_reference(gpu, oracle, medium, through):
    w = h = 48
    rs = oracle.RefScene(ru.scene_file(f"aov_{int(medium)}", seed=1, width=w, height=h, medium=medium, subdiv=2))
    sd, d65, adapt, to_rgb = _inputs(rs)

    def ours(kind, spp):
        return render.render_aov(sd, w, h, kind, spp, seed=5, through_specular=through, d65_spectrum=d65,
                                 white_adaptation=adapt, xyz_to_rgb=to_rgb)

    # Depth: the nearest hit over 64 jittered samples per pixel; silhouettes aside, the same.
    g, c = ours(render.AOV_DEPTH, 64)[..., 0], rs.render_aov(render.AOV_DEPTH, 64, 9, through)[..., 0]
    rel = np.abs(g - c) / np.maximum(c, 1e-6)
    assert np.mean(rel < 0.02) >= 0.95, f"depth: {np.mean(rel < 0.02):.3f} of pixels within 2 %"
    # Position: the mean hit point.
    g, c = ours(render.AOV_POSITION, 64), rs.render_aov(render.AOV_POSITION, 64, 9, through)
    d = np.linalg.norm(g - c, axis=-1)
    assert np.mean(d < 0.03) >= 0.95, f"position: {np.mean(d < 0.03):.3f} of pixels within 0.03"
    # Normal: normalised sum of shading normals.
    g, c = ours(render.AOV_NORMAL, 64), rs.render_aov(render.AOV_NORMAL, 64, 9, through)
    dots = np.sum(g * c, axis=-1)
    ok = (np.linalg.norm(c, axis=-1) > 0) & (np.linalg.norm(g, axis=-1) > 0)
    assert np.mean(dots[ok] > 0.98) >= 0.95, f"normal: {np.mean(dots[ok] > 0.98):.3f} of pixels within 11 deg"
    # Albedo: a Monte Carlo estimate on both sides (8 BSDF samples per camera sample).
    g, c = ours(render.AOV_ALBEDO, 256), rs.render_aov(render.AOV_ALBEDO, 256, 9, through)
    diff = np.abs(g - c).max(axis=-1)
    print(f"aov medium={medium} through={through}: albedo mean gpu {g.mean(axis=(0, 1))} ref {c.mean(axis=(0, 1))}, "
          f"pixels within 0.05: {np.mean(diff < 0.05):.3f}")
    assert np.mean(diff < 0.05) >= 0.95, f"albedo: {np.mean(diff < 0.05):.3f} of pixels within 0.05"
    np.testing.assert_allclose(g.mean(axis=(0, 1)), c.mean(axis=(0, 1)), rtol=0.02, atol=0.002)
