"""GPU path tracer (prgpu_render / prgpu_render_ex) against the oracle: the reference's own
PathIntegrator (src/integrators/path.cpp:113-238) rendering the same scene, loaded by the
reference loader and handed to this module exactly as the reference host would (the exported v4
SceneDesc, src/integrators/gpu_path.cpp:284-456)."""

import numpy as np
import pytest

import render_util as ru
from prgpu import render

pytestmark = pytest.mark.gpu


def _gpu_seeds(desc, w, h, spp, seeds, max_depth):
    return np.stack([render.render_ex(desc, w, h, spp, seed=1000 + k, max_depth=max_depth) / spp for k in range(seeds)])


def _cpu_seeds(rs, spp, seeds, max_depth):
    return np.stack([rs.render(spp, 2000 + k, max_depth)[0].astype(np.float64) / spp for k in range(seeds)])


@pytest.mark.parametrize("medium", [False, True])
def test_box_scene_agrees_with_reference_path_tracer(gpu, oracle, medium):
    """Config-0 family at 48x48: per-pixel z of the mean over 16 independent renders each side;
    |z| < 4 on >= 99.5% of values, mean luminance within 1.5% (the statistical error of the
    mean luminance here is about 0.3%)."""
    w = h = 48
    path = ru.scene_file(f"box_m{int(medium)}", seed=0, width=w, height=h, medium=medium)
    rs = oracle.RefScene(path)
    desc = rs.export()
    g = _gpu_seeds(desc, w, h, 256, 16, 8)
    c = _cpu_seeds(rs, 256, 16, 8)
    z = ru.z_scores(g, c)
    frac = np.mean(np.abs(z) < 4)
    yg, yc = g[..., 1].mean(), c[..., 1].mean()
    assert frac >= 0.995, f"only {frac:.4f} of values within |z| < 4"
    assert abs(yg / yc - 1) < 0.015, f"mean Y gpu {yg} cpu {yc}"


def test_unlimited_depth_russian_roulette(gpu, oracle):
    w = h = 32
    path = ru.scene_file("box_rr", seed=3, width=w, height=h)
    rs = oracle.RefScene(path)
    desc = rs.export()
    g = _gpu_seeds(desc, w, h, 256, 12, 0)
    c = _cpu_seeds(rs, 256, 12, 0)
    assert abs(g[..., 1].mean() / c[..., 1].mean() - 1) < 0.02
    assert np.mean(np.abs(ru.z_scores(g, c)) < 4) >= 0.99


def test_fp64_film_resume_is_bit_identical(gpu, oracle):
    """Sample streams are indexed by sample number and each sample is added to the FP64 film in
    order, so 3 + 5 samples in two calls give exactly the bits of 8 samples in one."""
    w, h = 40, 30
    rs = oracle.RefScene(ru.scene_file("box_resume", seed=1, width=w, height=h, medium=True))
    desc = rs.export()
    one = render.render_ex(desc, w, h, 8, first_sample=0, seed=7, max_depth=8)
    two = render.render_ex(desc, w, h, 3, first_sample=0, seed=7, max_depth=8)
    two = render.render_ex(desc, w, h, 5, first_sample=3, seed=7, max_depth=8, out=two)
    assert one.any()
    np.testing.assert_array_equal(one.view(np.int64), two.view(np.int64))
    # Different chunking of the wavefront (paths in flight) does not change a bit either.
    small = render.render_ex(desc, w, h, 8, seed=7, max_depth=8, ext=render.make_ext(wavefront_paths=1024))
    np.testing.assert_array_equal(one.view(np.int64), small.view(np.int64))


def test_v4_entry_point_adds_float_sums(gpu, oracle):
    w, h = 32, 24
    rs = oracle.RefScene(ru.scene_file("box_v4", seed=2, width=w, height=h))
    desc = rs.export()
    ref = render.render_ex(desc, w, h, 4, seed=3, max_depth=8)
    out = np.full((h, w, 3), 0.5, dtype=np.float32)
    render.render_v4(desc, w, h, 4, seed=3, max_depth=8, out=out)
    np.testing.assert_allclose(out - 0.5, ref, rtol=1e-5, atol=1e-5)


def test_stats_and_determinism(gpu, oracle):
    w, h = 32, 32
    rs = oracle.RefScene(ru.scene_file("box_stats", seed=4, width=w, height=h))
    desc = rs.export()
    a, st = render.render_ex(desc, w, h, 4, seed=9, max_depth=8, stats=True)
    b = render.render_ex(desc, w, h, 4, seed=9, max_depth=8)
    np.testing.assert_array_equal(a, b)
    assert st.pathSamples == w * h * 4
    assert st.closestRays >= st.pathSamples and st.shadowRays > 0 and st.deviceMs > 0
