"""The unbiasedness gate on the plain path tracer: the GPU image against a 65,536-spp render of the
reference PathIntegrator (16 seeds x 4096 spp, src/integrators/path.cpp:113-238) of the same
box-and-spheres scene (box filter, depth 8). Per-pixel variances come from independent seeds on
both sides, as tests/test_quality.cpp:146-173 of the reference estimates them; the pass bar is
|z| < 4 on >= 99.9% of values (all three XYZ channels of every pixel) and mean luminance within
0.5%."""

import numpy as np
import pytest

import render_util as ru
from prgpu import render

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

SEEDS = 16
SPP = 4096


@pytest.mark.parametrize("medium", [False, True])
def test_plain_path_tracer_is_unbiased_against_65536_spp_reference(gpu, oracle, medium):
    w = h = 32
    rs = oracle.RefScene(ru.scene_file(f"gate_m{int(medium)}", seed=0, width=w, height=h, medium=medium))
    oracle.set_threads(0)
    desc = rs.export()
    g = np.stack([render.render_ex(desc, w, h, SPP, seed=5000 + k, max_depth=8) / SPP for k in range(SEEDS)])
    c = np.stack([rs.render(SPP, 9000 + k, 8)[0].astype(np.float64) / SPP for k in range(SEEDS)])
    z = ru.z_scores(g, c)
    frac = np.mean(np.abs(z) < 4)
    yg, yc = g[..., 1].mean(), c[..., 1].mean()
    assert frac >= 0.999, f"only {frac:.5f} of values within |z| < 4 (max |z| {np.abs(z).max():.2f})"
    assert abs(yg / yc - 1) < 0.005, f"mean Y gpu {yg} cpu {yc} ({yg / yc - 1:+.4%})"
