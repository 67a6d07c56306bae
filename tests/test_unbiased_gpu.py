"""The unbiasedness gate on the plain path tracer: the GPU image against a 65,536-spp render of the
reference PathIntegrator (16 seeds x 4096 spp, src/integrators/path.cpp:113-238) of the same
box-and-spheres scene (box filter, depth 8). Per-pixel variances come from independent seeds on
both sides, as tests/test_quality.cpp:146-173 of the reference estimates them; the pass bar is
|z| < 4 on >= 99.9% of values (all three XYZ channels of every pixel) and mean luminance within
0.5%."""

import os

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


GATE_FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "gate_c0.npz")


def test_c0_image_is_unbiased_against_65536_spp_reference_fixture(gpu, oracle):
    """The gate at the configuration's own size: the box-and-spheres scene at 256 x 256, depth 8, as
    the reference host hands it to the module (loaded by the reference's loader and flattened by its
    exporter into the v4 SceneDesc), 16 GPU seeds x 4096 spp, against the reference
    PathIntegrator's 16 seeds x 4096 spp (65,536 spp) of the same scene, precomputed into
    tests/golden/gate_c0.npz by tests/golden/make_gate.py (per-pixel mean and across-seed variance).
    |z| < 4 on >= 99.9% of the 196,608 values and mean luminance within 0.5%. (The library's own
    host builder, which the benchmark renders for throughput, uplifts RGB albedos with a fit under a
    6504 K blackbody in place of the reference's D65 table: saturated wall colours move by up to 4 %
    in Z, so that scene is not this gate's subject.)"""
    fx = np.load(GATE_FIXTURE)
    n, side, depth = int(fx["seeds"]), int(fx["side"]), int(fx["depth"])
    assert (side, depth, int(fx["spp"])) == (256, 8, SPP)
    rs = oracle.RefScene(ru.scene_file("gate_c0", seed=0, width=side, height=side))
    desc = rs.export()
    g = np.stack([render.render_ex(desc, side, side, SPP, seed=5000 + k, max_depth=depth) / SPP for k in range(SEEDS)])
    mg, vg = g.mean(0), g.var(0, ddof=1) / SEEDS
    mc, vc = fx["mean"].astype(np.float64), fx["var"].astype(np.float64) / n
    den = np.sqrt(vg + vc)
    z = np.where(den > 0, (mg - mc) / np.where(den > 0, den, 1), np.where(mg == mc, 0.0, np.inf))
    frac = np.mean(np.abs(z) < 4)
    yg, yc = mg[..., 1].mean(), float(fx["mean_y"])
    print(f"C0 gate: frac {frac:.5f} (max |z| {np.abs(z).max():.2f}), mean Y gpu {yg:.6f} cpu {yc:.6f} "
          f"({yg / yc - 1:+.4%})")
    assert frac >= 0.999, f"only {frac:.5f} of values within |z| < 4 (max |z| {np.abs(z).max():.2f})"
    assert abs(yg / yc - 1) < 0.005, f"mean Y gpu {yg} cpu {yc} ({yg / yc - 1:+.4%})"
