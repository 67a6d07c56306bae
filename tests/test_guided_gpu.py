"""Path guiding in the renderer: diffuse vertices sample the one-sample mixture c q + (1 - c) p_bsdf
of the guide network (tensor-core inference per bounce) and the BSDF, with both pdfs from the same
decoded parameters, so the image must stay unbiased -- for fixed weights and while the network
trains online between wavefront chunks -- and a trained guide must lower the error where light
arrives through a narrow slit."""

import numpy as np
import pytest

import guide_ref as G
import render_util as ru
from prgpu import guide, hostscene, render, scenes

pytestmark = pytest.mark.gpu


def _weights(seed):
    """Random weights with non-trivial biases: peaked, badly placed lobes stress unbiasedness."""
    p = G.init_params(seed).astype(np.float64)
    rng = np.random.default_rng(seed + 1)
    W = G.split(p)
    W[0][:, G.CONST_IN] = rng.normal(0, 0.5, W[0].shape[0])
    for l in range(1, 5):
        W[l][:, G.CONST_HID] = rng.normal(0, 0.5, W[l].shape[0])
    for l in range(4):
        W[l][G.CONST_HID, :] = 0
    W[4][41:, :] = 0
    W[4][40, G.CONST_HID] = 1.5  # select the guide often
    return p.astype(np.float32)


def _cpu_seeds(rs, spp, seeds, depth):
    return np.stack([rs.render(spp, 2000 + k, depth)[0].astype(np.float64) / spp for k in range(seeds)])


@pytest.mark.parametrize("mode", ["fixed", "online"])
def test_guided_render_is_unbiased(gpu, oracle, mode):
    """Box scene at 32 x 32 at the plain path tracer's gate bar: 16 guided renders of 1,024 spp
    against 16 reference renders of 1,024 spp; |z| < 4 on >= 99.9% of values, mean luminance within
    0.5% (its statistical error here is about 0.15%). 'fixed': random, badly placed lobes selected
    often; 'online': the network trains during the render (4,096-path wavefronts). Both exercise
    the one-sample MIS with the BSDF, NEE's MIS against the mixture pdf, and the Russian roulette
    that tests the BSDF-sampling throughput at guided vertices."""
    w = h = 32
    spp = 1024
    rs = oracle.RefScene(ru.scene_file("guided_box", seed=0, width=w, height=h))
    desc = rs.export()
    guide.set_weights(_weights(7))
    flags = render.GUIDE_SAMPLE | (render.GUIDE_TRAIN if mode == "online" else 0)
    ext = render.make_ext(guide=flags, wavefront_paths=4096 if mode == "online" else 0)
    g = np.stack([render.render_ex(desc, w, h, spp, seed=1000 + k, max_depth=8, ext=ext) / spp for k in range(16)])
    oracle.set_threads(0)
    c = _cpu_seeds(rs, spp, 16, 8)
    z = ru.z_scores(g, c)
    frac = np.mean(np.abs(z) < 4)
    yg, yc = g[..., 1].mean(), c[..., 1].mean()
    print(f"guided ({mode}) vs reference: frac {frac:.5f}, mean Y {yg:.6f} vs {yc:.6f} ({yg / yc - 1:+.3%})")
    assert frac >= 0.999, f"only {frac:.5f} of values within |z| < 4"
    assert abs(yg / yc - 1) < 0.005, f"mean Y guided {yg} reference {yc}"
    if mode == "online":
        assert not np.array_equal(guide.get_weights(), _weights(7))


def _gain(desc, w, depth, train_spp, seeds=12, spp=64):
    """(relMSE plain, relMSE guided, device ms per render plain, guided) after training the guide
    online from fresh weights over train_spp samples per pixel (65,536-path wavefronts, Adam lr
    1e-3 as the guided-vs-plain configuration specifies); relMSE against an 8,192-spp plain render in
    the form of tests/test_quality.cpp:241-248, averaged over `seeds` renders of `spp`."""
    ref = render.render_ex(desc, w, w, 8192, seed=77, max_depth=depth) / 8192
    guide.set_options()
    guide.set_learning_rate(1e-3)
    train = render.make_ext(guide=render.GUIDE_SAMPLE | render.GUIDE_TRAIN | render.GUIDE_RESET, wavefront_paths=65536)
    render.render_ex(desc, w, w, train_spp, seed=5, max_depth=depth, ext=train)
    use = render.make_ext(guide=render.GUIDE_SAMPLE)

    def run(ext):
        errs, ms = [], []
        for k in range(seeds):
            img, st = render.render_ex(desc, w, w, spp, seed=900 + k, max_depth=depth, ext=ext, stats=True)
            errs.append(float(np.mean((img / spp - ref) ** 2 / (ref ** 2 + 1e-2))))
            ms.append(st.deviceMs)
        return float(np.mean(errs)), float(np.median(ms))

    (ep, tp), (eg, tg) = run(None), run(use)
    return ep, eg, tp, tg


def test_trained_guide_gains_on_the_indirectly_lit_box(gpu):
    """The box-and-spheres scene lit only indirectly (its light faces the ceiling: all light reaches
    the room by way of the bright patch above it), 128 x 128, depth 16: after 4,096 spp of online
    training the guided renders' relMSE is at least 2x lower than BSDF sampling's at equal sample
    count and at least 1.5x lower at equal device time of the renders (measured: 3.3x and 2.3x)."""
    w, depth = 128, 16
    desc = hostscene.build_box_scene(scenes.indirect_scene(seed=0, width=w, height=w, max_depth=depth, subdiv=2)).desc()
    ep, eg, tp, tg = _gain(desc, w, depth, 4096)
    print(f"indirect box: relMSE plain {ep:.4e} ({tp:.2f} ms), guided {eg:.4e} ({tg:.2f} ms): "
          f"{ep / eg:.2f}x at equal spp, {ep * tp / (eg * tg):.2f}x at equal time")
    assert ep / eg >= 2.0
    assert ep * tp / (eg * tg) >= 1.5


def test_trained_guide_on_slit_scene_reports_its_gain(gpu):
    """The guided-vs-plain scene (light only through a 0.1-wide slit, 12 subsurface BK7 spheres),
    128 x 128, depth 16: the trained guide lowers relMSE at equal sample count (measured 1.15x;
    asserted > 1.05x). Most of this image's error is in the subsurface spheres' pixels (about 60 %,
    which guiding at diffuse vertices does not reach), so at equal time the guided form's extra
    cost per sample (inference per bounce, about 45 % here) outweighs the gain: the ratio is printed."""
    w, depth = 128, 16
    desc = hostscene.build_box_scene(scenes.slit_scene(seed=0, width=w, height=w, subdiv=2, max_depth=depth)).desc()
    ep, eg, tp, tg = _gain(desc, w, depth, 4096)
    print(f"slit scene: relMSE plain {ep:.4e} ({tp:.2f} ms), guided {eg:.4e} ({tg:.2f} ms): "
          f"{ep / eg:.2f}x at equal spp, {ep * tp / (eg * tg):.2f}x at equal time")
    assert ep / eg > 1.05
