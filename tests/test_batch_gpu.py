"""Batched renders (prgpu_render_batch): renders of uneven resolution, sample count and path length
in one wavefront, run as one CUDA graph launch with a device-side loop. Every path depends only on
its own (pixel, sample index, seed) stream and each film adds its samples in sample order, so a
batch must reproduce, bit for bit, what prgpu_render_ex gives for each render alone -- whatever
the wave packing (small wavefronts force many waves and pixel-range chunks)."""

import numpy as np
import pytest

import render_util as ru
from prgpu import abi, hostscene, render, scenes

pytestmark = pytest.mark.gpu


def _mixed_batch(oracle):
    """(scene, ext, params, w, h) for 6 renders: plain, homogeneous medium, grid smoke; sizes from
    16x16 to 40x24, 3 to 16 spp, depth 4, 8 and unlimited."""
    out = []
    specs = [(0, 16, 16, 8, 8, False), (1, 40, 24, 3, 0, True), (2, 32, 32, 16, 4, False),
             (3, 24, 40, 5, 8, True), (4, 20, 20, 7, 8, False)]
    for seed, w, h, spp, depth, medium in specs:
        rs = oracle.RefScene(ru.scene_file(f"batch_{seed}", seed=seed, width=w, height=h, medium=medium))
        out.append((rs, None, dict(spp=spp, seed=100 + seed, max_depth=depth), w, h))
    path, s = ru.grid_scene_file("batch_grid", seed=5, width=24, height=24)
    rs = oracle.RefScene(path)
    sd, ext = ru.grid_scene_inputs(rs, s)
    out.append(((rs, sd), ext, dict(spp=6, seed=105, max_depth=8), 24, 24))
    return out


def _desc(scene):
    if isinstance(scene, tuple):
        return scene[1]
    return scene.export()


def _alone(batch):
    films = []
    for scene, ext, p, w, h in batch:
        films.append(render.render_ex(_desc(scene), w, h, p["spp"], seed=p["seed"], max_depth=p["max_depth"], ext=ext))
    return films


@pytest.mark.parametrize("capacity", [1024, 1 << 20])
def test_batch_matches_single_renders_bit_for_bit(gpu, oracle, capacity):
    batch = _mixed_batch(oracle)
    ref = _alone(batch)
    films = [np.zeros((h, w, 3)) for *_, w, h in batch]
    st = render.render_batch([(_desc(sc), ext, p, f) for (sc, ext, p, _, _), f in zip(batch, films)],
                             config=render.batch_config(capacity, 128), stats=True)
    for k, (a, b) in enumerate(zip(films, ref)):
        assert np.array_equal(a, b), f"render {k} differs (max |d| {np.abs(a - b).max()})"
    assert st.pathSamples == sum(w * h * p["spp"] for _, _, p, w, h in batch)
    assert st.waves >= (8 if capacity == 1024 else 1) and st.loopIterations > 0 and st.closestRays > 0


def test_host_driven_loop_gives_the_same_films(gpu, oracle):
    """The host-driven mode (no graph; for profilers) runs the same iteration kernels."""
    batch = _mixed_batch(oracle)[:4]
    ref = _alone(batch)
    films = [np.zeros((h, w, 3)) for *_, w, h in batch]
    st = render.render_batch([(_desc(sc), ext, p, f) for (sc, ext, p, _, _), f in zip(batch, films)],
                             config=render.batch_config(2048, 256, host_loop=True), stats=True)
    assert st.graphBuilt == 0
    for a, b in zip(films, ref):
        assert np.array_equal(a, b)


def test_batch_adds_onto_films_and_resumes(gpu, oracle):
    """Films are accumulated onto (read, added to, written back): 3 + 5 samples equal 8."""
    batch = _mixed_batch(oracle)[:3]
    full = [np.zeros((h, w, 3)) for *_, w, h in batch]
    render.render_batch([(_desc(sc), ext, dict(p, spp=8), f) for (sc, ext, p, _, _), f in zip(batch, full)],
                        config=render.batch_config(4096, 256))
    part = [np.zeros((h, w, 3)) for *_, w, h in batch]
    items = [(_desc(sc), ext, dict(p, spp=3), f) for (sc, ext, p, _, _), f in zip(batch, part)]
    render.render_batch(items, config=render.batch_config(4096, 256))
    items = [(_desc(sc), ext, dict(p, spp=5, first_sample=3), f) for (sc, ext, p, _, _), f in zip(batch, part)]
    render.render_batch(items, config=render.batch_config(8192, 128))
    for a, b in zip(full, part):
        assert np.array_equal(a, b)


def test_autotuner_picks_a_valid_config_and_caches_it(gpu):
    """Host-built scenes (no reference loader): the tuner times its candidates once per batch
    shape; render_batch with no config then reuses the choice."""
    hs = [hostscene.build_box_scene(scenes.box_scene(seed=k, width=32, height=32, medium=bool(k % 2)))
          for k in range(4)]
    items = [(h.desc(), None, dict(spp=16, seed=k, max_depth=8), np.zeros((32, 32, 3))) for k, h in enumerate(hs)]
    cfg = render.autotune_batch(items)
    assert cfg.wavefrontPaths in (1 << 20, 1 << 21, 1 << 22, 1 << 23) and cfg.shadeBlock in (128, 256)
    st = render.render_batch(items, stats=True)
    assert st.tuned == 0 and st.wavefrontPaths == cfg.wavefrontPaths and st.shadeBlock == cfg.shadeBlock
    for k, (h, _, p, f) in enumerate(items):
        alone = render.render_ex(h, 32, 32, 16, seed=k, max_depth=8)
        assert np.array_equal(f, alone)


def test_batch_input_validation(gpu):
    h = hostscene.build_box_scene(scenes.box_scene(seed=0, width=8, height=8))
    film = np.zeros((8, 8, 3))
    item = [(h.desc(), None, dict(spp=1), film)]
    with pytest.raises(abi.PrgpuError, match="shadeBlock"):
        render.render_batch(item, config=render.batch_config(4096, 100))
    with pytest.raises(abi.PrgpuError, match="wavefrontPaths"):
        render.render_batch(item, config=render.batch_config(100, 128))
    with pytest.raises(abi.PrgpuError, match="batch size"):
        render.render_batch([], config=render.batch_config(4096, 128))
    assert not film.any()


def _guide_weights(seed):
    """Fixed random weights with peaked, badly placed lobes (the unbiasedness tests' stress case)."""
    import guide_ref as G

    p = G.init_params(seed).astype(np.float64)
    rng = np.random.default_rng(seed + 1)
    W = G.split(p)
    W[0][:, G.CONST_IN] = rng.normal(0, 0.5, W[0].shape[0])
    for l in range(1, 5):
        W[l][:, G.CONST_HID] = rng.normal(0, 0.5, W[l].shape[0])
    for l in range(4):
        W[l][G.CONST_HID, :] = 0
    W[4][41:, :] = 0
    W[4][40, G.CONST_HID] = 1.5
    return p.astype(np.float32)


def test_guided_batch_matches_guided_single_renders_bit_for_bit(gpu):
    """The guided, batched form with fixed weights: per-render guide flags (two renders sampling with
    the guide, one plain) in one graph launch give exactly the films of one prgpu_render_ex per
    render -- the network's inference per bounce runs inside the batch's graph on the shared
    diffuse queue, and a path's decision depends only on its own row."""
    from prgpu import guide

    guide.set_weights(_guide_weights(11))
    specs = [(0, 40, 24, 6, 8, render.GUIDE_SAMPLE), (1, 32, 32, 5, 8, 0), (2, 24, 40, 7, 6, render.GUIDE_SAMPLE)]
    items, alone = [], []
    for seed, w, h, spp, depth, flags in specs:
        hs = hostscene.build_box_scene(scenes.box_scene(seed=seed, width=w, height=h, medium=bool(seed % 2)))
        ext = render.make_ext(guide=flags) if flags else None
        p = dict(spp=spp, seed=300 + seed, max_depth=depth)
        alone.append(render.render_ex(hs.desc(), w, h, spp, seed=p["seed"], max_depth=depth, ext=ext))
        items.append((hs.desc(), ext, p, np.zeros((h, w, 3))))
    for capacity in (2048, 1 << 20):
        films = [np.zeros_like(f) for *_, f in items]
        render.render_batch([(d, e, p, f) for (d, e, p, _), f in zip(items, films)],
                            config=render.batch_config(capacity, 128))
        for k, (a, b) in enumerate(zip(films, alone)):
            assert np.array_equal(a, b), f"capacity {capacity}, render {k} differs (max |d| {np.abs(a - b).max()})"


def test_guided_batch_trains_online_and_stays_unbiased(gpu, oracle):
    """Guided renders that also train the network online inside the batch's graph (collect + Adam
    steps after every filmed wave): the weights move, Adam steps are taken, and the trained-on-the-fly
    image agrees with the reference PathIntegrator (16 batch items of 256 spp, |z| < 4 on >= 99.5%
    of values, mean luminance within 1.5%)."""
    from prgpu import guide

    w = h = 32
    rs = oracle.RefScene(ru.scene_file("guided_batch_box", seed=0, width=w, height=h))
    desc = rs.export()
    guide.set_weights(_guide_weights(7))
    before = guide.get_weights()
    steps0 = guide.stats()["steps"]
    ext = render.make_ext(guide=render.GUIDE_SAMPLE | render.GUIDE_TRAIN)
    films = [np.zeros((h, w, 3)) for _ in range(16)]
    render.render_batch([(desc, ext, dict(spp=256, seed=1000 + k, max_depth=8), f) for k, f in enumerate(films)],
                        config=render.batch_config(1 << 16, 128))
    assert not np.array_equal(guide.get_weights(), before)
    assert guide.stats()["steps"] > steps0
    g = np.stack(films) / 256
    c = np.stack([rs.render(256, 2000 + k, 8)[0].astype(np.float64) / 256 for k in range(16)])
    z = ru.z_scores(g, c)
    frac = np.mean(np.abs(z) < 4)
    yg, yc = g[..., 1].mean(), c[..., 1].mean()
    print(f"guided batch, online training: frac {frac:.4f}, mean Y {yg:.5f} vs {yc:.5f}, "
          f"{guide.stats()['steps'] - steps0} Adam steps")
    assert frac >= 0.995, f"only {frac:.4f} of values within |z| < 4"
    assert abs(yg / yc - 1) < 0.015, f"mean Y guided batch {yg} reference {yc}"
