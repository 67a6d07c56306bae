"""Coated and sheen materials on the GPU against the reference: pr::LayeredBxDF (dielectric coat
over a diffuse or conductor base, optional scattering layer; src/materials/bxdf.cpp:260-518) and
pr::SheenBxDF (bxdf.cpp:520-631) on identical local-frame inputs, and path-traced renders of
scenes that use them against the reference PathIntegrator.

The layered f, pdf and sampling walks are stochastic estimators seeded from their inputs; the
reference seeds its walks with its own hash, so single evaluations differ while their
expectations agree. The tests therefore compare (a) sheen over a single lobe exactly (1e-5),
(b) layered f and pdf averaged over 4,096 walks per call within 3 %, (c) samples that leave without
a walk exactly and the directional albedo of the rest within 4 standard errors, (d) images by
the per-pixel z statistic."""

import json
import os
import tempfile
import zlib

import numpy as np
import pytest

import render_util as ru
from prgpu import abi, render, scenes, workloads

pytestmark = pytest.mark.gpu


def _params(layered, kind, R=(0.2, 0.5, 0.8, 0.9), eta=(0.17, 0.43, 1.4, 1.66), k=(3.5, 2.46, 1.88, 1.96), etaD=1.5,
            alpha=(0.3, 0.3), coat_eta=1.5, coat_alpha=0.0, thickness=0.01, g=0.0, albedo=(0, 0, 0, 0), max_depth=64,
            samples=1, sheen_weight=0.0, sheen_rough=0.3, sheen_color=(0.9, 0.6, 0.4, 0.3)):
    p = np.zeros(36, np.float32)
    p[0], p[1] = float(layered), float(kind)
    p[2:6], p[6:10], p[10:14] = R, eta, k
    p[14], p[15], p[16] = etaD, alpha[0], alpha[1]
    p[17], p[18], p[19], p[20] = coat_eta, coat_alpha, thickness, g
    p[21:25] = albedo
    p[25], p[26] = max_depth, samples
    p[27], p[28] = sheen_weight, sheen_rough
    p[29:33] = sheen_color
    return p


def _inputs(rng, n):
    x = np.zeros((n, 9), np.float32)
    x[:, 0:3] = workloads.sphere_directions(rng.random((n, 2), dtype=np.float32))
    x[:, 3:6] = workloads.sphere_directions(rng.random((n, 2), dtype=np.float32))
    x[:, 6:9] = rng.random((n, 3), dtype=np.float32)
    return x


def _table(oracle):
    t = np.zeros(16 * 32, np.float32)
    oracle.ref_lib().prref_sheen_table(oracle._p(t))
    return t


def _run(gpu, oracle, params, x, table):
    ref = np.zeros((len(x), 16), np.float32)
    oracle.ref_lib().prref_full_bsdf(oracle._p(params), len(x), oracle._p(x), oracle._p(ref))
    out = np.zeros_like(ref)
    err = abi.err_buf()
    abi.check(gpu.prgpu_eval_full_bsdf(0, abi.ptr(params), abi.ptr(table), len(x), abi.ptr(x), abi.ptr(out), err,
                                       len(err)), err, "prgpu_eval_full_bsdf")
    return out, ref


def _close(a, b, what, rel=1e-5):
    a, b = a.astype(np.float64), b.astype(np.float64)
    scale = np.maximum(np.abs(a).max(axis=0, keepdims=True), 1e-30)
    tol = rel * np.maximum(np.maximum(np.abs(a), np.abs(b)), scale)
    bad = ~(np.abs(a - b) <= tol)
    assert not bad.any(), f"{what}: {bad.sum()} of {a.size} values beyond {rel}"


SHEEN = {
    "sheen_diffuse": _params(0, 0, sheen_weight=1.0, sheen_rough=0.35),
    "sheen_conductor": _params(0, 1, sheen_weight=0.7, sheen_rough=0.8),
    "sheen_dielectric_rough": _params(0, 2, etaD=1.5, alpha=(0.25, 0.25), sheen_weight=0.5, sheen_rough=0.1),
}


@pytest.mark.parametrize("name", sorted(SHEEN))
def test_sheen_over_a_lobe_matches_reference(gpu, oracle, name):
    """Sheen over one lobe is deterministic: f, pdf and samples within 1e-5."""
    x = _inputs(np.random.default_rng(zlib.crc32(name.encode())), 1 << 15)
    out, ref = _run(gpu, oracle, SHEEN[name], x, _table(oracle))
    _close(out[:, 0:4], ref[:, 0:4], f"{name} f")
    _close(out[:, 4:5], ref[:, 4:5], f"{name} pdf")
    np.testing.assert_array_equal(out[:, 5], ref[:, 5])
    ok = ref[:, 5] == 1
    np.testing.assert_array_equal(out[ok, 14], ref[ok, 14])
    np.testing.assert_array_equal(out[ok, 15], ref[ok, 15])
    _close(out[ok, 6:11], ref[ok, 6:11], f"{name} sample f/pdf")
    _close(out[ok, 11:14], ref[ok, 11:14], f"{name} sample wi")


LAYERED = {
    "coated_diffuse_smooth": _params(1, 0, coat_alpha=0.0),
    "coated_diffuse_rough_albedo": _params(1, 0, coat_alpha=0.2, thickness=0.1, g=0.3, albedo=(0.8, 0.5, 0.3, 0.9)),
    "coated_conductor_rough": _params(1, 1, eta=(0.11, 0.29, 0.93, 1.1), k=(2.3, 1.6, 1.25, 1.3), alpha=(0.2, 0.2),
                                      coat_alpha=0.05),
    "coated_diffuse_sheen": _params(1, 0, coat_alpha=0.1, sheen_weight=0.8, sheen_rough=0.5),
}


@pytest.mark.parametrize("name", sorted(LAYERED))
def test_layered_expectations_match_reference(gpu, oracle, name):
    """f and pdf from 4,096 walks per call on 48 direction pairs within 3 % (plus 2 % of the batch
    maximum, for values that average near zero)."""
    p = LAYERED[name].copy()
    p[26] = 4096
    x = _inputs(np.random.default_rng(zlib.crc32(name.encode()) + 1), 48)
    out, ref = _run(gpu, oracle, p, x, _table(oracle))
    for cols, what in ((slice(0, 4), "f"), (slice(4, 5), "pdf")):
        a, b = out[:, cols].astype(np.float64), ref[:, cols].astype(np.float64)
        tol = 0.03 * np.maximum(np.abs(a), np.abs(b)) + 0.02 * np.abs(b).max()
        bad = np.abs(a - b) > tol
        assert not bad.any(), f"{name} {what}: {bad.sum()} values beyond 3 %: gpu {a[bad][:4]} ref {b[bad][:4]}"


@pytest.mark.parametrize("name", sorted(LAYERED))
def test_layered_sampling_matches_reference(gpu, oracle, name):
    """Samples that reflect off the coat equal the reference's (1e-5); over all samples at four
    outgoing directions, the mean weight f |cos| / pdf (the directional albedo) agrees within 4
    standard errors."""
    table = _table(oracle)
    rng = np.random.default_rng(zlib.crc32(name.encode()) + 2)
    for cos_o in (0.95, 0.7, 0.4, 0.15):
        n = 1 << 16
        x = np.zeros((n, 9), np.float32)
        x[:, 0:3] = [np.sqrt(1 - cos_o ** 2), 0.0, cos_o]
        x[:, 3:6] = [0.0, 0.0, 1.0]
        x[:, 6:9] = rng.random((n, 3), dtype=np.float32)
        out, ref = _run(gpu, oracle, LAYERED[name], x, table)
        both = (out[:, 5] == 1) & (ref[:, 5] == 1)
        # Samples that need no walk (coat reflections, sheen's cosine lobe) leave in the same
        # direction with the same value; walk exits never coincide.
        same = both & np.all(np.abs(out[:, 11:14] - ref[:, 11:14]) <= 1e-6, axis=1)
        assert same.mean() > 0.02, f"{name}: only {same.mean():.3f} of samples left without a walk"
        np.testing.assert_array_equal(out[same, 14], ref[same, 14])
        _close(out[same, 6:11], ref[same, 6:11], f"{name} coat reflection f/pdf")
        wg = np.where(out[:, 5] == 1, out[:, 6:10].mean(1) * np.abs(out[:, 13]) / np.maximum(out[:, 10], 1e-30), 0.0)
        wr = np.where(ref[:, 5] == 1, ref[:, 6:10].mean(1) * np.abs(ref[:, 13]) / np.maximum(ref[:, 10], 1e-30), 0.0)
        se = np.sqrt(wg.var() / n + wr.var() / n)
        assert abs(wg.mean() - wr.mean()) < 4 * se + 1e-6, f"{name} cos {cos_o}: albedo gpu {wg.mean()} ref {wr.mean()}"


def _coated_scene_file(name, **kw):
    """The box scene with its spheres re-dressed in coated / sheen materials (reference JSON)."""
    s = scenes.box_scene(**kw)
    doc = scenes.to_reference_json(s)
    mats = doc["materials"]
    mats["coat_red"] = {"type": "coated_diffuse", "reflectance": [0.7, 0.15, 0.1], "coat_roughness": 0.1}
    mats["coat_smoke"] = {"type": "coated_diffuse", "reflectance": [0.2, 0.6, 0.8], "coat_roughness": 0.3,
                          "thickness": 0.2, "albedo": [0.9, 0.7, 0.5], "g": 0.4}
    mats["coat_gold"] = {"type": "coated_conductor", "metal": "Au", "roughness": 0.3, "coat_roughness": 0.05}
    mats["velvet"] = {"type": "diffuse", "reflectance": [0.4, 0.1, 0.3],
                      "sheen": {"color": [1.0, 0.8, 0.9], "roughness": 0.3, "weight": 1.0}}
    mats["sheen_coat"] = {"type": "coated_diffuse", "reflectance": [0.1, 0.4, 0.2],
                          "sheen": {"color": [0.9, 0.9, 0.6], "roughness": 0.6, "weight": 0.7}}
    cycle = ["coat_red", "coat_smoke", "coat_gold", "velvet", "sheen_coat"]
    k = 0
    for o in doc["objects"]:
        if o["geometry"].startswith("sphere"):
            o["material"] = cycle[k % len(cycle)]
            k += 1
    path = os.path.join(tempfile.gettempdir(), "prb_scenes", name + ".prscene.json")
    os.makedirs(os.path.dirname(path), exist_ok=True)
    with open(path, "w") as f:
        json.dump(doc, f)
    return path


def test_coated_and_sheen_scene_agrees_with_reference(gpu, oracle):
    """Box scene, 35 spheres cycling through coated diffuse (clear and with a scattering layer),
    coated gold, sheen over diffuse and sheen over a coat; 32 x 32, depth 8; 16 renders of 256 spp
    each side: |z| < 4 on >= 99.5 % of values, mean luminance within 4 standard errors."""
    w = h = 32
    rs = oracle.RefScene(_coated_scene_file("coated_box", seed=3, width=w, height=h, subdiv=2))
    desc = rs.export()
    g = np.stack([render.render_ex(desc, w, h, 256, seed=1000 + k, max_depth=8) / 256 for k in range(16)])
    c = np.stack([rs.render(256, 2000 + k, 8)[0].astype(np.float64) / 256 for k in range(16)])
    z = ru.z_scores(g, c)
    frac = np.mean(np.abs(z) < 4)
    mg, mc = g[..., 1].mean(axis=(1, 2)), c[..., 1].mean(axis=(1, 2))
    se = np.sqrt(mg.var(ddof=1) / len(mg) + mc.var(ddof=1) / len(mc))
    print(f"coated scene: frac {frac:.4f}, mean Y gpu {mg.mean():.5f} cpu {mc.mean():.5f} se {se:.5f}")
    assert frac >= 0.995, f"only {frac:.4f} of values within |z| < 4"
    assert abs(mg.mean() - mc.mean()) < 4 * se, f"mean Y gpu {mg.mean()} cpu {mc.mean()} (se {se})"
