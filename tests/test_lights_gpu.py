"""Light-BVH next-event estimation against the reference pr::BVHLightSampler
(src/lights/light_bvh.cpp:45-234), on a scene of 48 emitters of different power (the pattern of the
reference test "light BVH: PMF matches sampling frequencies and renders agree with power sampling",
tests/test_lights.cpp:137-204): the tree built by libprender_host.so from the same light bounds and
the device descent must pick the same light with the same probability, the device pmf walk must
match BVHLightSampler::PMF, and a render with the light BVH must agree with the reference."""

import ctypes as C
import json
import os
import tempfile

import numpy as np
import pytest

import render_util as ru
from prgpu import abi, render

pytestmark = pytest.mark.gpu


def _scene(path, w=32, h=32, seed=3):
    rng = np.random.default_rng(seed)
    lights = {}
    for i in range(48):
        pos = [float(x) for x in rng.uniform([-1.5, 0.4, -1.5], [1.5, 1.6, 1.5])]
        d = rng.normal(size=3)
        d[1] = -abs(d[1]) - 0.5
        lights[f"l{i}"] = {"type": "rect", "position": pos, "size": [0.12, 0.12], "direction": [float(x) for x in d],
                           "temperature": 5000, "luminance": float(rng.uniform(1, 12))}
    doc = {
        "materials": {"grey": {"type": "diffuse", "reflectance": [0.6, 0.6, 0.6]}},
        "geometry": {"floor": {"type": "mesh", "positions": [-2, 0, -2, 2, 0, -2, 2, 0, 2, -2, 0, 2],
                               "indices": [0, 2, 1, 0, 3, 2]},
                     "ball": {"type": "sphere", "radius": 0.3, "center": [0, 0.3, 0]}},
        "objects": [{"geometry": "floor", "material": "grey"}, {"geometry": "ball", "material": "grey"}],
        "lights": lights,
        "cameras": {"cam": {"type": "pinhole", "position": [0, 2.5, 3.5], "look_at": [0, 0, 0], "fov_y": 50}},
        "render": {"camera": "cam", "film": {"width": w, "height": h, "filter": "box"},
                   "integrator": {"type": "path", "spp": 16, "max_depth": 5}},
    }
    with open(path, "w") as f:
        json.dump(doc, f)
    return path


def _arr(addr, count, dtype):
    return np.ctypeslib.as_array((C.c_byte * (count * dtype.itemsize)).from_address(addr)).view(dtype).copy()


def _light_tree(sd):
    """Light bounds as the reference computes them for triangle area lights (light.cpp:90-103,
    shape.cpp:266-273): triangle box, face normal turned towards the vertex normals, a narrow
    normal cone (cosThetaO 1), emission to the hemisphere (cosThetaE 0), phi = scale * max(L) *
    area * pi; then this library's builder."""
    lights = _arr(sd.lights, sd.lightCount, abi.LIGHT)
    prims = _arr(sd.prims, sd.primCount, abi.PRIMITIVE)
    spec = np.ctypeslib.as_array((C.c_float * (sd.spectrumCount * abi.SPECTRUM_SAMPLES)).from_address(
        sd.spectra)).reshape(sd.spectrumCount, abi.SPECTRUM_SAMPLES).copy()
    lb = np.zeros((len(lights), 13), np.float32)
    for i, l in enumerate(lights):
        pr = prims[l["primitive"]]
        tri = np.stack([pr["p0"], pr["p1"], pr["p2"]]).astype(np.float64)
        n = np.cross(tri[1] - tri[0], tri[2] - tri[0])
        n /= np.linalg.norm(n)
        vn = pr["n0"] + pr["n1"] + pr["n2"]
        if np.dot(n, vn) < 0:
            n = -n
        lb[i, 0:3], lb[i, 3:6] = tri.min(0), tri.max(0)
        lb[i, 6:9] = n
        lb[i, 9] = l["scale"] * spec[l["spectrum"]].max() * l["area"] * np.pi
        lb[i, 10], lb[i, 11] = 1.0, 0.0
    nodes = np.zeros(2 * len(lights) - 1, abi.LIGHT_BVH_NODE)
    cnt = abi.host_lib().prhost_build_light_bvh(abi.ptr(lb), len(lights), abi.ptr(nodes))
    assert cnt == 2 * len(lights) - 1
    return nodes


@pytest.fixture(scope="module")
def lightscene(oracle):
    path = _scene(os.path.join(tempfile.gettempdir(), "prb_lights48.prscene.json"))
    rs = oracle.RefScene(path)
    sd = abi.SceneDesc.from_address(rs.export())
    return rs, sd, _light_tree(sd)


def test_light_bvh_sampling_and_pmf_match_reference(gpu, lightscene):
    rs, sd, nodes = lightscene
    assert rs.light_count() == sd.lightCount == 96  # two triangles per rect emitter
    rng = np.random.default_rng(9)
    n = 20000
    q = np.zeros((n, 7), np.float32)
    q[:, 0:3] = rng.uniform([-2, 0, -2], [2, 1.2, 2], (n, 3))
    nrm = rng.normal(size=(n, 3))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    nrm[: n // 4] = 0  # points in media (no receiver cosine)
    q[:, 3:6] = nrm
    q[:, 6] = rng.random(n, dtype=np.float32)
    ref_out, ref_pmf = rs.light_bvh_sample(q)
    out = np.zeros((n, 2), np.float32)
    pmf = np.zeros((n, 96), np.float32)
    err = abi.err_buf()
    abi.check(gpu.prgpu_eval_light_bvh(0, abi.ptr(nodes), len(nodes), 96, 1.0, n, abi.ptr(q), abi.ptr(out),
                                       abi.ptr(pmf), err, len(err)), err, "prgpu_eval_light_bvh")
    same = out[:, 0] == ref_out[:, 0]
    # A different light only where u falls within float rounding of a child-selection boundary.
    assert same.mean() > 0.999, same.mean()
    np.testing.assert_allclose(out[same, 1], ref_out[same, 1], rtol=2e-5)
    # Near-zero pmfs come from importance terms that cancel (cosines at the edge of a cone), where
    # float rounding alone moves them by ~1e-6.
    np.testing.assert_allclose(pmf, ref_pmf, rtol=2e-5, atol=5e-6)
    # The pmfs sum to at most 1: the sampler gives up (no light) below a node whose two children
    # both have zero importance (light_bvh.cpp:179-214), and that probability is missing alike.
    assert pmf.sum(1).max() < 1.0 + 1e-4
    np.testing.assert_allclose(pmf.sum(1), ref_pmf.sum(1), rtol=1e-4, atol=1e-4)
    # The pmf of the chosen light is the probability it was chosen with.
    np.testing.assert_allclose(out[same & (out[:, 0] >= 0), 1],
                               pmf[same & (out[:, 0] >= 0), out[same & (out[:, 0] >= 0), 0].astype(int)], rtol=2e-5)


def test_render_with_light_bvh_agrees_with_reference(gpu, lightscene):
    rs, sd, nodes = lightscene
    w = h = 32
    desc = rs.export()
    ext = render.make_ext(light_bvh=nodes, light_bvh_prob=1.0)
    g = np.stack([render.render_ex(desc, w, h, 128, seed=100 + k, max_depth=5, ext=ext) / 128 for k in range(12)])
    c = np.stack([rs.render(128, 200 + k, 5)[0].astype(np.float64) / 128 for k in range(12)])
    p = np.stack([render.render_ex(desc, w, h, 128, seed=300 + k, max_depth=5) / 128 for k in range(12)])
    assert abs(g[..., 1].mean() / c[..., 1].mean() - 1) < 0.02
    assert abs(g[..., 1].mean() / p[..., 1].mean() - 1) < 0.02
    assert np.mean(np.abs(ru.z_scores(g, c)) < 4) >= 0.99
