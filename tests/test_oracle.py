"""The oracle itself, pinned before it is trusted: the plain-C restatement (oracle/restate.c)
against the reference's compiled code (oracle/_ref/libprref.so), and both against the
reference's own known-answer tests (tests/test_bsdf.cpp:114-119, tests/test_spectrum.cpp:23-75)
and the committed golden vectors (tests/golden/, made by tests/golden/make_golden.py)."""

import os

import numpy as np
import pytest

from prgpu import abi, workloads

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _restate_trace(oracle, nodes, order, verts, rays8, any_hit=False):
    lib = oracle.restate_lib()
    n = rays8.shape[0]
    prim = np.empty(n, np.int32)
    t = np.empty(n, np.float32)
    nv = np.empty(n, np.int32)
    nt = np.empty(n, np.int32)
    st = lib.rs_trace(oracle._p(nodes), len(nodes), oracle._p(order), oracle._p(verts), oracle._p(rays8), n,
                      1 if any_hit else 0, oracle._p(prim), oracle._p(t), oracle._p(nv), oracle._p(nt))
    assert st == 0
    return prim, t, nv, nt


@pytest.mark.parametrize("ntris", [1, 7, 1 << 12])
def test_restated_traversal_is_bit_exact_with_reference(oracle, ntris):
    verts = workloads.triangle_soup(ntris, seed=ntris)
    b = oracle.SoupBVH(verts)
    nodes, order = b.export(abi.BVH_NODE)
    rays = workloads.rays_as_f8(workloads.soup_rays(1 << 14, seed=5))
    rp, rt, _, _, _ = b.trace(rays)
    p, t, nv, nt = _restate_trace(oracle, nodes, order, verts, rays)
    np.testing.assert_array_equal(p, rp)
    np.testing.assert_array_equal(t[rp >= 0].view(np.int32), rt[rp >= 0].view(np.int32))
    arays = workloads.rays_as_f8(workloads.soup_rays(1 << 14, seed=6, any_hit=True))
    ro, _ = b.trace(arays, any_hit=True)
    po, _, _, _ = _restate_trace(oracle, nodes, order, verts, arays, any_hit=True)
    np.testing.assert_array_equal(po, ro)


def test_golden_traversal_vectors(oracle):
    """Committed closest-hit answers of the reference on a small soup (tests/golden/traversal.npz)."""
    g = np.load(os.path.join(GOLDEN, "traversal.npz"))
    b = oracle.SoupBVH(g["verts"])
    prim, t, _, _, _ = b.trace(g["rays"])
    np.testing.assert_array_equal(prim, g["prim"])
    np.testing.assert_array_equal(t.view(np.int32), g["t_bits"])
    nodes, order = b.export(abi.BVH_NODE)
    p, t2, _, _ = _restate_trace(oracle, nodes, order, g["verts"], g["rays"])
    np.testing.assert_array_equal(p, g["prim"])


def test_reference_known_answers(oracle):
    """Fresnel limits and dispersion data (tests/test_bsdf.cpp:114-119, tests/test_spectrum.cpp:66-75)."""
    lib = oracle.ref_lib()
    assert abs(lib.prref_fr_dielectric(1.0, 1.5) - 0.04) < 1e-4
    assert lib.prref_fr_dielectric(0.1, 1 / 1.5) == pytest.approx(1.0)
    assert abs(lib.prref_fr_complex(1.0, 1.0, 0.0)) < 1e-6
    lam = np.array([587.6], np.float32)
    out = np.zeros(1, np.float32)
    lib.prref_spectrum(4, 0, 0, 0, b"BK7", 1, oracle._p(lam), oracle._p(out))
    assert abs(out[0] - 1.5168) < 1e-3
    lib.prref_spectrum(4, 0, 0, 0, b"SF11", 1, oracle._p(lam), oracle._p(out))
    assert abs(out[0] - 1.7847) < 1e-3
    lam[0] = 589.0
    lib.prref_spectrum(4, 0, 0, 0, b"diamond", 1, oracle._p(lam), oracle._p(out))
    assert abs(out[0] - 2.417) < 2e-3


def test_wavelength_pdf_integrates_to_one(oracle):
    """The hero-wavelength pdf integrates to 1 over 360-830 nm (tests/test_spectrum.cpp:23-27)."""
    lib = oracle.ref_lib()
    u = ((np.arange(1 << 16) + 0.5) / (1 << 16)).astype(np.float32)
    lam = np.zeros((len(u), 4), np.float32)
    pdf = np.zeros((len(u), 4), np.float32)
    lib.prref_sample_visible(len(u), oracle._p(u), oracle._p(lam), oracle._p(pdf))
    assert lam.min() >= 360 and lam.max() <= 830
    # E[1/pdf] over the sampled distribution is the length of the support.
    assert abs(np.mean(1.0 / pdf[:, 0]) - 470.0) / 470.0 < 5e-3


def test_golden_function_vectors(oracle):
    """BxDF / phase / medium outputs of the reference on fixed inputs (tests/golden/functions.npz)."""
    g = np.load(os.path.join(GOLDEN, "functions.npz"))
    lib = oracle.ref_lib()
    for kind in range(4):
        params = g[f"params{kind}"]
        inp = g[f"in{kind}"]
        out = np.zeros((inp.shape[0], 16), np.float32)
        lib.prref_bxdf(kind, oracle._p(params), inp.shape[0], oracle._p(inp), oracle._p(out))
        np.testing.assert_array_equal(out.view(np.int32), g[f"out{kind}"].view(np.int32))
