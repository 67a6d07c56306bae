"""The guide network's CPU oracle pinned on its own: there is no reference implementation of the
learned part, so its FP64 backward pass is checked against central finite differences, and its
mixture sampling against its pdf (no GPU)."""

import numpy as np
import pytest

import guide_ref as G


def _batch(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1, 1, (n, 3))
    nrm = rng.normal(size=(n, 3))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    wo = rng.normal(size=(n, 3))
    wo /= np.linalg.norm(wo, axis=1, keepdims=True)
    wi = rng.normal(size=(n, 3))
    wi /= np.linalg.norm(wi, axis=1, keepdims=True)
    X = G.features(x, nrm, wo, [-1, -1, -1], [2, 2, 2])
    pb = np.abs(wi[:, 2]) / np.pi + 0.05
    w = rng.exponential(1.0, n)
    return X, wi, pb, w


def test_features_layout():
    X, *_ = _batch(4, 0)
    assert X.shape == (4, 128)
    assert np.all(X[:, 81] == 1.0) and np.all(X[:, 82:] == 0.0)
    np.testing.assert_allclose(X[:, 3] ** 2 + X[:, 4] ** 2, 1.0)


def test_init_keeps_constant_units_inert():
    p = G.init_params(3).astype(np.float64)
    W = G.split(p)
    assert p.size == G.N_PARAMS == 23552
    for l in range(4):
        assert not W[l][63].any()
    assert not W[4][41:].any()


def test_output_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    n = 6
    o = rng.normal(0, 1.0, (n, 48))
    X, wi, pb, w = _batch(n, 2)
    nrm = X[:, 75:78]
    wi = np.where((wi * nrm).sum(1, keepdims=True) < 0, G.mirror(wi, nrm), wi)
    # The gradient is that of the surrogate whose mixture term holds q_n at its current value.
    q0 = G.mixture_q(o, wi, nrm)
    _, g = G.loss_and_grad_out(o, wi, pb, w, nrm, q_fixed=q0)
    h = 1e-6
    for i in list(range(0, 41)):
        d = np.zeros_like(o)
        d[:, i] = h
        lp, _ = G.loss_and_grad_out(o + d, wi, pb, w, nrm, q_fixed=q0)
        lm, _ = G.loss_and_grad_out(o - d, wi, pb, w, nrm, q_fixed=q0)
        np.testing.assert_allclose(g[:, i], (lp - lm) / (2 * h), rtol=1e-5, atol=1e-7)


def test_output_gradient_with_settings_matches_finite_differences():
    """Selection cap 0.6, log kappa capped at 3 (some lobes beyond it), second-moment selection
    objective: the analytic output gradient is that of the surrogate loss."""
    rng = np.random.default_rng(11)
    n = 6
    o = rng.normal(0, 1.5, (n, 48))
    o[:, 3:40:10] += 3.0  # lobes 0, 2, 4, 6 concentrated, some beyond the cap
    X, wi, pb, w = _batch(n, 12)
    nrm = X[:, 75:78]
    wi = np.where((wi * nrm).sum(1, keepdims=True) < 0, G.mirror(wi, nrm), wi)
    opts = dict(max_select=0.6, log_kappa_max=3.0, select_loss=1)
    q0 = G.mixture_q(o, wi, nrm, log_kappa_max=3.0)
    _, g = G.loss_and_grad_out(o, wi, pb, w, nrm, q_fixed=q0, **opts)
    assert (o[:, :40].reshape(n, 8, 5)[:, :, 3] > 3.0).any()
    h = 1e-6
    for i in range(41):
        d = np.zeros_like(o)
        d[:, i] = h
        lp, _ = G.loss_and_grad_out(o + d, wi, pb, w, nrm, q_fixed=q0, **opts)
        lm, _ = G.loss_and_grad_out(o - d, wi, pb, w, nrm, q_fixed=q0, **opts)
        np.testing.assert_allclose(g[:, i], (lp - lm) / (2 * h), rtol=1e-5, atol=1e-7)
    # The selection gradient is -w^2 (q - pb) / p times dc/do40.
    c = G.decode(o, 0.6, 3.0)[3]
    p = c * q0 + (1 - c) * pb
    s = 1 / (1 + np.exp(-o[:, 40]))
    np.testing.assert_allclose(g[:, 40], -w * w * (q0 - pb) / p * 0.6 * s * (1 - s), rtol=1e-12)


def test_weight_gradient_matches_finite_differences():
    p = G.init_params(5).astype(np.float64)
    X, wi, pb, w = _batch(8, 6)
    _, grad = G.backward(p, X, wi, pb, w, round16=False)
    rng = np.random.default_rng(7)
    idx = np.concatenate([rng.choice(np.flatnonzero(p != 0), 40, replace=False), [81, 8192 + 64 * 5 + 63]])
    h = 1e-4  # the loss carries ~1e-12 of rounding noise, so smaller steps lose digits
    nrm = X[:, 75:78]
    q0 = G.mixture_q(G.forward(p, X, False)[0], wi, nrm)
    for i in idx:
        d = np.zeros_like(p)
        d[i] = h
        lp = G.loss_and_grad_out(G.forward(p + d, X, False)[0], wi, pb, w, nrm, q_fixed=q0)[0].sum()
        lm = G.loss_and_grad_out(G.forward(p - d, X, False)[0], wi, pb, w, nrm, q_fixed=q0)[0].sum()
        assert abs(grad[i] - (lp - lm) / (2 * h)) <= 1e-3 * max(0.1, abs(grad[i])), i


def test_mixture_sampling_follows_its_pdf():
    """E[g(w) / q(w)] over mixture samples equals the integral of g over the sphere (g = 1 and a
    smooth test function), for one random mixture."""
    rng = np.random.default_rng(9)
    o = rng.normal(0, 1.0, (1, 48))
    o[0, 3:40:5] = rng.uniform(-1, 4, 8)
    n = 200000
    oo = np.repeat(o, n, 0)
    w = G.sample(oo, rng.random(n), rng.random(n), rng.random(n))
    np.testing.assert_allclose(np.linalg.norm(w, axis=1), 1.0, atol=1e-9)
    q, _ = G.mixture_pdf(oo, w)
    est = np.mean(1.0 / q)
    assert abs(est - 4 * np.pi) < 0.05 * 4 * np.pi
    gfun = 1.0 + w[:, 2] ** 2
    est2 = np.mean(gfun / q)
    assert abs(est2 - 4 * np.pi * (1 + 1 / 3)) < 0.05 * 4 * np.pi * 4 / 3


def test_adam_moves_against_the_gradient():
    p = np.ones(5)
    g = np.array([1.0, -2.0, 0.0, 3.0, -0.5])
    p2, m, v = G.adam(p, np.zeros(5), np.zeros(5), g, 1)
    assert np.all(np.sign(p2 - p) == -np.sign(g))
