"""The guide network on the tensor cores against its FP64 oracle (oracle/guide_ref.py) on the same
FP16-rounded weights: inference outputs, the mixture pdf they define, and one training pass (loss
and weight gradient). The oracle rounds activations and backward signals to FP16 where the GPU
does, so what remains is FP32 accumulation order and rare FP16 rounding-boundary flips."""

import numpy as np
import pytest

import guide_ref as G
from prgpu import guide

pytestmark = pytest.mark.gpu


def _inputs(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1, 1, (n, 3))
    nrm = rng.normal(size=(n, 3))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    wo = rng.normal(size=(n, 3))
    wo /= np.linalg.norm(wo, axis=1, keepdims=True)
    return G.features(x, nrm, wo, [-1, -1, -1], [2, 2, 2])


def _weights(seed):
    p = G.init_params(seed).astype(np.float64)
    rng = np.random.default_rng(seed + 1)
    W = G.split(p)
    # Non-zero biases so every unit is exercised.
    W[0][:, G.CONST_IN] = rng.normal(0, 0.3, W[0].shape[0])
    for l in range(1, 5):
        W[l][:, G.CONST_HID] = rng.normal(0, 0.3, W[l].shape[0])
    for l in range(4):
        W[l][G.CONST_HID, :] = 0
    W[4][41:, :] = 0
    return p.astype(np.float32)


@pytest.mark.parametrize("n", [1, 300, 4096])
def test_inference_matches_fp64_oracle(gpu, n):
    w = _weights(11)
    guide.set_weights(w)
    X = _inputs(n, 12)
    out = guide.infer(X)
    ref, _ = G.forward(w, X, round16=True)
    scale = np.abs(ref).max() + 1.0
    err = np.abs(out - ref)
    assert err.max() <= 1e-2 * scale, (err.max(), scale)
    assert err.mean() <= 1e-3 * scale, (err.mean(), scale)


def test_mixture_pdf_error_against_fp64_evaluation(gpu):
    """The pdf the renderer uses (FP16 network, FP32 decode) against an FP64 evaluation of the same
    weights without FP16 rounding: relative error median < 1%, 99th percentile < 5%."""
    w = _weights(21)
    guide.set_weights(w)
    n = 4096
    X = _inputs(n, 22)
    out = guide.infer(X).astype(np.float64)
    ref, _ = G.forward(w, X, round16=False)
    rng = np.random.default_rng(23)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    q, _ = G.mixture_pdf(out, d)
    qr, _ = G.mixture_pdf(ref, d)
    rel = np.abs(q - qr) / qr
    print(f"guide pdf relative error vs FP64: median {np.median(rel):.2e}, p99 {np.quantile(rel, 0.99):.2e}, "
          f"max {rel.max():.2e}")
    assert np.median(rel) < 1e-2 and np.quantile(rel, 0.99) < 5e-2


@pytest.mark.parametrize("n", [128, 1000])
def test_training_gradient_matches_oracle(gpu, n):
    w = _weights(31)
    guide.set_weights(w)
    X = _inputs(n, 32)
    rng = np.random.default_rng(33)
    wi = rng.normal(size=(n, 3))
    wi /= np.linalg.norm(wi, axis=1, keepdims=True)
    pb = np.abs(wi[:, 2]) / np.pi + 0.02
    wt = rng.exponential(1.0, n)
    loss, g = guide.gradient(X, wi, pb, wt)
    lref, gref = G.backward(w, X, wi.astype(np.float32).astype(np.float64), pb.astype(np.float32).astype(np.float64),
                            wt.astype(np.float32).astype(np.float64), round16=True)
    assert abs(loss - lref * n) <= 1e-3 * abs(lref * n)
    cos = float(g @ gref / (np.linalg.norm(g) * np.linalg.norm(gref)))
    rel = float(np.linalg.norm(g - gref) / np.linalg.norm(gref))
    assert cos > 0.999 and rel < 3e-2, (cos, rel)
    # The constant units' incoming weights get no gradient.
    W = G.split(g.astype(np.float64))
    for l in range(4):
        assert not W[l][G.CONST_HID].any()


@pytest.fixture
def default_guide_options(gpu):
    yield
    guide.set_options()


def test_training_gradient_with_settings_matches_oracle(gpu, default_guide_options):
    """The same pass with non-default settings (selection cap 0.7, log kappa capped at 2, the
    second-moment selection objective) against the oracle with those settings."""
    n = 1000
    w = _weights(41)
    guide.set_weights(w)
    guide.set_options(max_select=0.7, log_kappa_max=2.0, select_loss=1)
    assert guide.get_options() == dict(max_select=pytest.approx(0.7), log_kappa_max=2.0, select_loss=1,
                                       train_passes=1, bands=12, weight_clamp=20.0)
    X = _inputs(n, 42)
    rng = np.random.default_rng(43)
    wi = rng.normal(size=(n, 3))
    wi /= np.linalg.norm(wi, axis=1, keepdims=True)
    pb = np.abs(wi[:, 2]) / np.pi + 0.02
    wt = rng.exponential(1.0, n)
    loss, g = guide.gradient(X, wi, pb, wt)
    f64 = lambda a: np.asarray(a, np.float32).astype(np.float64)  # noqa: E731
    lref, gref = G.backward(w, X, f64(wi), f64(pb), f64(wt), round16=True, max_select=np.float32(0.7),
                            log_kappa_max=2.0, select_loss=1)
    assert abs(loss - lref * n) <= 1e-3 * abs(lref * n)
    cos = float(g @ gref / (np.linalg.norm(g) * np.linalg.norm(gref)))
    rel = float(np.linalg.norm(g - gref) / np.linalg.norm(gref))
    assert cos > 0.999 and rel < 3e-2, (cos, rel)
    # Defaults give a different gradient (the settings reached the kernel).
    guide.set_options()
    _, g0 = guide.gradient(X, wi, pb, wt)
    assert float(np.linalg.norm(g0 - g) / np.linalg.norm(g)) > 0.05


def test_guide_options_are_validated(gpu, default_guide_options):
    from prgpu import abi

    for bad in (dict(max_select=0.0), dict(max_select=1.0), dict(log_kappa_max=9.0), dict(select_loss=2),
                dict(train_passes=0), dict(bands=13), dict(weight_clamp=-1.0)):
        with pytest.raises(abi.PrgpuError, match="out of range"):
            guide.set_options(**bad)
    assert guide.get_options()["max_select"] == pytest.approx(0.5)


def test_adam_steps_reduce_the_training_loss(gpu):
    w = _weights(41)
    guide.set_weights(w)
    n = 2048
    X = _inputs(n, 42)
    rng = np.random.default_rng(43)
    # Incident light concentrated around +z: the guide should learn to point there.
    wi = rng.normal(size=(n, 3)) * 0.3 + np.array([0, 0, 1.0])
    wi /= np.linalg.norm(wi, axis=1, keepdims=True)
    pb = np.full(n, 1 / (4 * np.pi))
    wt = np.ones(n)
    first, _ = guide.gradient(X, wi, pb, wt)
    for _ in range(60):
        loss, _ = guide.gradient(X, wi, pb, wt)
        guide.adam_step(1.0 / n, 5e-3)
    last, _ = guide.gradient(X, wi, pb, wt)
    assert last < first - 0.3 * n, (first / n, last / n)
    w2 = guide.get_weights()
    assert not np.array_equal(w2, w)
