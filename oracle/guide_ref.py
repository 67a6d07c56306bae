"""CPU oracle (test infrastructure only) for the path-guiding network: an FP64 NumPy restatement of
the network the module evaluates and trains on the GPU. There is no reference implementation: the
reference renderer has no learned component (its PathIntegrator samples the BSDF only,
src/integrators/path.cpp:215-224), so this file is written from the network's definition, and its
own backward pass is pinned by finite differences (tests/test_guide.py).

Network (the module's csrc/guide.cuh): 128 inputs -> 4 hidden ReLU layers of 64 -> 48 outputs;
input 81 and hidden unit 63 are held at 1 (biases folded into the weights). Weights are FP16 on
the GPU with FP32 accumulation and FP16 activations between layers; `round16=True` rounds the
activations (and backward signals) to FP16 at the same points, so the remaining difference is the
FP32 accumulation order.

Outputs, per lobe k < 8: direction (3, normalised), log kappa (clamped to [-4, 8]), weight
logit; output 40 the selection logit, c = 0.5 sigmoid. Mixture pdf of a unit direction w:
q(w) = sum_k pi_k kappa_k / (2 pi (1 - e^{-2 kappa_k})) exp(kappa_k (mu_k . w - 1)).
The renderer folds the mixture onto the hemisphere of the shading normal n that holds the sample:
q_n(w) = q(w) + q(w - 2 (w.n) n). Loss per sample, two parts: -w log q_n(wi) trains the lobes,
-w log(c q_n(wi) + (1 - c) pb) trains the selection output with q_n held fixed (its gradient is
taken as if q_n were a constant).

Settings (prgpu_guide_set_options; the defaults above): the selection cap (c = max_select
sigmoid), the upper clamp of log kappa, and c's objective: select_loss = 1 replaces the selection
term by the surrogate -w w' log(c q_n + (1 - c) pb) with w' = w held fixed, whose derivative in c
is the sample estimate -w^2 (q_n - pb) / p of the derivative of the one-sample estimator's second
moment E[(f Li)^2 / p].
"""

from __future__ import annotations

import numpy as np

IN, HID, OUT, LOBES, BANDS = 128, 64, 48, 8, 12
CONST_IN, CONST_HID = 81, 63
LAYER_IN = [IN, HID, HID, HID, HID]
LAYER_OUT = [HID, HID, HID, HID, OUT]
N_PARAMS = sum(a * b for a, b in zip(LAYER_IN, LAYER_OUT))
MAX_SELECT = 0.5


def split(params: np.ndarray):
    """Flat master weights -> list of [out x in] matrices (views)."""
    out, o = [], 0
    for i, n in zip(LAYER_IN, LAYER_OUT):
        out.append(params[o:o + i * n].reshape(n, i))
        o += i * n
    return out


def init_params(seed: int) -> np.ndarray:
    """He-uniform weights; the constant units' outgoing columns (biases) start at 0, and the rows
    producing the constant hidden unit are 0 (their value is replaced by 1)."""
    rng = np.random.default_rng(seed)
    ws = []
    for l, (i, n) in enumerate(zip(LAYER_IN, LAYER_OUT)):
        lim = np.sqrt(6.0 / (82 if l == 0 else i))
        w = rng.uniform(-lim, lim, (n, i))
        if l == 0:
            w[:, CONST_IN + 1:] = 0.0
            w[:, CONST_IN] = 0.0
        else:
            w[:, CONST_HID] = 0.0
        if l < 4:
            w[CONST_HID, :] = 0.0
        else:
            w[41:, :] = 0.0
        ws.append(w.ravel())
    return np.concatenate(ws).astype(np.float32)


def features(x, n, wo, bmin, bext):
    x = np.asarray(x, np.float64)
    xn = np.clip((x - np.asarray(bmin, np.float64)) / np.asarray(bext, np.float64), 0.0, 1.0)
    f = np.zeros((x.shape[0], IN))
    f[:, 0:3] = xn
    for b in range(BANDS):
        for a in range(3):
            f[:, 3 + 6 * b + 2 * a] = np.sin(np.pi * (2.0 ** b) * xn[:, a])
            f[:, 3 + 6 * b + 2 * a + 1] = np.cos(np.pi * (2.0 ** b) * xn[:, a])
    f[:, 75:78] = n
    f[:, 78:81] = wo
    f[:, CONST_IN] = 1.0
    return f


def _r16(a, on):
    return a.astype(np.float16).astype(np.float64) if on else a


def forward(params, X, round16=True):
    """Returns (outputs (N, 48), cache for backward)."""
    W = [_r16(w.astype(np.float64), round16) for w in split(np.asarray(params, np.float32))]
    A = _r16(np.asarray(X, np.float64), round16)
    acts, zs = [A], []
    for l in range(5):
        Z = A @ W[l].T
        zs.append(Z)
        if l < 4:
            H = np.maximum(Z, 0.0)
            H[:, CONST_HID] = 1.0
            A = _r16(H, round16)
            acts.append(A)
        else:
            A = Z
    return A, (W, acts, zs)


def decode(o, max_select=MAX_SELECT, log_kappa_max=8.0):
    v = o[:, :40].reshape(-1, LOBES, 5)
    d = v[:, :, 0:3]
    l = np.linalg.norm(d, axis=2, keepdims=True)
    mu = np.where(l > 1e-6, d / np.maximum(l, 1e-300), np.array([0.0, 0.0, 1.0]))
    kappa = np.exp(np.clip(v[:, :, 3], -4.0, log_kappa_max))
    a = v[:, :, 4]
    e = np.exp(a - a.max(1, keepdims=True))
    pi = e / e.sum(1, keepdims=True)
    c = max_select / (1.0 + np.exp(-o[:, 40]))
    return mu, kappa, pi, c


def vmf(mu, kappa, w):
    t = np.einsum("nkc,nc->nk", mu, w) - 1.0
    small = kappa < 1e-4
    val = kappa / (2 * np.pi * -np.expm1(-2 * kappa)) * np.exp(kappa * t)
    return np.where(small, 1.0 / (4 * np.pi), val)


def mixture_pdf(o, w):
    mu, kappa, pi, c = decode(o)
    return (pi * vmf(mu, kappa, w)).sum(1), c


def mirror(w, n):
    return w - 2.0 * (w * n).sum(1, keepdims=True) * n


def loss_and_grad_out(o, wi, pb, wgt, n, q_fixed=None, max_select=MAX_SELECT, log_kappa_max=8.0, select_loss=0):
    """Loss per sample and its gradient w.r.t. the 48 outputs (FP64, analytic); n: the shading
    normals (folding planes). The mixture part uses q_fixed when given (the value whose gradient
    is stopped), else the current q_n."""
    o = np.asarray(o, np.float64)
    mu, kappa, pi, c = decode(o, max_select, log_kappa_max)
    wr = mirror(wi, n)
    v1 = vmf(mu, kappa, wi)
    v2 = vmf(mu, kappa, wr)
    vk = v1 + v2
    q = (pi * vk).sum(1)
    qm = q if q_fixed is None else q_fixed
    p = c * qm + (1 - c) * pb
    ok = (p > 0) & (q > 0) & (wgt > 0)
    ps = np.where(ok, p, 1.0)
    qs = np.where(ok, q, 1.0)
    ws = wgt * wgt if select_loss == 1 else wgt  # the selection term's weight
    loss = np.where(ok, -wgt * np.log(qs) - ws * np.log(ps), 0.0)
    dq = np.where(ok, -wgt / qs, 0.0)
    dc = np.where(ok, -ws * (qm - pb) / ps, 0.0)
    g = np.zeros_like(o)
    s = 1.0 / (1.0 + np.exp(-o[:, 40]))
    g[:, 40] = dc * max_select * s * (1 - s)
    gpi = dq[:, None] * vk
    sum_pig = (pi * gpi).sum(1, keepdims=True)
    ga = pi * gpi - pi * sum_pig
    d1 = dq[:, None] * pi * v1
    d2 = dq[:, None] * pi * v2
    raw = o[:, :40].reshape(-1, LOBES, 5)[:, :, 3]
    e = np.exp(-2 * kappa)
    base = 1.0 / kappa - 2 * e / -np.expm1(-2 * kappa)
    t1 = np.einsum("nkc,nc->nk", mu, wi) - 1.0
    t2 = np.einsum("nkc,nc->nk", mu, wr) - 1.0
    gk = np.where((raw > -4) & (raw < log_kappa_max) & (kappa >= 1e-4), (d1 * (base + t1) + d2 * (base + t2)) * kappa,
                  0.0)
    d = o[:, :40].reshape(-1, LOBES, 5)[:, :, 0:3]
    l = np.linalg.norm(d, axis=2, keepdims=True)
    gm = (wi[:, None, :] * d1[:, :, None] + wr[:, None, :] * d2[:, :, None]) * kappa[:, :, None]
    gv = (gm - mu * np.einsum("nkc,nkc->nk", mu, gm)[:, :, None]) / np.maximum(l, 1e-300)
    gv = np.where(l > 1e-6, gv, 0.0)
    G = g[:, :40].reshape(-1, LOBES, 5)
    G[:, :, 0:3] = gv
    G[:, :, 3] = gk
    G[:, :, 4] = ga
    g[:, :40] = G.reshape(-1, 40)
    return loss, g


def mixture_q(o, wi, n, log_kappa_max=8.0):
    """The folded mixture density q_n(wi) (wi on the side of n it was sampled on)."""
    mu, kappa, pi, _ = decode(np.asarray(o, np.float64), log_kappa_max=log_kappa_max)
    return (pi * (vmf(mu, kappa, wi) + vmf(mu, kappa, mirror(wi, n)))).sum(1)


def backward(params, X, wi, pb, wgt, round16=True, n=None, **opts):
    """Mean loss over the batch and the gradient of the SUMMED loss w.r.t. the flat weights
    (n: folding normals, by default the normal inputs X[:, 75:78]; opts: the settings of
    loss_and_grad_out)."""
    out, (W, acts, zs) = forward(params, X, round16)
    if n is None:
        n = np.asarray(X, np.float64)[:, 75:78]
    loss, g = loss_and_grad_out(out, wi, pb, wgt, n, **opts)
    grads = [None] * 5
    dZ = _r16(g, round16)
    for l in range(4, -1, -1):
        grads[l] = dZ.T @ acts[l]
        if l == 0:
            break
        dH = dZ @ W[l]
        dH[:, CONST_HID] = 0.0
        dZ = _r16(dH * (zs[l - 1] > 0), round16)
    return loss.mean(), np.concatenate([gg.ravel() for gg in grads])


def adam(params, m, v, grad, step, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step (in place on float64 copies); returns the new (params, m, v)."""
    m = b1 * m + (1 - b1) * grad
    v = b2 * v + (1 - b2) * grad * grad
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    return params - lr * mh / (np.sqrt(vh) + eps), m, v


def sample(o, u0, u1, u2):
    """Directions drawn from the decoded mixture (the GPU's lobe choice and vMF warp)."""
    mu, kappa, pi, c = decode(o)
    cdf = np.cumsum(pi, 1)
    k = np.minimum((u0[:, None] >= cdf).sum(1), LOBES - 1)
    idx = np.arange(len(k))
    kap = kappa[idx, k]
    m = mu[idx, k]
    ct = np.where(kap < 1e-4, 1 - 2 * u1, 1 + np.log(u1 + (1 - u1) * np.exp(-2 * kap)) / kap)
    ct = np.clip(ct, -1, 1)
    st = np.sqrt(np.maximum(0, 1 - ct * ct))
    phi = 2 * np.pi * u2
    sgn = np.where(m[:, 2] >= 0, 1.0, -1.0)
    a = -1.0 / (sgn + m[:, 2])
    bb = m[:, 0] * m[:, 1] * a
    t = np.stack([1 + sgn * m[:, 0] ** 2 * a, sgn * bb, -sgn * m[:, 0]], 1)
    b = np.stack([bb, sgn + m[:, 1] ** 2 * a, -m[:, 1]], 1)
    return t * (st * np.cos(phi))[:, None] + b * (st * np.sin(phi))[:, None] + m * ct[:, None]
