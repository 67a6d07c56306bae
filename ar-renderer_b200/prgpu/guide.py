"""The path-guiding network through the C ABI (weights, inference, one training pass, Adam)."""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi

N_PARAMS = 23552
N_IN, N_OUT = 128, 48


def set_weights(w: np.ndarray, device: int = 0) -> None:
    w = np.ascontiguousarray(w, np.float32)
    assert w.size == N_PARAMS
    err = abi.err_buf()
    abi.check(abi.gpu_lib().prgpu_guide_set_weights(device, abi.ptr(w), err, len(err)), err, "prgpu_guide_set_weights")


def get_weights(device: int = 0) -> np.ndarray:
    w = np.zeros(N_PARAMS, np.float32)
    err = abi.err_buf()
    abi.check(abi.gpu_lib().prgpu_guide_get_weights(device, abi.ptr(w), err, len(err)), err, "prgpu_guide_get_weights")
    return w


def infer(features: np.ndarray, device: int = 0) -> np.ndarray:
    f = np.ascontiguousarray(features, np.float32).reshape(-1, N_IN)
    out = np.zeros((f.shape[0], N_OUT), np.float32)
    err = abi.err_buf()
    abi.check(abi.gpu_lib().prgpu_guide_infer(device, f.shape[0], abi.ptr(f), abi.ptr(out), err, len(err)), err,
              "prgpu_guide_infer")
    return out


def gradient(features: np.ndarray, wi: np.ndarray, pb: np.ndarray, w: np.ndarray, n: np.ndarray | None = None,
             device: int = 0):
    """(summed loss, gradient of the summed loss) from one GPU training pass. n: shading normals
    (the folding planes; default: features[:, 75:78])."""
    f = np.ascontiguousarray(features, np.float32).reshape(-1, N_IN)
    if n is None:
        n = f[:, 75:78]
    s = np.ascontiguousarray(np.concatenate([np.asarray(wi, np.float32).reshape(-1, 3),
                                             np.asarray(pb, np.float32).reshape(-1, 1),
                                             np.asarray(w, np.float32).reshape(-1, 1),
                                             np.asarray(n, np.float32).reshape(-1, 3)], 1))
    g = np.zeros(N_PARAMS, np.float32)
    loss = C.c_float(0.0)
    err = abi.err_buf()
    abi.check(abi.gpu_lib().prgpu_guide_gradient(device, f.shape[0], abi.ptr(f), abi.ptr(s), C.byref(loss), abi.ptr(g),
                                                 err, len(err)), err, "prgpu_guide_gradient")
    return float(loss.value), g


def adam_step(grad_scale: float, lr: float = 1e-3, device: int = 0) -> None:
    err = abi.err_buf()
    abi.check(abi.gpu_lib().prgpu_guide_adam_step(device, grad_scale, lr, err, len(err)), err, "prgpu_guide_adam_step")


def stats(device: int = 0) -> dict:
    """Last training pass: summed loss, online batch rows and weight sum, Adam steps taken."""
    out = np.zeros(4, np.float32)
    err = abi.err_buf()
    abi.check(abi.gpu_lib().prgpu_guide_stats(device, abi.ptr(out), err, len(err)), err, "prgpu_guide_stats")
    return {"loss_sum": float(out[0]), "rows": int(out[1]), "weight_sum": float(out[2]), "steps": int(out[3])}


def set_learning_rate(lr: float, device: int = 0) -> None:
    err = abi.err_buf()
    abi.check(abi.gpu_lib().prgpu_guide_set_learning_rate(device, lr, err, len(err)), err,
              "prgpu_guide_set_learning_rate")


DEFAULT_OPTIONS = dict(max_select=0.5, log_kappa_max=8.0, select_loss=0, train_passes=1, bands=12, weight_clamp=20.0)


def set_options(max_select: float = 0.5, log_kappa_max: float = 8.0, select_loss: int = 0, train_passes: int = 1,
                bands: int = 12, weight_clamp: float = 20.0, device: int = 0) -> None:
    """Sampling and training settings of the guide (prgpu_guide_set_options): the cap of the
    selection probability c, the cap of log kappa, c's objective (0 KL, 1 second moment of the
    one-sample estimator), the online training passes over each chunk's samples, the position
    encoding bands in use and the clamp of the batch-normalised training weights (0 off)."""
    o = abi.GuideOptions(max_select, log_kappa_max, select_loss, train_passes, bands, weight_clamp)
    err = abi.err_buf()
    abi.check(abi.gpu_lib().prgpu_guide_set_options(device, C.byref(o), err, len(err)), err, "prgpu_guide_set_options")


def get_options(device: int = 0) -> dict:
    o = abi.GuideOptions()
    err = abi.err_buf()
    abi.check(abi.gpu_lib().prgpu_guide_get_options(device, C.byref(o), err, len(err)), err, "prgpu_guide_get_options")
    return dict(max_select=o.maxSelect, log_kappa_max=o.logKappaMax, select_loss=o.selectLoss,
                train_passes=o.trainPasses, bands=o.bands, weight_clamp=o.weightClamp)
