"""Device BxDF, phase-function and homogeneous-medium code against the reference implementations
on identical inputs (pr::DiffuseBxDF / ConductorBxDF / DielectricBxDF / ThinDielectricBxDF,
HenyeyGreenstein, HomogeneousMedium; src/materials/bxdf.cpp, src/media/medium.cpp): every value
within 1e-5 relative (|a - b| <= 1e-5 * max(|a|, |b|)), beside an absolute floor of 1e-5 times the
largest magnitude of that output over the batch for values produced by cancellation."""

import zlib

import numpy as np
import pytest

from prgpu import abi, workloads

pytestmark = pytest.mark.gpu
REL = 1e-5


def _close(a, b, what):
    a = a.astype(np.float64)
    b = b.astype(np.float64)
    scale = np.maximum(np.abs(a).max(axis=0, keepdims=True), 1e-30)
    tol = REL * np.maximum(np.maximum(np.abs(a), np.abs(b)), scale)
    bad = ~(np.abs(a - b) <= tol)
    if bad.any():
        rel = np.abs(a - b) / np.maximum(np.maximum(np.abs(a), np.abs(b)), 1e-30)
        i = np.unravel_index(np.argmax(np.where(bad, rel, 0)), a.shape)
        raise AssertionError(f"{what}: {bad.sum()} of {a.size} values beyond 1e-5; worst at {i}: gpu {a[i]!r} "
                             f"ref {b[i]!r} rel {rel[i]:.3g}")


def _inputs(rng, n):
    x = np.zeros((n, 9), np.float32)
    x[:, 0:3] = workloads.sphere_directions(rng.random((n, 2), dtype=np.float32))
    x[:, 3:6] = workloads.sphere_directions(rng.random((n, 2), dtype=np.float32))
    x[:, 6:9] = rng.random((n, 3), dtype=np.float32)
    return x


PARAMS = {
    "diffuse": (0, [0.2, 0.5, 0.8, 0.9] + [0] * 8 + [1.0, 0.0, 0.0, 0.0]),
    "conductor_rough_aniso": (1, [0] * 4 + [0.17, 0.43, 1.4, 1.66] + [3.5, 2.46, 1.88, 1.96] + [1.0, 0.2, 0.35, 0.0]),
    "conductor_gold_c0": (1, [0] * 4 + [0.25, 0.43, 0.97, 1.4] + [2.98, 2.46, 1.87, 1.88] + [1.0, 0.2, 0.2, 0.0]),
    "conductor_smooth": (1, [0] * 4 + [0.17, 0.43, 1.4, 1.66] + [3.5, 2.46, 1.88, 1.96] + [1.0, 0.0, 0.0, 0.0]),
    "dielectric_rough": (2, [0] * 12 + [1.5168, 0.3, 0.3, 0.0]),
    "dielectric_rough_importance": (2, [0] * 12 + [1.5168, 0.25, 0.4, 1.0]),
    "dielectric_smooth": (2, [0] * 12 + [1.5168, 0.0, 0.0, 0.0]),
    "thin": (3, [0] * 12 + [1.45, 0.0, 0.0, 0.0]),
}


@pytest.mark.parametrize("name", sorted(PARAMS))
def test_bxdf_matches_reference(gpu, oracle, name):
    kind, params = PARAMS[name]
    params = np.array(params, np.float32)
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    x = _inputs(rng, 1 << 16)
    ref = np.zeros((len(x), 16), np.float32)
    oracle.ref_lib().prref_bxdf(kind, oracle._p(params), len(x), oracle._p(x), oracle._p(ref))
    out = np.zeros_like(ref)
    err = abi.err_buf()
    abi.check(gpu.prgpu_eval_bxdf(0, kind, abi.ptr(params), len(x), abi.ptr(x), abi.ptr(out), err, len(err)), err,
              "prgpu_eval_bxdf")
    _close(out[:, 0:4], ref[:, 0:4], f"{name} f")
    _close(out[:, 4:5], ref[:, 4:5], f"{name} pdf")
    # Samples: the same decision (sampled or not, lobe flags) and the same values.
    np.testing.assert_array_equal(out[:, 5], ref[:, 5])
    ok = ref[:, 5] == 1
    np.testing.assert_array_equal(out[ok, 14], ref[ok, 14])
    _close(out[ok, 6:11], ref[ok, 6:11], f"{name} sample f/pdf")
    _close(out[ok, 11:14], ref[ok, 11:14], f"{name} sample wi")
    _close(out[ok, 15:16], ref[ok, 15:16], f"{name} sample eta")


def test_henyey_greenstein_matches_reference(gpu, oracle):
    rng = np.random.default_rng(3)
    n = 1 << 16
    x = np.zeros((n, 7), np.float32)
    x[:, 0] = rng.uniform(-1, 1, n)
    x[:, 1] = rng.choice(np.array([-0.9, -0.3, 0.0, 0.0005, 0.6, 0.8, 0.95], np.float32), n)
    x[:, 2:5] = workloads.sphere_directions(rng.random((n, 2), dtype=np.float32))
    x[:, 5:7] = rng.random((n, 2), dtype=np.float32)
    ref = np.zeros((n, 5), np.float32)
    oracle.ref_lib().prref_hg(n, oracle._p(x), oracle._p(ref))
    out = np.zeros_like(ref)
    err = abi.err_buf()
    abi.check(gpu.prgpu_eval_phase(0, n, abi.ptr(x), abi.ptr(out), err, len(err)), err, "prgpu_eval_phase")
    _close(out[:, 0:1], ref[:, 0:1], "HG value")
    _close(out[:, 4:5], ref[:, 4:5], "HG sample pdf")
    _close(out[:, 1:4], ref[:, 1:4], "HG sample direction")


def test_homogeneous_medium_matches_reference(gpu, oracle):
    rng = np.random.default_rng(4)
    n = 1 << 16
    x = np.zeros((n, 10), np.float32)
    x[:, 0:4] = rng.uniform(0, 0.5, (n, 4))
    x[:, 4:8] = rng.uniform(0, 5, (n, 4))
    x[:, 8] = np.where(rng.random(n) < 0.1, np.inf, rng.uniform(0, 3, n)).astype(np.float32)
    x[:, 9] = rng.random(n, dtype=np.float32)
    ref = np.zeros((n, 14), np.float32)
    oracle.ref_lib().prref_homogeneous(n, None, oracle._p(x), oracle._p(ref))
    out = np.zeros_like(ref)
    err = abi.err_buf()
    abi.check(gpu.prgpu_eval_homogeneous(0, n, abi.ptr(x), abi.ptr(out), err, len(err)), err, "prgpu_eval_homogeneous")
    np.testing.assert_array_equal(out[:, 4], ref[:, 4])
    _close(out[:, 0:4], ref[:, 0:4], "transmittance")
    _close(out[:, 5:6], ref[:, 5:6], "distance")
    _close(out[:, 6:10], ref[:, 6:10], "weight")
    _close(out[:, 10:14], ref[:, 10:14], "pdf ratio")
