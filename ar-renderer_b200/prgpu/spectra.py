"""Spectral tables for scenes built without PRender's loader: 95 samples at 5 nm from 360 nm (the
SceneDesc spectrum format, src/gpu/gpu_api.h:19-21).

* blackbody(T): Planck's law normalised to unit CIE Y (the "temperature" emitters).
* sellmeier(B, C): refractive index n(lambda) from Sellmeier coefficients (lambda in um).
* metal_nk(name): conductor n, k for Au / Ag / Cu / Al (coarse tables, see below).
* rgb_albedo(rgb): a smooth reflectance with the given linear-sRGB colour: the sigmoid-of-quadratic
  spectrum of Jakob & Hanika (2019), fitted directly for this colour by Gauss-Newton on the CIELab
  difference under a 6504 K blackbody illuminant (a stand-in for D65; the reference fits against
  tabulated D65 and interpolates from a 64^3 table, so its spectra differ slightly).
"""

from __future__ import annotations

import numpy as np

LAMBDA = 360.0 + 5.0 * np.arange(95)
_FINE = np.linspace(360.0, 830.0, 471)  # 1 nm, integration grid


def _g(x, mu, s1, s2):
    t = (x - mu) / np.where(x < mu, s1, s2)
    return np.exp(-0.5 * t * t)


def cie_xyz(lam):
    """Wyman-Sloan-Shirley multi-lobe fit of the CIE 1931 2-degree observer (JCGT 2013)."""
    x = 1.056 * _g(lam, 599.8, 37.9, 31.0) + 0.362 * _g(lam, 442.0, 16.0, 26.7) - 0.065 * _g(lam, 501.1, 20.4, 26.2)
    y = 0.821 * _g(lam, 568.8, 46.9, 40.5) + 0.286 * _g(lam, 530.9, 16.3, 31.1)
    z = 1.217 * _g(lam, 437.0, 11.8, 36.0) + 0.681 * _g(lam, 459.0, 26.0, 13.8)
    return np.stack([x, y, z])


def cie_y_integral() -> float:
    """Sum of y over integer wavelengths 360..830 nm (the film's normalisation constant)."""
    return float(np.sum(cie_xyz(np.arange(360, 831, dtype=np.float64))[1]))


def planck(lam_nm, T):
    c, h, kb = 299792458.0, 6.62606957e-34, 1.3806488e-23
    l = lam_nm * 1e-9
    return (2 * h * c * c) / (l ** 5 * (np.exp((h * c) / (l * kb * T)) - 1))


def blackbody(T: float) -> np.ndarray:
    """Planck spectrum normalised to unit luminance Y (1 nm Riemann sum over 360-830 nm)."""
    s = planck(_FINE, T)
    y = np.sum(s * cie_xyz(_FINE)[1]) / cie_y_integral()
    return (planck(LAMBDA, T) / y).astype(np.float32)


def sellmeier(B, C) -> np.ndarray:
    l2 = (LAMBDA * 1e-3) ** 2
    n2 = 1.0 + sum(b * l2 / (l2 - c) for b, c in zip(B, C))
    return np.sqrt(np.maximum(n2, 1.0)).astype(np.float32)


BK7 = ((1.03961212, 0.231792344, 1.01046945), (0.00600069867, 0.0200179144, 103.560653))  # Schott N-BK7

# Metal optical constants sampled every 50 nm over the visible range (the values PRender ships as
# its named metals, after Johnson & Christy 1972 and Rakic 1995; src/core/spectrum.cpp:171-188).
_METAL_L = np.array([360, 400, 450, 500, 550, 600, 650, 700, 750, 830], np.float64)
_METALS = {
    "Au": ([1.72, 1.66, 1.40, 0.97, 0.43, 0.25, 0.17, 0.16, 0.16, 0.17],
           [1.92, 1.96, 1.88, 1.87, 2.46, 2.98, 3.50, 3.95, 4.40, 5.10]),
    "Cu": ([1.26, 1.18, 1.17, 1.13, 1.03, 0.27, 0.21, 0.21, 0.23, 0.27],
           [2.30, 2.40, 2.53, 2.56, 2.58, 3.24, 3.67, 4.18, 4.60, 5.20]),
    "Ag": ([0.07, 0.05, 0.04, 0.05, 0.06, 0.06, 0.07, 0.08, 0.09, 0.10],
           [1.60, 2.10, 2.66, 3.13, 3.59, 4.00, 4.44, 4.80, 5.20, 5.80]),
    "Al": ([0.40, 0.49, 0.62, 0.77, 0.96, 1.20, 1.47, 1.83, 2.40, 2.70],
           [4.35, 4.86, 5.47, 6.08, 6.69, 7.26, 7.79, 8.31, 8.62, 8.30]),
}


def metal_nk(name: str):
    n, k = _METALS[name]
    return (np.interp(LAMBDA, _METAL_L, n).astype(np.float32), np.interp(LAMBDA, _METAL_L, k).astype(np.float32))


_SRGB_TO_XYZ = np.array([[0.4124564, 0.3575761, 0.1804375], [0.2126729, 0.7151522, 0.0721750],
                         [0.0193339, 0.1191920, 0.9503041]])


def _lab(xyz, white):
    def f(v):
        d = 6.0 / 29.0
        return np.where(v > d ** 3, np.cbrt(v), v / (3 * d * d) + 4.0 / 29.0)

    fx, fy, fz = f(xyz[0] / white[0]), f(xyz[1] / white[1]), f(xyz[2] / white[2])
    return np.array([116 * fy - 16, 500 * (fx - fy), 200 * (fy - fz)])


def _sigmoid(x):
    return 0.5 + x / (2.0 * np.sqrt(1.0 + x * x))


def _fit_tables():
    illum = planck(_FINE, 6504.0)
    cmf = cie_xyz(_FINE)
    w = illum * cmf  # (3, n)
    w = w / np.sum(illum * cmf[1])  # a unit reflector has Y = 1
    white = w.sum(axis=1)
    return w, white


_W, _WHITE = _fit_tables()


def _spectrum_xyz(coeffs, lam=_FINE):
    t = (lam - 360.0) / 470.0
    return _sigmoid(coeffs[0] * t * t + coeffs[1] * t + coeffs[2])


def fit_rgb(rgb) -> np.ndarray:
    """Sigmoid-polynomial coefficients (in normalised wavelength) reproducing a linear-sRGB albedo."""
    rgb = np.clip(np.asarray(rgb, np.float64), 0.0, 1.0)
    target = _lab(_SRGB_TO_XYZ @ rgb * _WHITE / (_SRGB_TO_XYZ @ np.ones(3)), _WHITE)
    c = np.zeros(3)
    for _ in range(40):
        def resid(cc):
            xyz = _W @ _spectrum_xyz(cc)
            return target - _lab(xyz, _WHITE)

        r = resid(c)
        J = np.zeros((3, 3))
        for i in range(3):
            e = np.zeros(3)
            e[i] = 1e-5
            J[:, i] = (resid(c + e) - resid(c - e)) / 2e-5
        try:
            step = np.linalg.solve(J, r)
        except np.linalg.LinAlgError:
            break
        c = c - step
        m = np.max(np.abs(c))
        if m > 200:
            c *= 200 / m
        if np.dot(r, r) < 1e-10:
            break
    return c


def rgb_albedo(rgb) -> np.ndarray:
    return _spectrum_xyz(fit_rgb(rgb), LAMBDA).astype(np.float32)


def constant(v: float) -> np.ndarray:
    return np.full(95, v, np.float32)


def preetham_sky(sun_dir, turbidity: float = 3.0, ground_albedo: float = 0.3, width: int = 512,
                 height: int = 256) -> np.ndarray:
    """The Preetham sky map (height, width, 3) linear sRGB from the host library
    (prhost_preetham_sky, the daylight PRender builds for a sun_sky light)."""
    from . import abi

    d = np.ascontiguousarray(sun_dir, np.float32)
    out = np.zeros((height, width, 3), np.float32)
    assert abi.host_lib().prhost_preetham_sky(abi.ptr(d), turbidity, ground_albedo, width, height, abi.ptr(out)) == 0
    return out


def sun_radiance(sun_dir, turbidity: float = 3.0, radius_deg: float = 0.2665, lam: np.ndarray = LAMBDA) -> np.ndarray:
    """The sun's spectral radiance at wavelengths lam (prhost_sun_radiance)."""
    from . import abi

    d = np.ascontiguousarray(sun_dir, np.float32)
    lam = np.ascontiguousarray(lam, np.float32)
    out = np.zeros(lam.shape, np.float32)
    assert abi.host_lib().prhost_sun_radiance(abi.ptr(d), turbidity, radius_deg, lam.size, abi.ptr(lam),
                                              abi.ptr(out)) == 0
    return out


def rgb_to_sigmoid(rgb: np.ndarray, illuminant: np.ndarray) -> np.ndarray:
    """Environment-map texels (n, 4) = (c0, c1, c2, scale) of unbounded RGBs (prhost_rgb_to_sigmoid)
    fitted under the given 95-sample illuminant."""
    from . import abi

    rgb = np.ascontiguousarray(rgb, np.float32).reshape(-1, 3)
    ill = np.ascontiguousarray(illuminant, np.float32)
    assert ill.size == 95
    out = np.zeros((rgb.shape[0], 4), np.float32)
    assert abi.host_lib().prhost_rgb_to_sigmoid(rgb.shape[0], abi.ptr(rgb), abi.ptr(ill), 0, abi.ptr(out)) == 0
    return out
