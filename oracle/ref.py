"""ctypes access to the oracle: the reference renderer's own CPU code (oracle/_ref/libprref.so,
built by oracle/Makefile from the reference sources plus oracle/ref_harness.cpp) and the plain-C
restatement (oracle/_ref/librestate.so, oracle/restate.c).

TEST INFRASTRUCTURE ONLY. tests/, __graft_entry__.smoke() and bench.py's CPU-baseline /
reference arm use it as the checker or as the timed CPU reference; the product never imports it.
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
REF_LIB = os.path.join(REF_DIR, "libprref.so")
RESTATE_LIB = os.path.join(REF_DIR, "librestate.so")

_P = C.c_void_p
_ref = None
_restate = None


def available() -> bool:
    return os.path.exists(REF_LIB)


def ref_lib() -> C.CDLL:
    global _ref
    if _ref is None:
        if not os.path.exists(REF_LIB):
            raise RuntimeError(f"{REF_LIB} missing: build it with `make -C oracle` where the reference tree exists")
        lib = C.CDLL(REF_LIB)
        lib.prref_set_threads.argtypes = [C.c_int]
        lib.prref_thread_count.restype = C.c_int
        lib.prref_set_cache_dir.argtypes = [C.c_char_p]
        lib.prref_soup_new.argtypes = [_P, C.c_int64]
        lib.prref_soup_new.restype = _P
        lib.prref_soup_free.argtypes = [_P]
        lib.prref_soup_node_count.argtypes = [_P]
        lib.prref_soup_node_count.restype = C.c_int64
        lib.prref_soup_export.argtypes = [_P, _P, _P]
        lib.prref_soup_trace.argtypes = [_P, _P, C.c_int64, C.c_int, _P, _P, _P, _P]
        lib.prref_soup_trace.restype = C.c_double
        lib.prref_bxdf.argtypes = [C.c_int, _P, C.c_int64, _P, _P]
        lib.prref_full_bsdf.argtypes = [_P, C.c_int64, _P, _P]
        lib.prref_sheen_table.argtypes = [_P]
        lib.prref_render_aov.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_uint64, C.c_int, _P]
        lib.prref_aov_matrices.argtypes = [_P, _P]
        lib.prref_checkpoint_write.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint64, C.c_uint64,
                                               _P, C.c_int32, C.c_char_p, C.c_int]
        lib.prref_checkpoint_read.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint64, C.c_uint64,
                                              _P, C.POINTER(C.c_int32), C.c_char_p, C.c_int]
        lib.prref_fr_dielectric.argtypes = [C.c_float, C.c_float]
        lib.prref_fr_dielectric.restype = C.c_float
        lib.prref_fr_complex.argtypes = [C.c_float, C.c_float, C.c_float]
        lib.prref_fr_complex.restype = C.c_float
        lib.prref_hg.argtypes = [C.c_int64, _P, _P]
        lib.prref_homogeneous.argtypes = [C.c_int64, _P, _P, _P]
        lib.prref_sample_visible.argtypes = [C.c_int64, _P, _P, _P]
        lib.prref_cie.argtypes = [C.c_int64, _P, _P]
        lib.prref_cie_y_integral.restype = C.c_float
        lib.prref_spectrum.argtypes = [C.c_int, C.c_float, C.c_float, C.c_float, C.c_char_p, C.c_int64, _P, _P]
        lib.prref_spectrum.restype = C.c_int
        lib.prref_scene_load.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_char_p, C.c_int]
        lib.prref_scene_load.restype = _P
        lib.prref_scene_free.argtypes = [_P]
        lib.prref_scene_prim_count.argtypes = [_P]
        lib.prref_scene_prim_count.restype = C.c_int64
        lib.prref_scene_width.argtypes = [_P]
        lib.prref_scene_height.argtypes = [_P]
        lib.prref_scene_export.argtypes = [_P, C.c_char_p, C.c_int]
        lib.prref_scene_export.restype = _P
        lib.prref_render.argtypes = [_P, C.c_int, C.c_uint64, C.c_int, C.c_int, _P, C.c_char_p, C.c_int]
        lib.prref_render.restype = C.c_double
        lib.prref_light_bvh_sample.argtypes = [_P, C.c_int64, _P, _P, _P]
        lib.prref_scene_light_count.argtypes = [_P]
        lib.prref_scene_infinite.argtypes = [_P, C.c_int, _P, _P]
        lib.prref_rgb_uplift.argtypes = [C.c_int64, _P, _P]
        lib.prref_preetham_sky.argtypes = [_P, C.c_float, C.c_float, C.c_int, C.c_int, _P]
        lib.prref_sun_radiance.argtypes = [_P, C.c_float, C.c_float, C.c_int64, _P, _P]
        lib.prref_scene_grid_count.argtypes = [_P]
        lib.prref_scene_grid_info.argtypes = [_P, C.c_int, C.c_char_p, C.c_int, _P]
        lib.prref_scene_grid_density.argtypes = [_P, C.c_int, C.c_int64, _P, _P]
        lib.prref_write_fog_sphere.argtypes = [C.c_char_p, C.c_double, C.c_double, C.c_double]
        # The RGB->spectrum table is built once (a few seconds) and cached beside the library.
        lib.prref_set_cache_dir(REF_DIR.encode())
        _ref = lib
    return _ref


def restate_lib() -> C.CDLL:
    global _restate
    if _restate is None:
        if not os.path.exists(RESTATE_LIB):
            raise RuntimeError(f"{RESTATE_LIB} missing: run `make -C oracle restate`")
        lib = C.CDLL(RESTATE_LIB)
        lib.rs_trace.argtypes = [_P, C.c_int64, _P, _P, _P, C.c_int64, C.c_int, _P, _P, _P, _P]
        lib.rs_trace.restype = C.c_int
        _restate = lib
    return _restate


def _p(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


class SoupBVH:
    """The reference pr::BVH built over a triangle soup ((n, 3, 3) float32)."""

    def __init__(self, verts: np.ndarray):
        self.lib = ref_lib()
        self.verts = np.ascontiguousarray(verts, dtype=np.float32).reshape(-1, 3, 3)
        self.h = self.lib.prref_soup_new(_p(self.verts), self.verts.shape[0])

    def export(self, node_dtype):
        n = self.lib.prref_soup_node_count(self.h)
        nodes = np.zeros(n, dtype=node_dtype)
        order = np.zeros(self.verts.shape[0], dtype=np.int32)
        self.lib.prref_soup_export(self.h, _p(nodes), _p(order))
        return nodes, order

    def trace(self, rays: np.ndarray, any_hit=False):
        """rays: (n, 8) float32 (o, d, tmax, pad). Returns prim, t, b1, b2 (closest) or occluded flags,
        and the elapsed seconds."""
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        n = rays.shape[0]
        prim = np.empty(n, dtype=np.int32)
        if any_hit:
            dt = self.lib.prref_soup_trace(self.h, _p(rays), n, 1, _p(prim), None, None, None)
            return prim, dt
        t = np.empty(n, dtype=np.float32)
        b1 = np.empty(n, dtype=np.float32)
        b2 = np.empty(n, dtype=np.float32)
        dt = self.lib.prref_soup_trace(self.h, _p(rays), n, 0, _p(prim), _p(t), _p(b1), _p(b2))
        return prim, t, b1, b2, dt

    def close(self):
        if self.h:
            self.lib.prref_soup_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class RefScene:
    """A scene loaded by the reference loader (LoadScene), exportable as the v4 SceneDesc its host
    would hand the GPU module, and renderable with the reference PathIntegrator."""

    def __init__(self, path: str, width: int = 0, height: int = 0):
        self.lib = ref_lib()
        err = C.create_string_buffer(2048)
        self.h = self.lib.prref_scene_load(path.encode(), width, height, err, len(err))
        if not self.h:
            raise RuntimeError("reference LoadScene failed: " + err.value.decode())
        self.width = self.lib.prref_scene_width(self.h)
        self.height = self.lib.prref_scene_height(self.h)
        self._desc = None

    def export(self) -> int:
        """Address of the exported prgpu::SceneDesc (valid while this object lives)."""
        if self._desc is None:
            err = C.create_string_buffer(2048)
            p = self.lib.prref_scene_export(self.h, err, len(err))
            if not p:
                raise RuntimeError("scene export failed: " + err.value.decode())
            self.warnings = err.value.decode()
            self._desc = p
        return self._desc

    def render(self, spp: int, seed: int, max_depth: int, light_bvh: bool = True):
        """Per-pixel XYZ sums over spp samples, shape (h, w, 3), and the render seconds."""
        out = np.zeros((self.height, self.width, 3), dtype=np.float32)
        err = C.create_string_buffer(2048)
        dt = self.lib.prref_render(self.h, spp, seed, max_depth, 1 if light_bvh else 0, _p(out), err, len(err))
        if dt < 0:
            raise RuntimeError("reference render failed: " + err.value.decode())
        return out, dt

    def light_count(self) -> int:
        return self.lib.prref_scene_light_count(self.h)

    def render_aov(self, kind: int, spp: int, seed: int, through_specular: bool) -> np.ndarray:
        """pr::RenderAOV: (height, width, 3) float32 (kind 0 albedo, 1 normal, 2 depth, 3 position)."""
        out = np.zeros((self.height, self.width, 3), np.float32)
        self.lib.prref_render_aov(self.h, kind, spp, seed, 1 if through_specular else 0, _p(out))
        return out

    def infinite_lights(self):
        """(type, pmf) of the exported lights outside the v4 table, in scene order: image environment
        (2), sun (3), spot (4), distant (5), goniometric (6)."""
        self.export()
        t = np.zeros(64, np.int32)
        p = np.zeros(64, np.float32)
        n = self.lib.prref_scene_infinite(self.h, 64, _p(t), _p(p))
        return [(int(t[i]), float(p[i])) for i in range(min(n, 64))]

    def grid_density(self, k: int, pts: np.ndarray) -> np.ndarray:
        """Density of grid medium k's field at medium-space points (n, 3)."""
        pts = np.ascontiguousarray(pts, dtype=np.float32).reshape(-1, 3)
        out = np.zeros(len(pts), np.float32)
        self.export()
        if self.lib.prref_scene_grid_density(self.h, k, len(pts), _p(pts), _p(out)) != 0:
            raise RuntimeError("no grid medium %d" % k)
        return out

    def grid_media(self):
        """Heterogeneous media of the export, in index order (index = mediumCount + k): a list of
        (name, bounds (2, 3) float32 in medium space as the loader fitted them)."""
        self.export()
        out = []
        for k in range(self.lib.prref_scene_grid_count(self.h)):
            name = C.create_string_buffer(256)
            b = np.zeros(6, dtype=np.float32)
            if self.lib.prref_scene_grid_info(self.h, k, name, len(name), _p(b)) != 0:
                raise RuntimeError("grid medium %d is not a voxel grid" % k)
            out.append((name.value.decode(), b.reshape(2, 3)))
        return out

    def light_bvh_sample(self, pts: np.ndarray, with_pmf: bool = True):
        """pts: (n, 7) float32 (p, n, u). Returns (light index, pmf) and the per-light PMF table."""
        pts = np.ascontiguousarray(pts, dtype=np.float32)
        out = np.zeros((pts.shape[0], 2), dtype=np.float32)
        pm = np.zeros((pts.shape[0], self.light_count()), dtype=np.float32) if with_pmf else None
        self.lib.prref_light_bvh_sample(self.h, pts.shape[0], _p(pts), _p(out), _p(pm))
        return out, pm

    def close(self):
        if self.h:
            self.lib.prref_scene_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def set_threads(n: int) -> None:
    ref_lib().prref_set_threads(n)


def thread_count() -> int:
    return ref_lib().prref_thread_count()


def rgb_uplift(rgb: np.ndarray) -> np.ndarray:
    """(n, 4) sigmoid-polynomial coefficients (c0, c1, c2, scale) of unbounded RGB values, as the
    reference's RGB-to-spectrum table gives them."""
    rgb = np.ascontiguousarray(rgb, np.float32).reshape(-1, 3)
    out = np.zeros((rgb.shape[0], 4), np.float32)
    ref_lib().prref_rgb_uplift(rgb.shape[0], _p(rgb), _p(out))
    return out


def preetham_sky(sun_dir, turbidity: float, ground_albedo: float, width: int, height: int) -> np.ndarray:
    d = np.ascontiguousarray(sun_dir, np.float32)
    out = np.zeros((height, width, 3), np.float32)
    ref_lib().prref_preetham_sky(_p(d), turbidity, ground_albedo, width, height, _p(out))
    return out


def sun_radiance(sun_dir, turbidity: float, radius_deg: float, lam: np.ndarray) -> np.ndarray:
    d = np.ascontiguousarray(sun_dir, np.float32)
    lam = np.ascontiguousarray(lam, np.float32)
    out = np.zeros(lam.shape[0], np.float32)
    ref_lib().prref_sun_radiance(_p(d), turbidity, radius_deg, lam.shape[0], _p(lam), _p(out))
    return out


def write_fog_sphere(path: str, radius: float, voxel_size: float, half_width: float = 3.0) -> str:
    """A NanoVDB fog-volume sphere (grid "density", centred at the origin, index -> world = index x
    voxel_size) written with NanoVDB's own tools, as the reference's tests make one."""
    if ref_lib().prref_write_fog_sphere(path.encode(), radius, voxel_size, half_width) != 0:
        raise RuntimeError("cannot write " + path)
    return path
