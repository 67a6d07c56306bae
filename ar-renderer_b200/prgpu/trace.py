"""Ray queries through the C ABI: BVH construction (libprender_host.so) and closest-hit / any-hit
traversal on the GPU (libprender_gpu.so: prgpu_trace_rays, prgpu_accel_*)."""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi


def build_bvh_triangles(verts: np.ndarray, max_leaf: int = 4, threads: int = 0):
    """Binned-SAH BVH over a triangle soup. verts: (n, 3, 3) float32. Returns (nodes, primOrder)."""
    verts = np.ascontiguousarray(verts, dtype=np.float32).reshape(-1, 3, 3)
    n = verts.shape[0]
    nodes = np.zeros(max(1, 2 * n - 1), dtype=abi.BVH_NODE)
    order = np.zeros(max(1, n), dtype=np.int32)
    cnt = abi.host_lib().prhost_build_bvh_triangles(abi.ptr(verts), n, max_leaf, threads, abi.ptr(nodes),
                                                    abi.ptr(order))
    if cnt < 0:
        raise abi.PrgpuError("prhost_build_bvh_triangles rejected its arguments")
    return nodes[:cnt].copy(), order[:n].copy()


def build_bvh_bounds(bmin: np.ndarray, bmax: np.ndarray, max_leaf: int = 4, threads: int = 0):
    """Binned-SAH BVH over primitive bounds ((n, 3) float32 each). Returns (nodes, primOrder)."""
    bmin = np.ascontiguousarray(bmin, dtype=np.float32)
    bmax = np.ascontiguousarray(bmax, dtype=np.float32)
    n = bmin.shape[0]
    nodes = np.zeros(max(1, 2 * n - 1), dtype=abi.BVH_NODE)
    order = np.zeros(max(1, n), dtype=np.int32)
    cnt = abi.host_lib().prhost_build_bvh(abi.ptr(bmin), abi.ptr(bmax), n, max_leaf, threads, abi.ptr(nodes),
                                          abi.ptr(order))
    if cnt < 0:
        raise abi.PrgpuError("prhost_build_bvh rejected its arguments")
    return nodes[:cnt].copy(), order[:n].copy()


def make_rays(o: np.ndarray, d: np.ndarray, tmax) -> np.ndarray:
    r = np.zeros(o.shape[0], dtype=abi.RAY)
    r["o"] = o
    r["d"] = d
    r["tMax"] = tmax
    return r


def trace_rays(nodes, order, verts, rays, any_hit=False, device=0, barycentrics=False):
    """One-shot query with host buffers (prgpu_trace_rays). Returns prim (and t, b1, b2)."""
    lib = abi.gpu_lib()
    verts = np.ascontiguousarray(verts, dtype=np.float32).reshape(-1, 3, 3)
    n = rays.shape[0]
    prim = np.empty(n, dtype=np.int32)
    t = None if any_hit else np.empty(n, dtype=np.float32)
    b1 = np.empty(n, dtype=np.float32) if barycentrics and not any_hit else None
    b2 = np.empty(n, dtype=np.float32) if barycentrics and not any_hit else None
    err = abi.err_buf()
    rc = lib.prgpu_trace_rays(device, abi.ptr(nodes), len(nodes), abi.ptr(order), abi.ptr(verts), verts.shape[0],
                              abi.ptr(rays), n, 1 if any_hit else 0, abi.ptr(prim), abi.ptr(t), abi.ptr(b1),
                              abi.ptr(b2), err, len(err))
    abi.check(rc, err, "prgpu_trace_rays")
    if any_hit:
        return prim
    return (prim, t, b1, b2) if barycentrics else (prim, t)


class Accel:
    """Device-resident BVH for repeated queries (prgpu_accel_*)."""

    def __init__(self, nodes, order, verts, device=0):
        self.lib = abi.gpu_lib()
        verts = np.ascontiguousarray(verts, dtype=np.float32).reshape(-1, 3, 3)
        h = C.c_void_p()
        err = abi.err_buf()
        rc = self.lib.prgpu_accel_create(device, abi.ptr(nodes), len(nodes), abi.ptr(order), abi.ptr(verts),
                                         verts.shape[0], C.byref(h), err, len(err))
        abi.check(rc, err, "prgpu_accel_create")
        self.handle = h

    @property
    def nbytes(self) -> int:
        return int(self.lib.prgpu_accel_bytes(self.handle))

    def trace_device(self, rays_ptr: int, n: int, prim_ptr: int, t_ptr: int | None, any_hit: bool,
                     stream: int = 0) -> None:
        """Queue a query on `stream` with device pointers (no synchronisation)."""
        err = abi.err_buf()
        rc = self.lib.prgpu_accel_trace(self.handle, C.c_void_p(rays_ptr), n, 1 if any_hit else 0,
                                        C.c_void_p(prim_ptr), C.c_void_p(t_ptr) if t_ptr else None,
                                        C.c_void_p(stream), err, len(err))
        abi.check(rc, err, "prgpu_accel_trace")

    def trace_host(self, rays: np.ndarray, prim: np.ndarray, t: np.ndarray | None, any_hit: bool) -> None:
        err = abi.err_buf()
        rc = self.lib.prgpu_accel_trace_host(self.handle, abi.ptr(rays), rays.shape[0], 1 if any_hit else 0,
                                             abi.ptr(prim), abi.ptr(t), err, len(err))
        abi.check(rc, err, "prgpu_accel_trace_host")

    def status(self) -> int:
        return int(self.lib.prgpu_accel_status(self.handle))

    def close(self) -> None:
        if self.handle:
            self.lib.prgpu_accel_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
