"""prgpu_trace_rays_noalloc: the ray query for callers that cannot allocate device memory while
they work (their HBM is held by another allocator's pool, or a cudaMalloc / cudaFree with its
device-wide synchronisation is not allowed at that point). It takes all its device memory from a
fixed array the library reserves per GPU, so it must give exactly what prgpu_trace_rays gives --
on two calls in a row, since the second call finds the first call's data still in that array.

This file is named to be collected last: run alone in a fresh process or after every other test,
the results must be the same."""

import ctypes

import numpy as np
import pytest

from prgpu import abi, trace, workloads

pytestmark = pytest.mark.gpu


def _noalloc(nodes, order, verts, rays, any_hit=False):
    lib = abi.gpu_lib()
    verts = np.ascontiguousarray(verts, dtype=np.float32).reshape(-1, 3, 3)
    n = len(rays)
    prim = np.full(n, -7, np.int32)
    t = None if any_hit else np.full(n, -7.0, np.float32)
    b1 = None if any_hit else np.full(n, -7.0, np.float32)
    b2 = None if any_hit else np.full(n, -7.0, np.float32)
    err = abi.err_buf()
    rc = lib.prgpu_trace_rays_noalloc(0, abi.ptr(nodes), len(nodes), abi.ptr(order), abi.ptr(verts), verts.shape[0],
                                      abi.ptr(rays), n, 1 if any_hit else 0, abi.ptr(prim), abi.ptr(t), abi.ptr(b1),
                                      abi.ptr(b2), err, len(err))
    abi.check(rc, err, "prgpu_trace_rays_noalloc")
    return prim if any_hit else (prim, t, b1, b2)


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.int32)


def test_noalloc_matches_allocating_entry_point_twice_in_a_row(gpu):
    # First call: a 100,000-triangle soup, 600,000 rays (three passes through the staging area).
    v1 = workloads.triangle_soup(100_000, seed=31)
    n1, o1 = trace.build_bvh_triangles(v1)
    r1 = workloads.soup_rays(600_000, seed=32)
    want = trace.trace_rays(n1, o1, v1, r1, barycentrics=True)
    got = _noalloc(n1, o1, v1, r1)
    np.testing.assert_array_equal(got[0], want[0])
    hit = want[0] >= 0
    assert hit.sum() > 1000
    for g, w in zip(got[1:], want[1:]):
        np.testing.assert_array_equal(_bits(g[hit]), _bits(w[hit]))
    # Second call right after, on a smaller scene: the first call's nodes and rays are still in
    # the array and must not leak into this answer.
    v2 = workloads.triangle_soup(5_000, seed=33)
    n2, o2 = trace.build_bvh_triangles(v2)
    r2 = workloads.soup_rays(70_000, seed=34, any_hit=True)
    want_occ = trace.trace_rays(n2, o2, v2, r2, any_hit=True)
    np.testing.assert_array_equal(_noalloc(n2, o2, v2, r2, any_hit=True), want_occ)
    r3 = workloads.soup_rays(70_000, seed=35)
    wp, wt = trace.trace_rays(n2, o2, v2, r3)
    gp, gt, _, _ = _noalloc(n2, o2, v2, r3)
    np.testing.assert_array_equal(gp, wp)
    np.testing.assert_array_equal(_bits(gt[wp >= 0]), _bits(wt[wp >= 0]))


def _device_free_bytes() -> int:
    """Free device memory as the driver reports it for the context current on this thread (the
    primary context the library made current), through libcuda's cuMemGetInfo."""
    cu = ctypes.CDLL("libcuda.so.1")
    free, total = ctypes.c_size_t(), ctypes.c_size_t()
    assert cu.cuMemGetInfo_v2(ctypes.byref(free), ctypes.byref(total)) == 0
    return free.value


def test_noalloc_calls_after_the_first_leave_device_memory_untouched(gpu):
    # The first call of each kernel variant may do the runtime's one-time set-up (symbol address,
    # lazy module load, local-memory reserve); every later call must allocate nothing.
    v = workloads.triangle_soup(20_000, seed=41)
    nodes, order = trace.build_bvh_triangles(v)
    rc = workloads.soup_rays(300_000, seed=42)
    ra = workloads.soup_rays(300_000, seed=43, any_hit=True)
    first = _noalloc(nodes, order, v, rc)
    first_occ = _noalloc(nodes, order, v, ra, any_hit=True)
    free0 = _device_free_bytes()
    again = _noalloc(nodes, order, v, rc)
    again_occ = _noalloc(nodes, order, v, ra, any_hit=True)
    free1 = _device_free_bytes()
    assert free1 == free0, f"device free memory changed by {free1 - free0} bytes across two calls"
    np.testing.assert_array_equal(again[0], first[0])
    np.testing.assert_array_equal(_bits(again[1]), _bits(first[1]))
    np.testing.assert_array_equal(again_occ, first_occ)


def test_noalloc_rejects_scenes_beyond_its_limit(gpu):
    v = workloads.triangle_soup(131_073, seed=36)
    nodes = np.zeros(1, dtype=abi.BVH_NODE)
    nodes[0]["nPrims"] = 1
    order = np.arange(len(v), dtype=np.int32)
    rays = workloads.soup_rays(16)
    with pytest.raises(abi.PrgpuError, match="at most 131072 triangles"):
        _noalloc(nodes, order, v, rays)
