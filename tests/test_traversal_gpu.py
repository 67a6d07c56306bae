"""GPU parity of the ray-query path (prgpu_trace_rays / prgpu_accel_*) against the oracle: the
reference's own pr::BVH::Intersect / IntersectP (src/geometry/bvh.cpp:158-232) run on the same
rays over the same BVH. Closest-hit primitive IDs, distances and barycentrics must be bit-exact;
any-hit flags must be identical."""

import numpy as np
import pytest

from prgpu import abi, trace, workloads

pytestmark = pytest.mark.gpu


def _ref_closest(oracle, verts, rays):
    b = oracle.SoupBVH(verts)
    prim, t, b1, b2, _ = b.trace(workloads.rays_as_f8(rays))
    nodes, order = b.export(abi.BVH_NODE)
    b.close()
    return nodes, order, prim, t, b1, b2


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.int32)


@pytest.mark.parametrize("ntris,nrays", [(1 << 12, 1 << 16), (1 << 16, 1 << 18)])
def test_closest_hit_bit_exact_on_reference_bvh(gpu, oracle, ntris, nrays):
    verts = workloads.triangle_soup(ntris, seed=1)
    rays = workloads.soup_rays(nrays, seed=2)
    nodes, order, rp, rt, rb1, rb2 = _ref_closest(oracle, verts, rays)
    gp, gt, gb1, gb2 = trace.trace_rays(nodes, order, verts, rays, barycentrics=True)
    assert (rp >= 0).sum() > 100
    np.testing.assert_array_equal(gp, rp)
    hit = rp >= 0
    np.testing.assert_array_equal(_bits(gt[hit]), _bits(rt[hit]))
    np.testing.assert_array_equal(_bits(gb1[hit]), _bits(rb1[hit]))
    np.testing.assert_array_equal(_bits(gb2[hit]), _bits(rb2[hit]))


def test_any_hit_identical_on_reference_bvh(gpu, oracle):
    verts = workloads.triangle_soup(1 << 15, seed=3)
    rays = workloads.soup_rays(1 << 18, seed=4, any_hit=True)
    b = oracle.SoupBVH(verts)
    ref_occ, _ = b.trace(workloads.rays_as_f8(rays), any_hit=True)
    nodes, order = b.export(abi.BVH_NODE)
    occ = trace.trace_rays(nodes, order, verts, rays, any_hit=True)
    assert 0 < ref_occ.sum() < len(ref_occ)
    np.testing.assert_array_equal(occ, ref_occ)


def test_full_size_soup_bit_exact(gpu, oracle):
    """The full 1,048,576-triangle soup; 2^21 of the benchmark's rays are checked against the
    reference (its CPU traversal of all 2^24 takes minutes), closest and any-hit."""
    verts = workloads.triangle_soup(1 << 20, seed=1)
    rays = workloads.soup_rays(1 << 21, seed=2)
    nodes, order, rp, rt, _, _ = _ref_closest(oracle, verts, rays)
    gp, gt = trace.trace_rays(nodes, order, verts, rays)
    np.testing.assert_array_equal(gp, rp)
    np.testing.assert_array_equal(_bits(gt[rp >= 0]), _bits(rt[rp >= 0]))
    arays = workloads.soup_rays(1 << 20, seed=5, any_hit=True)
    b = oracle.SoupBVH(verts)
    ref_occ, _ = b.trace(workloads.rays_as_f8(arays), any_hit=True)
    b.close()
    np.testing.assert_array_equal(trace.trace_rays(nodes, order, verts, arays, any_hit=True), ref_occ)


def test_own_bvh_agrees_except_exact_ties(gpu, oracle):
    """With this library's own SAH BVH the tree differs, so only exact distance ties may resolve
    to a different primitive (the reference keeps the first one it visits)."""
    verts = workloads.triangle_soup(1 << 16, seed=7)
    rays = workloads.soup_rays(1 << 18, seed=8)
    _, _, rp, rt, _, _ = _ref_closest(oracle, verts, rays)
    nodes, order = trace.build_bvh_triangles(verts, max_leaf=4)
    gp, gt = trace.trace_rays(nodes, order, verts, rays)
    np.testing.assert_array_equal(gp >= 0, rp >= 0)
    diff = gp != rp
    assert diff.sum() <= 2
    np.testing.assert_array_equal(_bits(gt[rp >= 0]), _bits(rt[rp >= 0]))


def test_edge_cases_match_reference(gpu, oracle):
    rng = np.random.default_rng(11)
    verts = workloads.triangle_soup(64, seed=12)
    # Degenerate triangles (zero area, coincident vertices) and an axis-aligned one.
    verts[0] = verts[0, 0]
    verts[1, 2] = verts[1, 1]
    verts[2] = np.array([[0.2, 0.2, 0.5], [0.8, 0.2, 0.5], [0.2, 0.8, 0.5]], np.float32)
    n = 4096
    r = np.zeros(n, dtype=abi.RAY)
    r["o"] = rng.uniform(-0.5, 1.5, (n, 3)).astype(np.float32)
    d = workloads.sphere_directions(rng.random((n, 2), dtype=np.float32))
    # Direction components exactly zero (infinite reciprocals, NaN slab products) and axis rays.
    d[:512, 0] = 0
    d[512:1024, 1:] = 0
    d[1024:1536] = [0, 0, -1]
    r["o"][1024:1536, :2] = rng.uniform(0.15, 0.85, (512, 2))
    r["d"] = d
    r["tMax"] = np.float32(np.inf)
    r["tMax"][1536:1800] = 0.0
    nodes, order, rp, rt, _, _ = _ref_closest(oracle, verts, r)
    gp, gt = trace.trace_rays(nodes, order, verts, r)
    np.testing.assert_array_equal(gp, rp)
    np.testing.assert_array_equal(_bits(gt[rp >= 0]), _bits(rt[rp >= 0]))
    assert (rp[1536:1800] == -1).all()


def test_single_triangle_and_empty_bvh(gpu, oracle):
    verts = np.array([[[0, 0, 0], [1, 0, 0], [0, 1, 0]]], np.float32)
    rays = np.zeros(3, dtype=abi.RAY)
    rays["o"] = [[0.2, 0.2, 1], [0.9, 0.9, 1], [0.2, 0.2, -1]]
    rays["d"] = [[0, 0, -1], [0, 0, -1], [0, 0, 1]]
    rays["tMax"] = np.inf
    nodes, order, rp, rt, _, _ = _ref_closest(oracle, verts, rays)
    assert len(nodes) == 1 and nodes[0]["nPrims"] == 1
    gp, gt = trace.trace_rays(nodes, order, verts, rays)
    np.testing.assert_array_equal(gp, [0, -1, 0])
    np.testing.assert_array_equal(gp, rp)
    empty = np.zeros(0, dtype=abi.BVH_NODE)
    gp, _ = trace.trace_rays(empty, np.zeros(0, np.int32), np.zeros((0, 3, 3), np.float32), rays)
    np.testing.assert_array_equal(gp, [-1, -1, -1])


def test_malformed_bvh_is_rejected(gpu):
    verts = workloads.triangle_soup(8)
    nodes, order = trace.build_bvh_triangles(verts)
    rays = workloads.soup_rays(16)
    bad = nodes.copy()
    bad[0]["offset"] = 0  # an interior node pointing at itself would loop
    with pytest.raises(abi.PrgpuError, match="malformed"):
        trace.trace_rays(bad, order, verts, rays)
    bad_order = order.copy()
    bad_order[0] = 1 << 20
    with pytest.raises(abi.PrgpuError, match="out of range"):
        trace.trace_rays(nodes, bad_order, verts, rays)


def test_device_resident_path_matches_host_path(gpu):
    import torch

    verts = workloads.triangle_soup(1 << 15, seed=21)
    nodes, order = trace.build_bvh_triangles(verts)
    rays = workloads.soup_rays(1 << 17, seed=22)
    hp, ht = trace.trace_rays(nodes, order, verts, rays)
    acc = trace.Accel(nodes, order, verts)
    dr = torch.from_numpy(rays.view(np.uint8).copy()).cuda()
    dp = torch.empty(len(rays), dtype=torch.int32, device="cuda")
    dt = torch.empty(len(rays), dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    acc.trace_device(dr.data_ptr(), len(rays), dp.data_ptr(), dt.data_ptr(), any_hit=False, stream=stream)
    torch.cuda.synchronize()
    assert acc.status() == 0
    np.testing.assert_array_equal(dp.cpu().numpy(), hp)
    np.testing.assert_array_equal(_bits(dt.cpu().numpy()[hp >= 0]), _bits(ht[hp >= 0]))
    prim = np.empty(len(rays), np.int32)
    t = np.empty(len(rays), np.float32)
    acc.trace_host(rays, prim, t, any_hit=False)
    np.testing.assert_array_equal(prim, hp)
    acc.close()


def test_wide_tree_matches_reference(gpu, oracle):
    """The accel path traverses the 4-wide collapse of the tree (nearest child first); hits carry
    the reference's primitive and distance bits, except possibly at exactly equal distances (the
    visit order differs from the reference's), closest and any hit, on the full-size soup."""
    verts = workloads.triangle_soup(1 << 20, seed=1)
    rays = workloads.soup_rays(1 << 21, seed=2)
    nodes, order, rp, rt, _, _ = _ref_closest(oracle, verts, rays)
    acc = trace.Accel(nodes, order, verts)
    prim = np.empty(len(rays), np.int32)
    t = np.empty(len(rays), np.float32)
    acc.trace_host(rays, prim, t, any_hit=False)
    assert acc.status() == 0
    np.testing.assert_array_equal(prim >= 0, rp >= 0)
    assert (prim != rp).sum() <= 2
    np.testing.assert_array_equal(_bits(t[rp >= 0]), _bits(rt[rp >= 0]))
    arays = workloads.soup_rays(1 << 20, seed=5, any_hit=True)
    b = oracle.SoupBVH(verts)
    ref_occ, _ = b.trace(workloads.rays_as_f8(arays), any_hit=True)
    b.close()
    occ = np.empty(len(arays), np.int32)
    acc.trace_host(arays, occ, None, any_hit=True)
    np.testing.assert_array_equal(occ, ref_occ)
    acc.close()
