"""Per-ray work of the traversal microbenchmark's closest-hit and any-hit passes, the figures of its
roofline: mean BVH nodes visited and triangles tested per ray by the REFERENCE traversal over the
REFERENCE's own tree. MEASUREMENT INFRASTRUCTURE (the oracle): CPU only; the results are frozen
as constants beside the benchmark.

The tree is pr::BVH built by the reference (oracle/_ref/libprref.so, src/geometry/bvh.cpp) over the
benchmark's 1,048,576-triangle soup, exported in the v4 node layout; the counts come from the
oracle's restatement of pr::BVH::Intersect (oracle/restate.c, src/geometry/bvh.cpp:137-232), which
counts what it visits, on the first --rays of the benchmark's closest-hit and any-hit rays (same
seeds, same generator calls). Any other tree the device kernel runs on is credited with this work.

    python oracle/measure_trace_work.py [--rays 262144]
"""

import argparse
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path[:0] = [os.path.join(ROOT, "ar-renderer_b200"), HERE]

import numpy as np  # noqa: E402

import ref  # noqa: E402
from prgpu import abi, workloads  # noqa: E402

N_TRIS = 1 << 20
BENCH_RAYS = 1 << 24


def trace_work(rays_counted: int = 1 << 18) -> dict:
    """Mean nodes visited and triangles tested per ray, closest-hit and any-hit passes, over the
    reference's own tree on the first `rays_counted` rays of each benchmark pass."""
    verts = workloads.triangle_soup(N_TRIS, seed=1)
    rays = workloads.rays_as_f8(workloads.soup_rays(BENCH_RAYS, seed=2)[:rays_counted])
    b = ref.SoupBVH(verts)
    nodes, order = b.export(abi.BVH_NODE)
    rp, rt, _, _, _ = b.trace(rays)
    b.close()
    n = rays.shape[0]
    prim = np.empty(n, np.int32)
    t = np.empty(n, np.float32)
    nv = np.empty(n, np.int32)
    nt = np.empty(n, np.int32)
    lib = ref.restate_lib()
    vp = ref._p(np.ascontiguousarray(verts))
    assert lib.rs_trace(ref._p(nodes), len(nodes), ref._p(order), vp, ref._p(rays), n, 0, ref._p(prim), ref._p(t),
                        ref._p(nv), ref._p(nt)) == 0
    # The counting restatement answers as the reference build does.
    assert (prim == rp).all() and (t[rp >= 0].view(np.int32) == rt[rp >= 0].view(np.int32)).all()
    out = {"tree_nodes": len(nodes), "rays": n, "closest_nodes": float(nv.mean()), "closest_tris": float(nt.mean())}
    # The any-hit pass (tMax uniform in [0, 2]).
    arays = workloads.rays_as_f8(workloads.soup_rays(BENCH_RAYS, seed=3, any_hit=True)[:rays_counted])
    occ = np.empty(n, np.int32)
    assert lib.rs_trace(ref._p(nodes), len(nodes), ref._p(order), vp, ref._p(arays), n, 1, ref._p(occ), None,
                        ref._p(nv), ref._p(nt)) == 0
    out.update(any_nodes=float(nv.mean()), any_tris=float(nt.mean()), any_occluded=float(occ.mean()))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--rays", type=int, default=1 << 18)
    args = ap.parse_args()
    w = trace_work(args.rays)
    cb = 32 * w["closest_nodes"] + 36 * w["closest_tris"] + 32 + 8
    ab = 32 * w["any_nodes"] + 36 * w["any_tris"] + 32 + 4
    print(f"reference BVH ({w['tree_nodes']} nodes), {w['rays']} rays: {w['closest_nodes']:.2f} nodes and "
          f"{w['closest_tris']:.2f} triangles per ray; {cb:.2f} algorithmic bytes per closest-hit ray")
    print(f"any hit: {w['any_nodes']:.2f} nodes and {w['any_tris']:.2f} triangles per ray; {ab:.2f} algorithmic bytes "
          f"per any-hit ray ({w['any_occluded']:.3f} of the rays occluded)")


if __name__ == "__main__":
    main()
