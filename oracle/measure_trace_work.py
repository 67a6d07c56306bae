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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--rays", type=int, default=1 << 18)
    args = ap.parse_args()
    verts = workloads.triangle_soup(N_TRIS, seed=1)
    rays = workloads.rays_as_f8(workloads.soup_rays(BENCH_RAYS, seed=2)[: args.rays])
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
    assert lib.rs_trace(ref._p(nodes), len(nodes), ref._p(order), ref._p(np.ascontiguousarray(verts)), ref._p(rays), n,
                        0, ref._p(prim), ref._p(t), ref._p(nv), ref._p(nt)) == 0
    # The counting restatement answers as the reference build does.
    assert (prim == rp).all() and (t[rp >= 0].view(np.int32) == rt[rp >= 0].view(np.int32)).all()
    nodes_per_ray, tris_per_ray = float(nv.mean()), float(nt.mean())
    bytes_per_ray = 32 * nodes_per_ray + 36 * tris_per_ray + 32 + 8
    print(f"reference BVH ({len(nodes)} nodes), {n} rays: {nodes_per_ray:.2f} nodes and {tris_per_ray:.2f} triangles "
          f"per ray; {bytes_per_ray:.2f} algorithmic bytes per closest-hit ray")
    # The any-hit pass (tMax uniform in [0, 2]): the same counts, 4 bytes of flag out.
    arays = workloads.rays_as_f8(workloads.soup_rays(BENCH_RAYS, seed=3, any_hit=True)[: args.rays])
    occ = np.empty(n, np.int32)
    assert lib.rs_trace(ref._p(nodes), len(nodes), ref._p(order), ref._p(np.ascontiguousarray(verts)), ref._p(arays), n,
                        1, ref._p(occ), None, ref._p(nv), ref._p(nt)) == 0
    an, at = float(nv.mean()), float(nt.mean())
    print(f"any hit: {an:.2f} nodes and {at:.2f} triangles per ray; {32 * an + 36 * at + 32 + 4:.2f} algorithmic bytes "
          f"per any-hit ray ({occ.mean():.3f} of the rays occluded)")


if __name__ == "__main__":
    main()
