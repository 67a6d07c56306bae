"""Per-path work of the plain path tracer on the box-and-spheres scene (256 x 256, depth 8), the
figures of the path tracer's roofline: N_closest and N_shadow (rays per path sample) and, per ray,
the BVH nodes visited and triangles tested. MEASUREMENT INFRASTRUCTURE (the oracle): run once on a
GPU box, the results are frozen as constants beside the benchmark.

The rays are those the GPU path tracer traces for a seeded 2^16-path subset (wavefront slots
0..65535 of the first chunk: one sample of every pixel), copied out by the library's measurement
tap (SceneExt::rayTap). The node and triangle counts come from the oracle's restatement of the
reference traversal (oracle/restate.c: pr::BVH::Intersect / IntersectP, src/geometry/bvh.cpp:137-232,
which counts what it visits) over the scene's binary BVH in the reference layout, so they are the
reference algorithm's per-ray work on those rays.

    python oracle/measure_path_work.py [out.json]
"""

import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path[:0] = [os.path.join(ROOT, "ar-renderer_b200"), HERE]

import numpy as np  # noqa: E402

import ref  # noqa: E402
from prgpu import hostscene, render, scenes  # noqa: E402

PATHS = 1 << 16
BOUNCES = 16


def main():
    out = sys.argv[1] if len(sys.argv) > 1 else None
    s = scenes.box_scene(seed=0, width=256, height=256, spp=64, max_depth=8)
    h = hostscene.build_box_scene(s)
    desc = h.desc()
    tap = np.zeros((2, BOUNCES, PATHS, 8), np.float32)
    ext = render.make_ext()
    ext.rayTap = tap.ctypes.data
    ext.rayTapPaths = PATHS
    ext.rayTapBounces = BOUNCES
    _, st = render.render_ex(desc, 256, 256, 1, seed=1, max_depth=8, ext=ext, stats=True)
    pa = h.prim_array
    verts = np.ascontiguousarray(np.stack([pa["p0"], pa["p1"], pa["p2"]], axis=1), np.float32)
    nodes = np.ascontiguousarray(h.nodes)
    lib = ref.restate_lib()
    res = {"scene": "box + 35 icospheres, 256x256, depth 8, seed 0", "paths": PATHS,
           "triangles": int(len(pa)), "bvh_nodes": int(len(nodes))}
    for k, name in enumerate(("closest", "shadow")):
        recs = tap[k].reshape(-1, 8)
        recs = recs[recs[:, 7] == 1.0]
        rays = np.zeros((len(recs), 8), np.float32)
        rays[:, 0:3] = recs[:, 0:3]
        rays[:, 3:6] = recs[:, 4:7]
        rays[:, 6] = recs[:, 3]
        n = len(rays)
        prim = np.empty(n, np.int32)
        t = np.empty(n, np.float32)
        nv = np.empty(n, np.int32)
        nt = np.empty(n, np.int32)
        rc = lib.rs_trace(ref._p(nodes.view(np.uint8)), len(nodes), ref._p(h.order), ref._p(verts), ref._p(rays), n,
                          1 if k else 0, ref._p(prim), ref._p(t), ref._p(nv), ref._p(nt))
        assert rc == 0
        res[name] = {"rays_per_path": n / PATHS, "nodes_per_ray": float(nv.mean()), "tris_per_ray": float(nt.mean()),
                     "rays": n}
    # Whole-render ray counts of the GPU's own counters (all 65,536 pixels, 1 spp).
    res["gpu_counters"] = {"closest_per_path": st.closestRays / (256 * 256), "shadow_per_path": st.shadowRays / (256 * 256)}
    c, sh = res["closest"], res["shadow"]
    b_closest = 32 * c["nodes_per_ray"] + 36 * c["tris_per_ray"] + 32 + 8
    b_shadow = 32 * sh["nodes_per_ray"] + 36 * sh["tris_per_ray"] + 32 + 1
    res["bytes_per_closest_ray"] = b_closest
    res["bytes_per_shadow_ray"] = b_shadow
    res["bytes_per_path_sample"] = c["rays_per_path"] * b_closest + sh["rays_per_path"] * b_shadow + 24
    print(json.dumps(res, indent=1))
    if out:
        with open(out, "w") as f:
            json.dump(res, f, indent=1)


if __name__ == "__main__":
    main()
