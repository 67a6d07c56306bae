"""Generates the golden fixtures in this directory from the reference renderer's own code (the
oracle library oracle/_ref/libprref.so, compiled from the reference sources by oracle/Makefile).
Run from the repository root where the reference tree exists:

    make -C oracle && python tests/golden/make_golden.py

traversal.npz  -- a 512-triangle soup, 4096 rays and the reference's closest-hit answers
                  (pr::BVH::Intersect: primitive ids and distance bits).
functions.npz  -- for each BxDF kind (diffuse, conductor, dielectric, thin dielectric): the
                  parameters, 512 input tuples (wo, wi, uc, u0, u1) and the reference outputs
                  (f, pdf and one importance sample), bit for bit.
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "oracle"), os.path.join(ROOT, "ar-renderer_b200")]

import ref  # noqa: E402
from prgpu import workloads  # noqa: E402


def unit_vectors(rng, n, hemi=None):
    u = rng.random((n, 2)).astype(np.float32)
    d = workloads.sphere_directions(u)
    if hemi == "upper":
        d[:, 2] = np.abs(d[:, 2])
    return d


def bxdf_inputs(rng, n):
    x = np.zeros((n, 9), np.float32)
    x[:, 0:3] = unit_vectors(rng, n)
    x[:, 3:6] = unit_vectors(rng, n)
    x[:, 6:9] = rng.random((n, 3)).astype(np.float32)
    return x


def bxdf_params():
    p = []
    # diffuse
    p.append(np.array([0.2, 0.5, 0.8, 0.9] + [0] * 8 + [1.0, 0.0, 0.0, 0.0], np.float32))
    # rough anisotropic conductor (gold-like n, k at 4 wavelengths)
    p.append(np.array([0] * 4 + [0.17, 0.43, 1.4, 1.66] + [3.5, 2.46, 1.88, 1.96] + [1.0, 0.2, 0.35, 0.0], np.float32))
    # rough dielectric
    p.append(np.array([0] * 12 + [1.5168, 0.3, 0.3, 0.0], np.float32))
    # thin dielectric
    p.append(np.array([0] * 12 + [1.45, 0.0, 0.0, 0.0], np.float32))
    return p


def main():
    lib = ref.ref_lib()
    rng = np.random.default_rng(20261203)
    verts = workloads.triangle_soup(512, seed=9)
    rays = workloads.rays_as_f8(workloads.soup_rays(4096, seed=10))
    b = ref.SoupBVH(verts)
    prim, t, _, _, _ = b.trace(rays)
    np.savez_compressed(os.path.join(HERE, "traversal.npz"), verts=verts, rays=rays, prim=prim,
                        t_bits=t.view(np.int32))
    fx = {}
    for kind, params in enumerate(bxdf_params()):
        inp = bxdf_inputs(rng, 512)
        out = np.zeros((inp.shape[0], 16), np.float32)
        lib.prref_bxdf(kind, ref._p(params), inp.shape[0], ref._p(inp), ref._p(out))
        fx[f"params{kind}"] = params
        fx[f"in{kind}"] = inp
        fx[f"out{kind}"] = out
    np.savez_compressed(os.path.join(HERE, "functions.npz"), **fx)
    print("wrote", os.listdir(HERE))


if __name__ == "__main__":
    main()
