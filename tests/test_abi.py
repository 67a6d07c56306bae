"""The C-ABI boundary without a GPU: both libraries load and export exactly the entry points the
headers declare, the v4 structs keep the byte layout of the reference's gpu_api.h, and the host
BVH builders produce valid trees that answer ray queries like the reference BVH."""

import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from prgpu import abi, trace, workloads

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header: str, macro: str) -> set:
    text = open(os.path.join(ROOT, "include", header)).read()
    return set(re.findall(macro + r"\s+[\w\s\*:]+?\b(\w+)\s*\(", text))


def _exported(lib: str) -> set:
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True).stdout
    return {l.split()[-1] for l in out.splitlines() if " T " in l}


def test_gpu_library_exports_exactly_the_declared_entry_points():
    abi.gpu_lib()
    declared = _declared("prgpu_api.h", "PRGPU_API")
    assert {"prgpu_api_version", "prgpu_list_devices", "prgpu_render"} <= declared
    assert _exported(abi.GPU_LIB_PATH) == declared


def test_host_library_exports_exactly_the_declared_entry_points():
    abi.host_lib()
    assert _exported(abi.HOST_LIB_PATH) == _declared("prhost_api.h", "PRHOST_API")


def test_versions_without_a_device():
    lib = abi.gpu_lib()
    assert lib.prgpu_api_version() == 4
    assert lib.prgpu_ext_version() == 5
    buf = (abi.DeviceInfo * 4)()
    assert lib.prgpu_list_devices(C.cast(buf, C.c_void_p), 4) >= 0


def test_struct_layouts_match_reference_header():
    assert abi.BVH_NODE.itemsize == 32 and abi.PRIMITIVE.itemsize == 128 and abi.MATERIAL.itemsize == 88
    assert abi.LIGHT.itemsize == 48 and abi.MEDIUM.itemsize == 16 and abi.SPECTRUM.itemsize == 380
    assert C.sizeof(abi.SceneDesc) == 520 and abi.SceneDesc.cieYIntegral.offset == 512


def test_render_rejects_bad_input_without_a_device():
    lib = abi.gpu_lib()
    sd = abi.SceneDesc()
    sd.apiVersion = 3
    rp = abi.RenderParams(1, 0, 0, 8, 0.0)
    out = np.zeros(3, np.float32)
    err = abi.err_buf()
    rc = lib.prgpu_render(0, C.cast(C.pointer(sd), C.c_void_p), C.cast(C.pointer(rp), C.c_void_p), abi.ptr(out), err,
                          len(err))
    assert rc == 1 and b"version" in err.value


def _check_tree(nodes, order, n):
    seen = np.zeros(n, np.int32)
    stack = [0]
    while stack:
        i = stack.pop()
        nd = nodes[i]
        if nd["nPrims"] == 0:
            for c in (i + 1, int(nd["offset"])):
                assert c > i and c < len(nodes)
                ch = nodes[c]
                assert (ch["bmin"] >= nd["bmin"]).all() and (ch["bmax"] <= nd["bmax"]).all()
                stack.append(c)
        else:
            seen[order[nd["offset"]:nd["offset"] + nd["nPrims"]]] += 1
    assert (seen == 1).all()


@pytest.mark.parametrize("n", [1, 2, 5, 1000, 50000])
def test_host_bvh_is_valid(n):
    verts = workloads.triangle_soup(n, seed=n)
    nodes, order = trace.build_bvh_triangles(verts, max_leaf=4)
    assert len(nodes) <= 2 * n - 1
    assert sorted(order.tolist()) == list(range(n))
    _check_tree(nodes, order, n)
    lo, hi = verts.min(axis=(0, 1)), verts.max(axis=(0, 1))
    np.testing.assert_array_equal(nodes[0]["bmin"], lo)
    np.testing.assert_array_equal(nodes[0]["bmax"], hi)


def test_host_bvh_answers_like_reference(oracle):
    verts = workloads.triangle_soup(1 << 13, seed=3)
    rays = workloads.rays_as_f8(workloads.soup_rays(1 << 14, seed=4))
    b = oracle.SoupBVH(verts)
    rp, rt, _, _, _ = b.trace(rays)
    nodes, order = trace.build_bvh_triangles(verts)
    lib = oracle.restate_lib()
    p = np.empty(len(rays), np.int32)
    t = np.empty(len(rays), np.float32)
    lib.rs_trace(oracle._p(nodes), len(nodes), oracle._p(order), oracle._p(verts), oracle._p(rays), len(rays), 0,
                 oracle._p(p), oracle._p(t), None, None)
    np.testing.assert_array_equal(p >= 0, rp >= 0)
    np.testing.assert_array_equal(t[rp >= 0].view(np.int32), rt[rp >= 0].view(np.int32))
    assert (p != rp).sum() <= 1  # only exact distance ties may differ


def test_light_bvh_builder_structure():
    rng = np.random.default_rng(5)
    n = 48
    lb = np.zeros((n, 13), np.float32)
    c = rng.uniform(-1, 1, (n, 3)).astype(np.float32)
    lb[:, 0:3] = c - 0.05
    lb[:, 3:6] = c + 0.05
    lb[:, 6:9] = [0, -1, 0]
    lb[:, 9] = rng.uniform(0.5, 2, n)
    lb[:, 10] = 1.0
    lb[:, 11] = 0.0
    nodes = np.zeros(2 * n - 1, dtype=abi.LIGHT_BVH_NODE)
    cnt = abi.host_lib().prhost_build_light_bvh(abi.ptr(lb), n, abi.ptr(nodes))
    assert cnt == 2 * n - 1
    leaves = nodes[nodes["light"] >= 0]
    assert sorted(leaves["light"].tolist()) == list(range(n))
    assert nodes[0]["parent"] == -1 and abs(nodes[0]["phi"] - lb[:, 9].sum()) < 1e-3 * lb[:, 9].sum()
    for i, nd in enumerate(nodes):
        if nd["light"] < 0:
            assert nodes[i + 1]["parent"] == i and nodes[nd["child1"]]["parent"] == i
