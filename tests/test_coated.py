"""Host side of coated and sheen materials: the scene exporter hands coats and sheen to the
module with the reference loader's parameters (the layout the reference's own host fills,
src/integrators/gpu_path.cpp:200-256), and the reference oracle's sheen albedo table is sane."""

import ctypes as C

import numpy as np

from prgpu import abi


def test_exporter_carries_coats_and_sheen(oracle):
    import test_coated_gpu as tc

    rs = oracle.RefScene(tc._coated_scene_file("coated_box_cpu", seed=3, width=16, height=16, subdiv=1))
    sd = abi.SceneDesc.from_address(rs.export())
    mats = np.ctypeslib.as_array((C.c_uint8 * (sd.materialCount * abi.MATERIAL.itemsize)).from_address(sd.materials))
    m = mats.view(abi.MATERIAL)
    types = set(int(t) for t in m["type"])
    assert {abi.MAT_COATED_DIFFUSE, abi.MAT_COATED_CONDUCTOR} <= types
    coated = m[m["type"] == abi.MAT_COATED_DIFFUSE]
    assert (coated["coatEta"] >= 0).all() and (coated["coatMaxDepth"] == 64).all() and (coated["coatSamples"] == 1).all()
    assert np.isclose(sorted(coated["thickness"]), [0.01, 0.01, 0.2]).all()
    assert (coated["coatAlbedo"] >= 0).sum() == 1
    sheen = m[m["sheenWeight"] > 0]
    assert len(sheen) == 2 and (sheen["sheenColor"] >= 0).all()
    assert sd.sheenAlbedo


def test_host_sheen_table_matches_reference(oracle):
    """The module's own sheen albedo table (for hosts that pass none) equals the reference's
    SheenBxDF::Albedo at the nodes (same stratified integration, float rounding apart)."""
    t = np.zeros(16 * 32, np.float32)
    oracle.ref_lib().prref_sheen_table(oracle._p(t))
    mine = np.zeros(16 * 32, np.float32)
    abi.gpu_lib().prgpu_sheen_albedo_table(abi.ptr(mine))
    np.testing.assert_allclose(mine, t, rtol=2e-4, atol=1e-6)
    t = t.reshape(16, 32)
    assert (t >= 0).all() and np.isfinite(t).all()
    assert t[-1, 0] > t[-1, -1]  # rough sheen reflects more at grazing angles
