"""Spot, distant and goniometric (IES) lights on the GPU against the reference PathIntegrator
(SpotLight, DistantLight, GoniometricLight + IESProfile: src/lights/light.cpp:161-192,
src/lights/sky.cpp:12-63, src/lights/ies.cpp:23-109): an outdoor scene lit only by those three,
from one scene file. The reference loads and exports the scene; its three lights reach the module
as SceneExt delta lights built from the scene file with the reference sampler's pmfs."""

import ctypes as C
import json
import math
import os
import tempfile

import numpy as np
import pytest

import render_util as ru
from prgpu import abi, render, spectra

pytestmark = pytest.mark.gpu

# A type C photometric file: rotationally symmetric candela falling off towards the horizon, with
# a second horizontal plane so that the phi interpolation runs too.
IES = """IESNA:LM-63-2002
[TEST] synthetic downlight
TILT=NONE
1 1000 1 6 2 1 1 0 0 0
1 1 100
0 15 30 45 60 90
0 90
1000 950 700 400 150 0
1000 900 600 300 100 0
"""


def _scene(path, ies_path, w, h):
    doc = {
        "materials": {"ground": {"type": "diffuse", "reflectance": [0.6, 0.6, 0.6]},
                      "red": {"type": "diffuse", "reflectance": [0.7, 0.2, 0.15]},
                      "gold": {"type": "conductor", "metal": "Au", "roughness": 0.3}},
        "media": {},
        "geometry": {"ground": {"type": "mesh", "positions": [-6, 0, -6, -6, 0, 6, 6, 0, 6, 6, 0, -6],
                                "indices": [0, 1, 2, 0, 2, 3]},
                     "s0": {"type": "sphere", "center": [-0.8, 0.5, 0], "radius": 0.5},
                     "s1": {"type": "sphere", "center": [0.8, 0.5, 0.2], "radius": 0.5}},
        "objects": [{"name": "ground", "geometry": "ground", "material": "ground"},
                    {"name": "s0", "geometry": "s0", "material": "red"},
                    {"name": "s1", "geometry": "s1", "material": "gold"}],
        "lights": {"a_spot": {"type": "spot", "position": [-1.5, 3.0, 1.5], "look_at": [-0.5, 0.0, 0.0],
                              "cone_angle": 35.0, "falloff_start": 20.0, "intensity": 6.0, "temperature": 3500},
                   "b_sun": {"type": "distant", "direction": [0.4, -1.0, -0.3], "irradiance": 0.8,
                             "temperature": 6500},
                   "c_ies": {"type": "point", "position": [1.2, 2.2, 0.8], "ies": ies_path,
                             "direction": [0.1, -1.0, 0.0], "rotation": 30.0, "intensity": 4.0,
                             "temperature": 2700}},
        "cameras": {"cam": {"type": "pinhole", "position": [0, 1.6, 4.0], "look_at": [0, 0.4, 0], "fov_y": 45}},
        "render": {"camera": "cam", "seed": 0, "film": {"width": w, "height": h, "filter": "box"},
                   "integrator": {"type": "path", "spp": 16, "max_depth": 6}},
    }
    with open(path, "w") as f:
        json.dump(doc, f)
    return doc


def _frame_from_z(z):
    sign = math.copysign(1.0, z[2])
    a = -1.0 / (sign + z[2])
    b = z[0] * z[1] * a
    x = np.array([1 + sign * z[0] * z[0] * a, sign * b, -sign * z[0]])
    y = np.array([b, sign + z[1] * z[1] * a, -z[1]])
    return x, y


def _ies_profile(text):
    """(vAngles, hAngles, candela / peak) of a type C LM-63 file (the layout IESProfile::Parse
    reads, ies.cpp:23-76)."""
    nums = [float(v) for v in text.split("TILT=NONE", 1)[1].split()]
    n_v, n_h = int(nums[3]), int(nums[4])
    multiplier, ballast = nums[2], nums[10]
    rest = nums[13:]
    va, ha = rest[:n_v], rest[n_v:n_v + n_h]
    cd = np.maximum(0.0, np.array(rest[n_v + n_h:n_v + n_h + n_v * n_h]) * multiplier * ballast)
    return np.array(va, np.float32), np.array(ha, np.float32), (cd / cd.max()).astype(np.float32)


def _gpu_inputs(rs, doc):
    import ref as oracle_ref

    base = abi.SceneDesc.from_address(rs.export())
    sd = abi.SceneDesc()
    C.memmove(C.addressof(sd), C.addressof(base), C.sizeof(sd))
    old = np.ctypeslib.as_array((C.c_float * (95 * base.spectrumCount)).from_address(base.spectra)).reshape(-1, 95)
    lam = spectra.LAMBDA.astype(np.float32)
    names = sorted(doc["lights"])
    rows = []
    for name in names:
        out = np.zeros(95, np.float32)
        assert oracle_ref.ref_lib().prref_spectrum(3, float(doc["lights"][name]["temperature"]), 0, 0, None, 95,
                                                   oracle_ref._p(lam), oracle_ref._p(out)) == 0
        rows.append(out)
    table = np.ascontiguousarray(np.concatenate([old, np.stack(rows)]), np.float32)
    sd.spectra = table.ctypes.data
    sd.spectrumCount = table.shape[0]
    pmfs = rs.infinite_lights()
    assert [t for t, _ in pmfs] == [4, 5, 6], pmfs
    descs, keep = [], [table]
    for k, name in enumerate(names):
        l = doc["lights"][name]
        d = abi.DeltaLightDesc()
        d.spectrum = base.spectrumCount + k
        d.pmf = pmfs[k][1]
        if l["type"] == "spot":
            p, tgt = np.array(l["position"]), np.array(l["look_at"])
            ax = (tgt - p) / np.linalg.norm(tgt - p)
            d.type = abi.DELTA_SPOT
            d.scale = l["intensity"]
            d.position[:] = [float(v) for v in p]
            d.direction[:] = [float(v) for v in ax]
            d.cosFalloffEnd = math.cos(math.radians(l["cone_angle"]))
            d.cosFalloffStart = math.cos(math.radians(min(l["falloff_start"], l["cone_angle"])))
        elif l["type"] == "distant":
            dv = np.array(l["direction"], np.float64)
            d.type = abi.DELTA_DISTANT
            d.scale = l["irradiance"]
            d.direction[:] = [float(v) for v in -dv / np.linalg.norm(dv)]
        else:
            va, ha, cd = _ies_profile(IES)
            prof = np.ascontiguousarray(np.concatenate([va, ha, cd]), np.float32)
            keep.append(prof)
            z = np.array(l["direction"], np.float64)
            z /= np.linalg.norm(z)
            fx, fy = _frame_from_z(z)
            rot = math.radians(l["rotation"])
            x = fx * math.cos(rot) + fy * math.sin(rot)
            x -= z * np.dot(x, z)
            x /= np.linalg.norm(x)
            y = np.cross(z, x)
            d.type = abi.DELTA_GONIOMETRIC
            d.scale = l["intensity"]
            d.position[:] = [float(v) for v in l["position"]]
            d.frame[:] = [float(v) for v in np.concatenate([x, y, z])]
            d.nV, d.nH = len(va), len(ha)
            d.profile = prof.ctypes.data
        descs.append(d)
    ext = render.make_ext(delta_lights=descs)
    ext._keep += keep
    sd._keep = table
    return sd, ext


def test_spot_distant_and_ies_lights_agree_with_reference(gpu, oracle):
    """48 x 32, depth 6: per-pixel z of the mean over 16 renders of 256 spp each side, |z| < 4 on
    >= 99.5 % of values; mean luminance within 4 standard errors."""
    w, h = 48, 32
    d = os.path.join(tempfile.gettempdir(), "prb_scenes")
    os.makedirs(d, exist_ok=True)
    ies_path = os.path.join(d, "downlight.ies")
    with open(ies_path, "w") as f:
        f.write(IES)
    path = os.path.join(d, "delta_lights.prscene.json")
    doc = _scene(path, ies_path, w, h)
    rs = oracle.RefScene(path)
    sd, ext = _gpu_inputs(rs, doc)
    g = np.stack([render.render_ex(sd, w, h, 256, seed=1000 + k, max_depth=6, ext=ext) / 256 for k in range(16)])
    c = np.stack([rs.render(256, 2000 + k, 6)[0].astype(np.float64) / 256 for k in range(16)])
    z = ru.z_scores(g, c)
    frac = np.mean(np.abs(z) < 4)
    mg, mc = g[..., 1].mean(axis=(1, 2)), c[..., 1].mean(axis=(1, 2))
    se = np.sqrt(mg.var(ddof=1) / len(mg) + mc.var(ddof=1) / len(mc))
    print(f"delta lights: frac {frac:.4f}, mean Y gpu {mg.mean():.5f} cpu {mc.mean():.5f} se {se:.5f}")
    assert mc.mean() > 0
    assert frac >= 0.995, f"only {frac:.4f} of values within |z| < 4"
    assert abs(mg.mean() - mc.mean()) < 4 * se, f"mean Y gpu {mg.mean()} cpu {mc.mean()} (se {se})"
