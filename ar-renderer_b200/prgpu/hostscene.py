"""A SceneDesc built directly from scene data, without PRender's loader -- what a host that is not
PRender does to drive the module: flatten geometry into Primitive records, tabulate spectra, build
the BVH and light BVH with libprender_host.so, and fill the camera, filter and light tables.

build_box_scene() produces the box-and-spheres family of prgpu.scenes with the same geometry and
camera the JSON form gives the reference loader (spectra from prgpu.spectra).
"""

from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import abi, scenes, spectra, trace


class HostScene:
    def __init__(self):
        self.prims = []  # per-mesh Primitive arrays
        self._prim_count = 0
        self.materials = []
        self.lights = []
        self.spectra = []
        self.media = []
        self.camera = abi.Camera()
        self.filter = abi.Filter()
        self.camera_medium = -1
        self.env_spectrum = -1
        self.env_scale = 0.0
        self._desc = None

    # -- tables ---------------------------------------------------------------------------
    def spectrum(self, values) -> int:
        self.spectra.append(np.asarray(values, np.float32))
        return len(self.spectra) - 1

    def material(self, **kw) -> int:
        m = np.zeros(1, abi.MATERIAL)[0]
        for k in ("albedo", "albedoB", "eta", "k", "coatEta", "coatAlbedo", "sheenColor"):
            m[k] = -1
        for k, v in kw.items():
            m[k] = v
        self.materials.append(m)
        return len(self.materials) - 1

    def medium(self, sigma_a, sigma_s, g, scale=1.0) -> int:
        m = np.zeros(1, abi.MEDIUM)[0]
        m["sigmaA"] = self.spectrum(sigma_a)
        m["sigmaS"] = self.spectrum(sigma_s)
        m["scale"] = scale
        m["g"] = g
        self.media.append(m)
        return len(self.media) - 1

    def mesh(self, positions, indices, material, normals=None, light_spectrum=-1, light_scale=0.0,
             medium_inside=-1, medium_outside=-1):
        p = np.asarray(positions, np.float32).reshape(-1, 3)
        n = None if normals is None else np.asarray(normals, np.float32).reshape(-1, 3)
        tri = np.asarray(indices, np.int64).reshape(-1, 3)
        base = self._prim_count
        r = np.zeros(len(tri), abi.PRIMITIVE)
        r["type"] = abi.PRIM_TRIANGLE
        r["material"] = material
        r["light"] = -1
        r["mediumInside"], r["mediumOutside"] = medium_inside, medium_outside
        r["p0"], r["p1"], r["p2"] = p[tri[:, 0]], p[tri[:, 1]], p[tri[:, 2]]
        if n is not None:
            r["n0"], r["n1"], r["n2"] = n[tri[:, 0]], n[tri[:, 1]], n[tri[:, 2]]
        r["uv"] = [0, 0, 1, 0, 1, 1]
        if light_spectrum >= 0:
            for k in range(len(tri)):
                a, b_, c = p[tri[k, 0]], p[tri[k, 1]], p[tri[k, 2]]
                l = np.zeros(1, abi.LIGHT)[0]
                l["type"] = abi.LIGHT_AREA
                l["primitive"] = base + k
                l["spectrum"] = light_spectrum
                l["scale"] = light_scale
                l["area"] = 0.5 * np.linalg.norm(np.cross(b_ - a, c - a))
                r[k]["light"] = len(self.lights)
                self.lights.append(l)
        self.prims.append(r)
        self._prim_count += len(tri)

    # -- finalisation ---------------------------------------------------------------------
    def finish(self, cam_pos, cam_target, fov_y, width, height, max_leaf=2):
        self.prim_array = np.concatenate(self.prims) if self.prims else np.zeros(0, abi.PRIMITIVE)
        self.mat_array = np.array(self.materials, dtype=abi.MATERIAL)
        self.spec_array = np.ascontiguousarray(np.stack(self.spectra).astype(np.float32))
        self.media_array = np.array(self.media, dtype=abi.MEDIUM) if self.media else np.zeros(1, abi.MEDIUM)
        # Power-based light selection (pmf proportional to scale * Y(spectrum) * area), as PRender's
        # LightSampler does for the v4 interface.
        ybar = spectra.cie_xyz(spectra.LAMBDA)[1]
        power = np.array([l["scale"] * float(np.sum(self.spec_array[l["spectrum"]] * ybar)) * l["area"] * math.pi
                          for l in self.lights], np.float64)
        for l, pw in zip(self.lights, power):
            l["pmf"] = pw / power.sum() if power.sum() > 0 else 0.0
        self.light_array = np.array(self.lights, dtype=abi.LIGHT) if self.lights else np.zeros(1, abi.LIGHT)
        tris = np.stack([self.prim_array["p0"], self.prim_array["p1"], self.prim_array["p2"]], axis=1)
        self.nodes, self.order = trace.build_bvh_triangles(tris, max_leaf=max_leaf)
        pts = np.concatenate([tris.reshape(-1, 3), np.asarray([cam_pos], np.float32)])
        lo, hi = pts.min(0), pts.max(0)
        self.world_center = 0.5 * (lo + hi)
        self.world_radius = max(float(np.linalg.norm(hi - self.world_center)), 1e-3)
        # Camera: right-handed look-at, camera space +x right, +y up, +z forward.
        pos = np.asarray(cam_pos, np.float64)
        d = np.asarray(cam_target, np.float64) - pos
        d /= np.linalg.norm(d)
        right = np.cross(d, [0.0, 1.0, 0.0])
        right /= np.linalg.norm(right)
        up = np.cross(right, d)
        M = np.zeros((3, 4))
        M[:, 0], M[:, 1], M[:, 2], M[:, 3] = right, up, d, pos
        self.camera.cameraToWorld[:] = [float(x) for x in M.ravel()]
        self.camera.tanHalfFov = math.tan(math.radians(fov_y) / 2)
        self.camera.aspect = width / height
        self.camera.lensRadius = 0.0
        self.camera.focalDistance = float(np.linalg.norm(np.asarray(cam_target) - pos))
        self.camera.width, self.camera.height, self.camera.margin = width, height, 0
        # Box filter (radius 0.5): a uniform CDF.
        self.filter.type = abi.FILTER_BOX
        self.filter.radius = 0.5
        self.filter.norm = 1.0
        self.filter.cdf[:] = [i / abi.FILTER_BINS for i in range(abi.FILTER_BINS + 1)]
        return self

    def light_bvh(self):
        """Light-BVH nodes over the area lights (triangle bounds, normal cone, power bound)."""
        lb = np.zeros((len(self.lights), 13), np.float32)
        for i, l in enumerate(self.lights):
            pr = self.prim_array[l["primitive"]]
            tri = np.stack([pr["p0"], pr["p1"], pr["p2"]])
            n = np.cross(tri[1] - tri[0], tri[2] - tri[0])
            n = n / np.linalg.norm(n)
            lb[i, 0:3], lb[i, 3:6] = tri.min(0), tri.max(0)
            lb[i, 6:9] = n
            lb[i, 9] = l["scale"] * self.spec_array[l["spectrum"]].max() * l["area"] * math.pi
            lb[i, 10], lb[i, 11], lb[i, 12] = 1.0, 0.0, 0.0
        nodes = np.zeros(max(1, 2 * len(self.lights) - 1), abi.LIGHT_BVH_NODE)
        cnt = abi.host_lib().prhost_build_light_bvh(abi.ptr(lb), len(self.lights), abi.ptr(nodes))
        return nodes[:cnt].copy()

    def desc(self) -> abi.SceneDesc:
        if self._desc is None:
            sd = abi.SceneDesc()
            sd.apiVersion = abi.API_VERSION
            sd.nodes, sd.nodeCount = self.nodes.ctypes.data, len(self.nodes)
            sd.primOrder = self.order.ctypes.data
            sd.prims, sd.primCount = self.prim_array.ctypes.data, len(self.prim_array)
            sd.materials, sd.materialCount = self.mat_array.ctypes.data, len(self.mat_array)
            sd.lights, sd.lightCount = self.light_array.ctypes.data, len(self.lights)
            sd.spectra, sd.spectrumCount = self.spec_array.ctypes.data, len(self.spec_array)
            sd.media, sd.mediumCount = self.media_array.ctypes.data, len(self.media)
            sd.cameraMedium = self.camera_medium
            sd.envSpectrum, sd.envScale, sd.envPmf = self.env_spectrum, self.env_scale, 0.0
            sd.worldCenter = abi.Float3(*[float(x) for x in self.world_center])
            sd.worldRadius = self.world_radius
            sd.camera = self.camera
            sd.filter = self.filter
            sd.cieYIntegral = spectra.cie_y_integral()
            # The descriptor points into this object's arrays: keep them alive with it.
            sd._owner = self
            self._desc = sd
        return self._desc


def build_box_scene(s: scenes.BoxScene) -> HostScene:
    h = HostScene()
    fog = -1
    if s.medium is not None:
        rgbu = lambda c: spectra.rgb_albedo(np.clip(np.asarray(c) / max(max(c), 1e-6), 0, 1)) * max(max(c), 1e-6)
        fog = h.medium(rgbu(s.medium["sigma_a"]) if max(s.medium["sigma_a"]) > 0 else spectra.constant(0.0),
                       rgbu(s.medium["sigma_s"]), s.medium["g"])
        h.camera_medium = fog
    mats = {
        "white": h.material(type=abi.MAT_DIFFUSE, albedo=h.spectrum(spectra.rgb_albedo((0.75, 0.75, 0.75)))),
        "red": h.material(type=abi.MAT_DIFFUSE, albedo=h.spectrum(spectra.rgb_albedo((0.63, 0.06, 0.05)))),
        "green": h.material(type=abi.MAT_DIFFUSE, albedo=h.spectrum(spectra.rgb_albedo((0.14, 0.45, 0.09)))),
    }
    n_au, k_au = spectra.metal_nk("Au")
    mats["gold"] = h.material(type=abi.MAT_CONDUCTOR, eta=h.spectrum(n_au), k=h.spectrum(k_au), alphaX=0.2, alphaY=0.2)
    mats["bk7"] = h.material(type=abi.MAT_DIELECTRIC, eta=h.spectrum(spectra.sellmeier(*spectra.BK7)), dispersive=1)
    black = h.material(type=abi.MAT_DIFFUSE, albedo=h.spectrum(spectra.constant(0.0)))
    for name, mat, quad in scenes.wall_quads():
        h.mesh(np.asarray(quad, np.float32), [0, 1, 2, 0, 2, 3], mats[mat], medium_inside=fog, medium_outside=fog)
    # Ceiling light: a 0.5 x 0.5 quad at (0, 0.999, -0.1) facing down (the "rect" light of the JSON form).
    c, hs = np.array([0.0, s.light_y, -0.1]), 0.25
    quad = np.array([[-hs, 0, -hs], [hs, 0, -hs], [hs, 0, hs], [-hs, 0, hs]])
    world = np.stack([quad[:, 2], -quad[:, 1], quad[:, 0]], axis=1) + c
    if s.light_up:  # facing the ceiling: the winding and normal flipped
        h.mesh(world.astype(np.float32), [0, 1, 2, 0, 2, 3], black, normals=np.tile([0.0, 1.0, 0.0], (4, 1)),
               light_spectrum=h.spectrum(spectra.blackbody(s.light_temperature)), light_scale=s.light_luminance,
               medium_inside=fog, medium_outside=fog)
    else:
        h.mesh(world.astype(np.float32), [0, 2, 1, 0, 3, 2], black, normals=np.tile([0.0, -1.0, 0.0], (4, 1)),
               light_spectrum=h.spectrum(spectra.blackbody(s.light_temperature)), light_scale=s.light_luminance,
               medium_inside=fog, medium_outside=fog)
    for sp in s.spheres:
        p, n, f = scenes.sphere_mesh(sp, s.subdiv)
        if sp.material == "lambert":
            m = h.material(type=abi.MAT_DIFFUSE, albedo=h.spectrum(spectra.rgb_albedo(sp.albedo)))
        else:
            m = mats[sp.material]
        h.mesh(p, f, m, normals=n, medium_inside=fog, medium_outside=fog)
    if s.slit > 0:
        for quad in scenes.occluder_quads(s):
            h.mesh(np.asarray(quad, np.float32), [0, 1, 2, 0, 2, 3], mats["white"], medium_inside=fog,
                   medium_outside=fog)
    for c_, r_, st in s.sss:
        p, n, f = scenes.sphere_mesh(scenes.Sphere(c_, r_, "bk7"), s.subdiv)
        med = h.medium(spectra.rgb_albedo(np.asarray(st) / max(st)) * 0.2 * max(st),
                       spectra.rgb_albedo(np.asarray(st) / max(st)) * 0.8 * max(st), 0.0)
        h.mesh(p, f, mats["bk7"], normals=n, medium_inside=med, medium_outside=fog)
    return h.finish(cam_pos=(0.0, -0.1, 0.98), cam_target=(0.0, -0.45, -0.3), fov_y=s.fov_y, width=s.width,
                    height=s.height)
