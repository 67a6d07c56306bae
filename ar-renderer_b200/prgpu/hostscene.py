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

    def spheres(self, centers, radii, materials, medium_inside=-1, medium_outside=-1):
        """Analytic spheres (the reference's Sphere shape, shape.cpp:42-85)."""
        c = np.asarray(centers, np.float32).reshape(-1, 3)
        r = np.zeros(len(c), abi.PRIMITIVE)
        r["type"] = abi.PRIM_SPHERE
        r["material"] = np.asarray(materials, np.int32)
        r["light"] = -1
        r["mediumInside"], r["mediumOutside"] = medium_inside, medium_outside
        r["p0"] = c
        r["r"] = np.asarray(radii, np.float32)
        self.prims.append(r)
        self._prim_count += len(c)

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
        pa = self.prim_array
        sph = pa["type"] == abi.PRIM_SPHERE
        if not sph.any():
            tris = np.stack([pa["p0"], pa["p1"], pa["p2"]], axis=1)
            self.nodes, self.order = trace.build_bvh_triangles(tris, max_leaf=max_leaf)
            lo = np.minimum(tris.reshape(-1, 3).min(0), np.asarray(cam_pos, np.float32))
            hi = np.maximum(tris.reshape(-1, 3).max(0), np.asarray(cam_pos, np.float32))
        else:
            bmin = np.minimum(np.minimum(pa["p0"], pa["p1"]), pa["p2"])
            bmax = np.maximum(np.maximum(pa["p0"], pa["p1"]), pa["p2"])
            rr = pa["r"][sph, None]
            bmin[sph] = pa["p0"][sph] - rr
            bmax[sph] = pa["p0"][sph] + rr
            self.nodes, self.order = trace.build_bvh_bounds(bmin, bmax, max_leaf=max_leaf)
            lo = np.minimum(bmin.min(0), np.asarray(cam_pos, np.float32))
            hi = np.maximum(bmax.max(0), np.asarray(cam_pos, np.float32))
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


def box_mesh(lo, hi):
    """(8 x 3 float32 corners, 12 x 3 indices) of an axis-aligned box, triangles counter-clockwise
    seen from outside (outward geometric normals)."""
    lo, hi = np.asarray(lo, np.float32), np.asarray(hi, np.float32)
    v = np.array([[(hi if (k >> a) & 1 else lo)[a] for a in range(3)] for k in range(8)], np.float32)
    f = [[0, 2, 3, 0, 3, 1], [4, 5, 7, 4, 7, 6], [0, 1, 5, 0, 5, 4], [2, 6, 7, 2, 7, 3], [0, 4, 6, 0, 6, 2],
         [1, 3, 7, 1, 7, 5]]
    return v, np.asarray(f, np.int64).reshape(-1, 3)


def fbm_heightfield(res: int, octaves: int = 8, seed: int = 0) -> np.ndarray:
    """(res, res) float32 fractional Brownian motion of value noise (bilinear lattice noise, gain
    0.5, lacunarity 2), seeded."""
    rng = np.random.default_rng(seed)
    h = np.zeros((res, res), np.float32)
    amp, total = 1.0, 0.0
    for o in range(octaves):
        cells = 4 * 2 ** o
        lat = rng.random((cells + 1, cells + 1)).astype(np.float32)
        t = np.linspace(0, cells, res, endpoint=False, dtype=np.float32)
        i = t.astype(np.int32)
        f = t - i
        f = f * f * (3 - 2 * f)
        a = lat[i][:, i] * (1 - f)[None, :] + lat[i][:, i + 1] * f[None, :]
        b = lat[i + 1][:, i] * (1 - f)[None, :] + lat[i + 1][:, i + 1] * f[None, :]
        h += amp * (a * (1 - f)[:, None] + b * f[:, None])
        total += amp
        amp *= 0.5
    return h / total


def fbm_cloud(res: int, octaves: int = 5, seed: int = 1, max_density: float = 4.0) -> np.ndarray:
    """(res, res, res) float32 cloud density: fBm value noise thresholded and faded by an
    ellipsoidal falloff towards the grid's edges, scaled to max_density."""
    rng = np.random.default_rng(seed)
    c = (np.arange(res, dtype=np.float32) + 0.5) / res
    d = np.zeros((res, res, res), np.float32)
    amp, total = 1.0, 0.0
    for o in range(octaves):
        cells = 3 * 2 ** o
        lat = rng.random((cells + 1,) * 3).astype(np.float32)
        t = c * cells
        i = np.minimum(t.astype(np.int32), cells - 1)
        f = t - i
        f = f * f * (3 - 2 * f)
        acc = np.zeros((res, res, res), np.float32)
        for dz in (0, 1):
            wz = (f if dz else 1 - f)[:, None, None]
            for dy in (0, 1):
                wy = (f if dy else 1 - f)[None, :, None]
                for dx in (0, 1):
                    wx = (f if dx else 1 - f)[None, None, :]
                    acc += lat[np.ix_(i + dz, i + dy, i + dx)] * wz * wy * wx
        d += amp * acc
        total += amp
        amp *= 0.5
    d /= total
    z, y, x = np.meshgrid(c * 2 - 1, c * 2 - 1, c * 2 - 1, indexing="ij")
    fall = np.clip(1 - (x * x + (y * 1.6) ** 2 + z * z), 0, 1)
    dens = np.clip((d * fall - 0.25) * 4.0, 0, 1) * max_density
    return dens.astype(np.float32)


METALS = ("Au", "Ag", "Cu", "Al")
CLOUD_TO_WORLD = np.array([[25, 0, 0, 0], [0, 6, 0, 22], [0, 0, 25, -5], [0, 0, 0, 1]], np.float64)
CLOUD_BOX = (np.array([-25.0, 16.0, -30.0]), np.array([25.0, 28.0, 20.0]))
SUN_ELEVATION, SUN_AZIMUTH = 20.0, math.degrees(0.6)
SUN_RADIUS_DEG = 0.2665     # the loader's sun radius (scene_loader.cpp:986)
SUN_SKY_INTENSITY = 0.03    # the loader's default sun_sky intensity (scene_loader.cpp:985)
CAMERA = dict(cam_pos=(0.0, 14.0, 45.0), cam_target=(0.0, 6.0, 0.0), fov_y=45.0)


def large_scene_layout(terrain_res: int = 4096, cloud_res: int = 256, spheres: int = 200, seed: int = 0) -> dict:
    """The seeded content of the large outdoor scene, shared by its host-built form
    (build_large_scene) and its reference JSON form: terrain vertices / triangles over
    [-50, 50]^2 (fBm height x 8), the cloud density ((nz, ny, nx) over [-1, 1]^3 in medium space,
    placed by CLOUD_TO_WORLD inside CLOUD_BOX) and the spheres (centre, radius, metal, GGX alpha)."""
    rng = np.random.default_rng(seed)
    hf = fbm_heightfield(terrain_res, 8, seed) * 8.0
    g = np.linspace(-50, 50, terrain_res, dtype=np.float32)
    X, Z = np.meshgrid(g, g)
    verts = np.stack([X, hf, Z], -1).reshape(-1, 3)
    ii = np.arange(terrain_res - 1)
    q = (ii[:, None] * terrain_res + ii[None, :]).ravel()
    tris = np.stack([q, q + terrain_res, q + terrain_res + 1, q, q + terrain_res + 1, q + 1], 1).reshape(-1, 3)
    sph = []
    for k in range(spheres):
        x, z = rng.uniform(-30, 30, 2)
        rr = float(rng.uniform(0.3, 1.2))
        iz = int(np.clip((z + 50) / 100 * (terrain_res - 1), 0, terrain_res - 1))
        ix = int(np.clip((x + 50) / 100 * (terrain_res - 1), 0, terrain_res - 1))
        sph.append(((float(x), float(hf[iz, ix]) + rr, float(z)), rr, METALS[k % 4], float(rng.uniform(0.05, 0.5))))
    return {"verts": verts, "tris": tris, "spheres": sph, "density": fbm_cloud(cloud_res, 5, seed + 1, 4.0)}


def build_large_scene(width: int = 3840, height: int = 2160, terrain_res: int = 4096, cloud_res: int = 256,
                      spheres: int = 200, seed: int = 0, turbidity: float = 3.0, sky_resolution: int = 512):
    """The large outdoor scene: a terrain_res^2 fBm heightfield (8 octaves, 2 (res - 1)^2 triangles,
    Lambert 0.3) over [-50, 50]^2, a cloud_res^3 fBm cloud density grid above it (max density 4,
    albedo 0.95, Henyey-Greenstein g = 0.8, spectral / ratio tracking inside an interface box),
    `spheres` analytic GGX conductor spheres (Au / Ag / Cu / Al, alpha uniform in [0.05, 0.5]) on
    the terrain, lit as PRender lights a "sun_sky" light (scene_loader.cpp:977-996): the sun 20
    degrees above the horizon with the spectral radiance of pr::MakeSunRadiance, the Preetham sky
    of pr::MakePreethamSky (turbidity 3, ground albedo 0.3, a sky_resolution x sky_resolution / 2
    equirect map, importance-sampled), both at the loader's intensity 0.03 and picked with
    probability 1/2 each, both from the host library (prhost_sun_radiance, prhost_preetham_sky).
    The sky texels are fitted to sigmoid polynomials under a 6504 K blackbody of unit luminance,
    which stands in for the reference's tabulated CIE D65 (same luminance and white point to
    within the fit; the reference interpolates its precomputed table of fits under D65).
    Returns (HostScene, SceneExt)."""
    from . import media, render

    lay = large_scene_layout(terrain_res, cloud_res, spheres, seed)
    h = HostScene()
    ground = h.material(type=abi.MAT_DIFFUSE, albedo=h.spectrum(spectra.constant(0.3)))
    h.mesh(lay["verts"], lay["tris"], ground)
    metals = {}
    for name in METALS:
        n_, k_ = spectra.metal_nk(name)
        metals[name] = (h.spectrum(n_), h.spectrum(k_))
    ms = [h.material(type=abi.MAT_CONDUCTOR, eta=metals[m][0], k=metals[m][1], alphaX=a, alphaY=a)
          for _, _, m, a in lay["spheres"]]
    if ms:
        h.spheres([c for c, _, _, _ in lay["spheres"]], [r for _, r, _, _ in lay["spheres"]], ms)
    absorb = h.spectrum(spectra.constant(0.05))
    scatter = h.spectrum(spectra.constant(0.95))
    sun_dir = scenes.sun_direction(SUN_ELEVATION, SUN_AZIMUTH)
    white = spectra.blackbody(6504.0)  # unit luminance: the D65 stand-in
    sky_ill = h.spectrum(white)
    sun_spec = h.spectrum(spectra.sun_radiance(sun_dir, turbidity, SUN_RADIUS_DEG))
    grid = media.grid_desc(absorb, scatter, lay["density"], [[-1, -1, -1], [1, 1, 1]], scale=1.0, g=0.8,
                           world_to_medium=media.affine_inverse(CLOUD_TO_WORLD))
    # The cloud's interface box, outward-facing: rays that cross it enter and leave grid medium 0
    # (grids are numbered after the SceneDesc's homogeneous media, of which there are none).
    bverts, bidx = box_mesh(*CLOUD_BOX)
    h.mesh(bverts, bidx, h.material(type=abi.MAT_INTERFACE), medium_inside=len(h.media), medium_outside=-1)
    h.finish(width=width, height=height, max_leaf=4, **CAMERA)
    # Sky: the Preetham map, its RGB texels uplifted to sigmoid-polynomial spectra times the
    # illuminant (the reference's RGBIlluminantSpectrum texels, light.cpp:243-265).
    sw, sh = sky_resolution, sky_resolution // 2
    sky = spectra.preetham_sky(sun_dir, turbidity, 0.3, sw, sh)
    texels = np.ascontiguousarray(spectra.rgb_to_sigmoid(sky.reshape(-1, 3), white).reshape(sh, sw, 4))
    env = abi.EnvMapDesc()
    env.width, env.height = sw, sh
    env.texels = texels.ctypes.data
    env.illuminant, env.scale, env.rotationDeg, env.pmf = sky_ill, SUN_SKY_INTENSITY, 0.0, 0.5
    sd = abi.SunDesc()
    for i, v in enumerate(sun_dir):
        sd.direction[i] = float(v)
    sd.cosThetaMax = math.cos(math.radians(SUN_RADIUS_DEG))
    sd.spectrum, sd.scale, sd.pmf = sun_spec, SUN_SKY_INTENSITY, 0.5
    ext = render.make_ext(grid_media=[grid])
    ext.envMap = C.addressof(env)
    ext.sun = C.addressof(sd)
    ext._keep += [env, texels, sd, grid, lay["density"]]
    return h, ext


def write_large_scene_json(path: str, width: int, height: int, spp: int = 16, max_depth: int = 64,
                           terrain_res: int = 48, cloud_res: int = 24, spheres: int = 12, seed: int = 0,
                           turbidity: float = 3.0, sky_resolution: int = 64) -> str:
    """The large outdoor scene in the reference's JSON form (the same seeded layout as
    build_large_scene; the cloud written as a .vol beside the JSON), lit by the reference's own
    Preetham sun and sky (turbidity, sun elevation 20 degrees). Returns the path."""
    import json
    import os

    from . import media

    lay = large_scene_layout(terrain_res, cloud_res, spheres, seed)
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    vol = media.write_vol(os.path.abspath(path) + ".vol", lay["density"], [[-1, -1, -1], [1, 1, 1]])
    f32 = lambda a: [float(x) for x in np.asarray(a, np.float32).ravel()]
    mats = {"ground": {"type": "diffuse", "reflectance": [0.3, 0.3, 0.3]}, "boundary": {"type": "interface"}}
    geometry = {"terrain": {"type": "mesh", "positions": f32(lay["verts"]),
                            "indices": [int(x) for x in lay["tris"].ravel()]}}
    objects = [{"name": "terrain", "geometry": "terrain", "material": "ground"}]
    for k, (c, r, metal, alpha) in enumerate(lay["spheres"]):
        mats[f"metal{k}"] = {"type": "conductor", "metal": metal, "roughness": math.sqrt(alpha)}
        geometry[f"ball{k}"] = {"type": "sphere", "center": f32(c), "radius": float(np.float32(r))}
        objects.append({"name": f"ball{k}", "geometry": f"ball{k}", "material": f"metal{k}"})
    bv, bi = box_mesh(*CLOUD_BOX)
    geometry["cloudbox"] = {"type": "mesh", "positions": f32(bv), "indices": [int(x) for x in bi.ravel()],
                            "closed": True}
    objects.append({"name": "cloudbox", "geometry": "cloudbox", "material": "boundary", "interior": "cloud",
                    "exterior": None})
    doc = {
        "materials": mats,
        "media": {"cloud": {"type": "grid", "file": vol, "sigma_a": [0.05, 0.05, 0.05], "sigma_s": [0.95, 0.95, 0.95],
                            "g": 0.8, "scale": 1.0, "bounds": [[-1, -1, -1], [1, 1, 1]],
                            "transform": {"matrix": f32(CLOUD_TO_WORLD)}}},
        "geometry": geometry, "objects": objects,
        "lights": {"sky": {"type": "sun_sky", "elevation": SUN_ELEVATION, "azimuth": SUN_AZIMUTH,
                           "turbidity": turbidity, "resolution": sky_resolution}},
        "cameras": {"cam": {"type": "pinhole", "position": list(CAMERA["cam_pos"]),
                            "look_at": list(CAMERA["cam_target"]), "fov_y": CAMERA["fov_y"]}},
        "render": {"camera": "cam", "seed": seed, "film": {"width": width, "height": height, "filter": "box"},
                   "integrator": {"type": "path", "spp": spp, "max_depth": max_depth}},
    }
    with open(path, "w") as f:
        json.dump(doc, f)
    return path
