"""The box-and-spheres scene family as data, written in PRender's native JSON scene format
(schemas/prscene.schema.json; loader src/scene/scene_loader.cpp) so the reference CPU renderer and
this module render the same geometry, materials, lights and camera.

Base scene (the plain path-tracer workload): a closed 2 x 2 x 2 box (6 walls, 12 triangles;
white 0.75, left wall red (0.63, 0.06, 0.05), right wall green (0.14, 0.45, 0.09)), a 0.5 x 0.5
ceiling quad light with a 6500 K blackbody emitter, and a 35-sphere pyramid (5 x 5 + 3 x 3 + 1,
radius 0.12) of subdivision-3 icospheres (1280 triangles each) whose materials are drawn with a
seeded uniform choice among Lambertian (random RGB albedo in [0.1, 0.9]), rough GGX gold
(alpha 0.2, i.e. roughness sqrt(0.2)) and smooth dispersive BK7. Options add a homogeneous
chromatic medium filling the box (the uneven-batch variant) and change resolution, samples and
path length.
"""

from __future__ import annotations

import functools
import json
import math
import os
from dataclasses import dataclass, field

import numpy as np


@functools.lru_cache(maxsize=8)
def _icosphere(subdiv: int):
    v, f = _icosphere_build(subdiv)
    v.setflags(write=False)
    f.setflags(write=False)
    return v, f


def icosphere(subdiv: int):
    """Unit icosphere: (vertices (n, 3) float64, faces (m, 3) int32), counter-clockwise outward."""
    v, f = _icosphere(subdiv)
    return v.copy(), f.copy()


def _icosphere_build(subdiv: int):
    t = (1.0 + 5 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
         (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
         (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    verts = [np.array(p, float) / np.linalg.norm(p) for p in v]
    faces = list(f)
    for _ in range(subdiv):
        cache = {}

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    return np.array(verts), np.array(faces, dtype=np.int32)


@dataclass
class Sphere:
    center: tuple
    radius: float
    material: str  # "lambert", "gold", "bk7"
    albedo: tuple = (0.5, 0.5, 0.5)


@dataclass
class BoxScene:
    width: int = 256
    height: int = 256
    spp: int = 64
    max_depth: int = 8
    seed: int = 0
    subdiv: int = 3
    light_temperature: float = 6500.0
    light_luminance: float = 30.0
    fov_y: float = 62.0
    medium: dict | None = None  # {"sigma_a": [r,g,b], "sigma_s": [r,g,b], "g": 0.6}
    # Slit variant: the ceiling light above a horizontal occluder at y = occluder_y with a slit of
    # this width along z through its middle (0 = no occluder).
    slit: float = 0.0
    occluder_y: float = 0.8
    # Subsurface spheres: (centre, radius, sigma_t rgb); BK7 surface, homogeneous interior with
    # albedo 0.8 (sigma_s = 0.8 sigma_t).
    sss: list = field(default_factory=list)
    # Indirect variant: the ceiling light turned to face up (lowered to y = light_y), so the room
    # is lit only by the bright patch it makes on the ceiling (next-event estimation finds no light).
    light_up: bool = False
    light_y: float = 0.999
    # Heterogeneous variant: {"sigma_a", "sigma_s", "g", "scale", "density" (nz, ny, nx) float32,
    # "bounds" (2, 3) medium space, "matrix" 4x4 medium-to-world}; replaces `medium`.
    grid: dict | None = None
    spheres: list = field(default_factory=list)
    filter: str = "box"

    def triangle_count(self) -> int:
        return 12 + 2 + len(self.spheres) * 20 * 4 ** self.subdiv


def pyramid_spheres(seed: int, radius: float = 0.12):
    """35 spheres: 5 x 5 + 3 x 3 + 1, touching, resting on the floor (y = -1) near the back."""
    rng = np.random.default_rng(seed)
    out = []
    layers = [(5, 0.0), (3, 1), (1, 2)]
    cz = -0.25
    for count, level in layers:
        y = -1.0 + radius + level * radius * math.sqrt(2.0)
        off = (count - 1) / 2.0
        for i in range(count):
            for k in range(count):
                x = (i - off) * 2 * radius
                z = cz + (k - off) * 2 * radius
                kind = ("lambert", "gold", "bk7")[int(rng.integers(0, 3))]
                albedo = tuple(float(a) for a in rng.uniform(0.1, 0.9, 3))
                out.append(Sphere((x, y, z), radius, kind, albedo))
    return out


def box_scene(seed: int = 0, width: int = 256, height: int = 256, spp: int = 64, max_depth: int = 8,
              medium: bool = False, subdiv: int = 3) -> BoxScene:
    s = BoxScene(width=width, height=height, spp=spp, max_depth=max_depth, seed=seed, subdiv=subdiv)
    s.spheres = pyramid_spheres(seed)
    if medium:
        rng = np.random.default_rng(1000 + seed)
        s.medium = {"sigma_s": [float(x) for x in rng.uniform(0.05, 0.5, 3)],
                    "sigma_a": [float(x) for x in rng.uniform(0.0, 0.1, 3)], "g": 0.6}
    return s


def slit_scene(seed: int = 0, width: int = 1024, height: int = 1024, spp: int = 64, max_depth: int = 32,
               subdiv: int = 3, sss_count: int = 12) -> BoxScene:
    """The guided-vs-plain scene: the box of box_scene, its ceiling light hidden behind a
    horizontal occluder at y = 0.8 so that light enters only through a 0.1-wide slit, plus
    `sss_count` subsurface BK7 spheres (interior sigma_t RGB uniform in [1, 20]) in place of the
    pyramid."""
    s = BoxScene(width=width, height=height, spp=spp, max_depth=max_depth, seed=seed, subdiv=subdiv)
    s.slit = 0.1
    rng = np.random.default_rng(5000 + seed)
    r = 0.14
    for k in range(sss_count):
        x = -0.75 + 0.3 * (k % 6)
        z = -0.55 + 0.45 * (k // 6)
        s.sss.append(((x, -1.0 + r, z), r, [float(v) for v in rng.uniform(1.0, 20.0, 3)]))
    return s


def occluder_quads(s: BoxScene):
    """The two occluder quads (corners counter-clockwise seen from below) leaving the slit open."""
    y, h = s.occluder_y, s.slit / 2
    return [[(-1, y, -1), (-1, y, 1), (-h, y, 1), (-h, y, -1)],
            [(h, y, -1), (h, y, 1), (1, y, 1), (1, y, -1)]]


def indirect_scene(seed: int = 0, width: int = 64, height: int = 64, spp: int = 64, max_depth: int = 16,
                   subdiv: int = 2) -> BoxScene:
    """The box-and-spheres scene lit only indirectly: its light faces the ceiling from y = 0.9."""
    s = box_scene(seed=seed, width=width, height=height, spp=spp, max_depth=max_depth, subdiv=subdiv)
    s.light_up = True
    s.light_y = 0.9
    s.light_luminance = 300.0
    return s


def outdoor_scene_json(width: int = 32, height: int = 32, spp: int = 64, max_depth: int = 8, elevation: float = 30.0,
                       azimuth: float = 40.0, turbidity: float = 3.0, sky_resolution: int = 64,
                       env_file: str | None = None, env_rotation: float = 0.0, sun_scale: float = 1.0,
                       sky_scale: float = 1.0) -> dict:
    """An outdoor test scene in the reference's JSON form: a 20 x 20 ground (albedo 0.3) with a
    Lambertian, a gold and a BK7 sphere, lit by the reference's Preetham sun and sky (sun_sky) or,
    with env_file, by an image environment map."""
    mats = {"ground": {"type": "diffuse", "reflectance": [0.3, 0.3, 0.3]},
            "red": {"type": "diffuse", "reflectance": [0.7, 0.2, 0.15]},
            "gold": {"type": "conductor", "metal": "Au", "roughness": 0.3},
            "bk7": {"type": "dielectric", "ior": "BK7"}}
    geometry = {"ground": {"type": "mesh", "positions": [-10, 0, -10, -10, 0, 10, 10, 0, 10, 10, 0, -10],
                           "indices": [0, 1, 2, 0, 2, 3]},
                "s0": {"type": "sphere", "center": [-1.2, 0.5, 0], "radius": 0.5},
                "s1": {"type": "sphere", "center": [0, 0.5, 0], "radius": 0.5},
                "s2": {"type": "sphere", "center": [1.2, 0.5, 0], "radius": 0.5}}
    objects = [{"name": "ground", "geometry": "ground", "material": "ground"},
               {"name": "s0", "geometry": "s0", "material": "red"},
               {"name": "s1", "geometry": "s1", "material": "gold"},
               {"name": "s2", "geometry": "s2", "material": "bk7"}]
    if env_file is None:
        lights = {"sky": {"type": "sun_sky", "elevation": elevation, "azimuth": azimuth, "turbidity": turbidity,
                          "resolution": sky_resolution, "sun_scale": sun_scale, "sky_scale": sky_scale}}
    else:
        lights = {"env": {"type": "environment", "file": env_file, "intensity": 1.0, "rotation": env_rotation}}
    return {"materials": mats, "media": {}, "geometry": geometry, "objects": objects, "lights": lights,
            "cameras": {"cam": {"type": "pinhole", "position": [0, 1.4, 4.0], "look_at": [0, 0.4, 0], "fov_y": 40}},
            "render": {"camera": "cam", "seed": 0, "film": {"width": width, "height": height, "filter": "box"},
                       "integrator": {"type": "path", "spp": spp, "max_depth": max_depth}}}


def sun_direction(elevation: float, azimuth: float) -> np.ndarray:
    """The reference loader's sun direction (scene_loader.cpp:977-984)."""
    el, az = math.radians(elevation), math.radians(azimuth)
    return np.array([math.cos(el) * math.sin(az), math.sin(el), math.cos(el) * math.cos(az)], np.float32)


def uneven_batch(count: int = 48, seed: int = 4242) -> list:
    """The uneven batch: `count` renders of the box family, scene seeds 0..count-1, each with a
    resolution drawn uniformly from {128, 256, 512, 1024}^2, spp from {16, 64, 256} and max depth
    from {8, 16, 32} (seeded draws); even scene seeds fill the box with the homogeneous chromatic
    medium of box_scene(medium=True)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        res = int(rng.choice([128, 256, 512, 1024]))
        spp = int(rng.choice([16, 64, 256]))
        depth = int(rng.choice([8, 16, 32]))
        out.append(box_scene(seed=k, width=res, height=res, spp=spp, max_depth=depth, medium=(k % 2 == 0)))
    return out


def smoke_density(res: int = 24, seed: int = 0) -> np.ndarray:
    """A smooth cloud on a res^3 grid over [-1, 1]^3 ((nz, ny, nx) float32): a floor layer that
    thins with height plus a few seeded Gaussian puffs, in [0, ~1.5]."""
    rng = np.random.default_rng(7000 + seed)
    c = (np.arange(res) + 0.5) / res * 2.0 - 1.0
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    d = 0.6 * np.exp(-2.5 * (y + 1.0))
    for _ in range(4):
        m = rng.uniform(-0.6, 0.6, 3)
        r = rng.uniform(0.25, 0.45)
        d += rng.uniform(0.5, 1.0) * np.exp(-((x - m[0]) ** 2 + (y - m[1]) ** 2 + (z - m[2]) ** 2) / (2 * r * r))
    return d.astype(np.float32)


def grid_box_scene(seed: int = 0, width: int = 256, height: int = 256, spp: int = 64, max_depth: int = 8,
                   subdiv: int = 3, res: int = 24, constant: float | None = None, turn_deg: float = 20.0,
                   scale: float = 1.1) -> BoxScene:
    """The box scene filled with a heterogeneous chromatic smoke (a voxel grid medium). The grid
    covers [-1, 1]^3 in medium space, mapped to the world by `scale`, a `turn_deg` turn about y
    and a 0.05 lift, inside a 2.2 interface box around the room. constant: a uniform density
    instead of the cloud (with turn_deg 0 and scale >= 1.2 the grid covers the whole interface
    box, and the medium equals a homogeneous one of sigma * constant)."""
    s = box_scene(seed=seed, width=width, height=height, spp=spp, max_depth=max_depth, subdiv=subdiv)
    rng = np.random.default_rng(2000 + seed)
    a = math.radians(turn_deg)
    m = np.array([[scale * math.cos(a), 0, scale * math.sin(a), 0.0], [0, scale, 0, 0.05],
                  [-scale * math.sin(a), 0, scale * math.cos(a), 0.0], [0, 0, 0, 1]], dtype=np.float64)
    dens = smoke_density(res, seed) if constant is None else np.full((res, res, res), constant, np.float32)
    s.grid = {"sigma_s": [float(x) for x in rng.uniform(0.3, 1.2, 3)],
              "sigma_a": [float(x) for x in rng.uniform(0.02, 0.2, 3)], "g": 0.4, "scale": 1.0,
              "density": dens, "bounds": np.array([[-1, -1, -1], [1, 1, 1]], np.float32),
              "matrix": m.astype(np.float32)}
    return s


def _f32(a) -> list:
    """float32 values as Python floats that round-trip exactly through JSON."""
    return [float(x) for x in np.asarray(a, dtype=np.float32).ravel()]


def sphere_mesh(sp: Sphere, subdiv: int):
    """World-space float32 positions, unit normals and indices of one icosphere."""
    v, f = icosphere(subdiv)
    p = (v * sp.radius + np.array(sp.center)).astype(np.float32)
    return p, v.astype(np.float32), f


def wall_quads():
    """The 6 walls as (name, material, 4 corners counter-clockwise seen from inside)."""
    return [
        ("floor", "white", [(-1, -1, -1), (-1, -1, 1), (1, -1, 1), (1, -1, -1)]),
        ("ceiling", "white", [(-1, 1, -1), (1, 1, -1), (1, 1, 1), (-1, 1, 1)]),
        ("back", "white", [(-1, -1, -1), (1, -1, -1), (1, 1, -1), (-1, 1, -1)]),
        ("front", "white", [(-1, -1, 1), (-1, 1, 1), (1, 1, 1), (1, -1, 1)]),
        ("left", "red", [(-1, -1, -1), (-1, 1, -1), (-1, 1, 1), (-1, -1, 1)]),
        ("right", "green", [(1, -1, -1), (1, -1, 1), (1, 1, 1), (1, 1, -1)]),
    ]


def to_reference_json(s: BoxScene) -> dict:
    mats = {
        "white": {"type": "diffuse", "reflectance": [0.75, 0.75, 0.75]},
        "red": {"type": "diffuse", "reflectance": [0.63, 0.06, 0.05]},
        "green": {"type": "diffuse", "reflectance": [0.14, 0.45, 0.09]},
        "gold": {"type": "conductor", "metal": "Au", "roughness": math.sqrt(0.2)},
        "bk7": {"type": "dielectric", "ior": "BK7"},
    }
    geometry, objects = {}, []
    for name, mat, quad in wall_quads():
        geometry[name] = {"type": "mesh", "positions": _f32(quad), "indices": [0, 1, 2, 0, 2, 3]}
        objects.append({"name": name, "geometry": name, "material": mat})
    for i, sp in enumerate(s.spheres):
        p, n, f = sphere_mesh(sp, s.subdiv)
        gid = f"sphere{i}"
        geometry[gid] = {"type": "mesh", "positions": _f32(p), "normals": _f32(n),
                         "indices": [int(x) for x in f.ravel()], "closed": True}
        if sp.material == "lambert":
            mid = f"lambert{i}"
            mats[mid] = {"type": "diffuse", "reflectance": list(sp.albedo)}
        else:
            mid = sp.material
        objects.append({"name": gid, "geometry": gid, "material": mid})
    media = {}
    if s.slit > 0:
        for k, quad in enumerate(occluder_quads(s)):
            gid = f"occluder{k}"
            geometry[gid] = {"type": "mesh", "positions": _f32(quad), "indices": [0, 1, 2, 0, 2, 3]}
            objects.append({"name": gid, "geometry": gid, "material": "white"})
    for k, (c, r, st) in enumerate(s.sss):
        p, n, f = sphere_mesh(Sphere(c, r, "bk7"), s.subdiv)
        gid = f"sss{k}"
        geometry[gid] = {"type": "mesh", "positions": _f32(p), "normals": _f32(n),
                         "indices": [int(x) for x in f.ravel()], "closed": True}
        media[gid] = {"type": "homogeneous", "sigma_s": [0.8 * v for v in st], "sigma_a": [0.2 * v for v in st],
                      "g": 0.0}
        objects.append({"name": gid, "geometry": gid, "material": "bk7", "interior": gid})
    if s.medium is not None:
        media["fog"] = {"type": "homogeneous", "sigma_a": s.medium["sigma_a"], "sigma_s": s.medium["sigma_s"],
                        "g": s.medium["g"]}
        # An invisible closed container slightly larger than the room holds the medium; the loader
        # gives every object inside it (walls, light, spheres) the medium as exterior, and the
        # camera inside picks it up too.
        geometry["fogbox"] = {"type": "box", "size": [2.2, 2.2, 2.2]}
        mats["boundary"] = {"type": "interface"}
        objects.append({"name": "fogbox", "geometry": "fogbox", "material": "boundary", "interior": "fog",
                        "exterior": None})
    if s.grid is not None:
        gr = s.grid
        media["smoke"] = {"type": "grid", "file": gr["file"], "sigma_a": gr["sigma_a"], "sigma_s": gr["sigma_s"],
                          "g": gr["g"], "scale": gr["scale"], "bounds": np.asarray(gr["bounds"]).tolist(),
                          "transform": {"matrix": _f32(gr["matrix"])}}
        geometry["smokebox"] = {"type": "box", "size": [2.2, 2.2, 2.2]}
        mats["boundary"] = {"type": "interface"}
        objects.append({"name": "smokebox", "geometry": "smokebox", "material": "boundary",
                        "interior": "smoke", "exterior": None})
    doc = {
        "materials": mats,
        "media": media,
        "geometry": geometry,
        "objects": objects,
        "lights": {"ceiling": {"type": "rect", "position": [0, 0.999, -0.1], "size": [0.5, 0.5],
                               "direction": [0, -1, 0], "temperature": s.light_temperature,
                               "luminance": s.light_luminance}},
        "cameras": {"cam": {"type": "pinhole", "position": [0, -0.1, 0.98], "look_at": [0, -0.45, -0.3],
                            "fov_y": s.fov_y}},
        "render": {"camera": "cam", "seed": s.seed,
                   "film": {"width": s.width, "height": s.height, "filter": s.filter},
                   "integrator": {"type": "path", "spp": s.spp, "max_depth": s.max_depth}},
    }
    return doc


def write_reference_json(s: BoxScene, path: str) -> str:
    """Writes the scene (and, for the grid variant, its density as a .vol beside it)."""
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    if s.grid is not None:
        from .media import write_vol
        s.grid["file"] = write_vol(os.path.abspath(path) + ".vol", s.grid["density"], s.grid["bounds"])
    with open(path, "w") as f:
        json.dump(to_reference_json(s), f)
    return path
