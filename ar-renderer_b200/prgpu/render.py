"""Rendering through the C ABI: prgpu_render (v4, float sums added into the caller's film) and
prgpu_render_ex (FP64 film accumulated in sample order, light BVH, statistics)."""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi


def _desc_ptr(scene) -> C.c_void_p:
    """A SceneDesc pointer: an int address, a ctypes SceneDesc, or an object with .desc()."""
    if isinstance(scene, int):
        return C.c_void_p(scene)
    if isinstance(scene, abi.SceneDesc):
        return C.cast(C.pointer(scene), C.c_void_p)
    return C.cast(C.pointer(scene.desc()), C.c_void_p)


def render_v4(scene, width: int, height: int, spp: int, first_sample: int = 0, seed: int = 0, max_depth: int = 0,
              clamp: float = 0.0, out: np.ndarray | None = None, device: int = 0) -> np.ndarray:
    """prgpu_render: returns (adds into) float32 XYZ sums of shape (height, width, 3)."""
    if out is None:
        out = np.zeros((height, width, 3), dtype=np.float32)
    rp = abi.RenderParams(spp, first_sample, seed, max_depth, clamp)
    err = abi.err_buf()
    rc = abi.gpu_lib().prgpu_render(device, _desc_ptr(scene), C.cast(C.pointer(rp), C.c_void_p), abi.ptr(out), err,
                                    len(err))
    abi.check(rc, err, "prgpu_render")
    return out


def render_ex(scene, width: int, height: int, spp: int, first_sample: int = 0, seed: int = 0, max_depth: int = 0,
              clamp: float = 0.0, out: np.ndarray | None = None, ext: abi.SceneExt | None = None, device: int = 0,
              stats: bool = False):
    """prgpu_render_ex: accumulates FP64 XYZ sums (height, width, 3) in sample order onto `out`."""
    if out is None:
        out = np.zeros((height, width, 3), dtype=np.float64)
    assert out.dtype == np.float64 and out.flags["C_CONTIGUOUS"]
    rp = abi.RenderParams(spp, first_sample, seed, max_depth, clamp)
    st = abi.RenderStats()
    err = abi.err_buf()
    extp = C.cast(C.pointer(ext), C.c_void_p) if ext is not None else None
    rc = abi.gpu_lib().prgpu_render_ex(device, _desc_ptr(scene), extp, C.cast(C.pointer(rp), C.c_void_p),
                                       abi.ptr(out), C.cast(C.pointer(st), C.c_void_p), err, len(err))
    abi.check(rc, err, "prgpu_render_ex")
    return (out, st) if stats else out


GUIDE_SAMPLE, GUIDE_TRAIN, GUIDE_RESET = 1, 2, 4


def make_ext(light_bvh: np.ndarray | None = None, light_bvh_prob: float = 1.0, wavefront_paths: int = 0,
             block_size: int = 0, grid_media=None, guide: int = 0, delta_lights=None, textures=None,
             material_textures=None, rgb_to_spectrum: np.ndarray | None = None,
             texture_nodes=None) -> abi.SceneExt:
    """SceneExt for prgpu_render_ex. grid_media: GridMediumDesc records (media.grid_desc), indexed
    after the SceneDesc's homogeneous media. guide: GUIDE_SAMPLE (sample diffuse vertices with the
    guide network), GUIDE_TRAIN (train it online, one Adam step per wavefront chunk), GUIDE_RESET
    (fresh weights first). delta_lights: DeltaLightDesc records (spot, distant, goniometric).
    textures / material_textures / rgb_to_spectrum: image textures (image_texture), per SceneDesc
    material its reflectance texture index (-1 none), a tuple (reflectance, normal map,
    strength, flip green[, bump map, bump channel, bump scale]) or a dict of MaterialTextures
    fields, and the RGB -> spectrum table (zNodes[64] then coefficients[3][64][64][64][3]).
    texture_nodes: TextureNode records (texture_node) that the *Node fields of the dicts index.
    The record keeps the arrays it points at alive."""
    e = abi.SceneExt()
    e.structSize = C.sizeof(abi.SceneExt)
    if light_bvh is not None and len(light_bvh):
        e.lightBVHNodeCount = len(light_bvh)
        e.lightBVH = light_bvh.ctypes.data
        e.lightBVHProb = light_bvh_prob
    e.wavefrontPaths = wavefront_paths
    e.blockSize = block_size
    e.flags = guide
    e._keep = [light_bvh]
    if grid_media:
        from .media import grid_array
        arr = grid_array(list(grid_media))
        e.gridMediumCount = len(arr)
        e.gridMedia = C.cast(arr, C.c_void_p)
        e._keep.append(arr)
    if delta_lights:
        arr = (abi.DeltaLightDesc * len(delta_lights))(*delta_lights)
        e.deltaLightCount = len(arr)
        e.deltaLights = C.cast(arr, C.c_void_p)
        e._keep += [arr, delta_lights]
    if textures:
        arr = (abi.ImageTextureDesc * len(textures))(*textures)
        e.textureCount = len(arr)
        e.textures = C.cast(arr, C.c_void_p)
        e._keep += [arr, textures]
    if material_textures is not None:
        mt = (abi.MaterialTextures * len(material_textures))()
        for i, t in enumerate(material_textures):
            if isinstance(t, dict):
                x = dict(MATERIAL_TEXTURES_DEFAULT, **t)
                for k, val in x.items():
                    setattr(mt[i], k, val)
                continue
            # an int (reflectance texture) or (reflectance, normal map, strength, flip green
            # [, bump map, bump channel, bump scale])
            v = (t, -1, 1.0, False) if isinstance(t, (int, np.integer)) else tuple(t)
            v = v + (-1, -1, 0.01)[len(v) - 4:] if len(v) < 7 else v
            mt[i].reflectance, mt[i].normalMap = int(v[0]), int(v[1])
            mt[i].normalStrength, mt[i].normalFlipGreen = float(v[2]), 1 if v[3] else 0
            mt[i].bumpMap, mt[i].bumpChannel, mt[i].bumpScale = int(v[4]), int(v[5]), float(v[6])
            for k in ("reflectanceNode", "bumpNode", "roughnessNodeU", "roughnessNodeV", "coatRoughnessNode",
                      "thicknessNode", "coatAlbedoNode", "sheenColorNode", "sheenRoughnessNode", "etaNode", "kNode"):
                setattr(mt[i], k, -1)
        e.materialTextureCount = len(mt)
        e.materialTextures = C.cast(mt, C.c_void_p)
        e._keep.append(mt)
    if texture_nodes:
        arr = (abi.TextureNode * len(texture_nodes))(*texture_nodes)
        e.textureNodeCount = len(arr)
        e.textureNodes = C.cast(arr, C.c_void_p)
        e._keep.append(arr)
    if rgb_to_spectrum is not None:
        table = np.ascontiguousarray(rgb_to_spectrum, np.float32)
        assert table.size == 64 + 3 * 64 ** 3 * 3
        e.rgbToSpectrum = table.ctypes.data
        e._keep.append(table)
    return e


MATERIAL_TEXTURES_DEFAULT = {"reflectance": -1, "normalMap": -1, "normalStrength": 1.0, "normalFlipGreen": 0,
                             "bumpMap": -1, "bumpChannel": -1, "bumpScale": 0.01, "reflectanceNode": -1,
                             "bumpNode": -1, "roughnessNodeU": -1, "roughnessNodeV": -1, "coatRoughnessNode": -1,
                             "thicknessNode": -1, "coatAlbedoNode": -1, "sheenColorNode": -1, "sheenRoughnessNode": -1,
                             "etaNode": -1, "kNode": -1}


def texture_node(kind: int, a: int = -1, b: int = -1, t: int = -1, channel: int = -1, value: float = 0.0,
                 frequency: float = 4.0, octaves: int = 5, turbulence: bool = False, world_space: bool = True,
                 offset=(0.0, 0.0, 0.0), uv_scale=(1.0, 1.0), uv_offset=(0.0, 0.0)) -> abi.TextureNode:
    """A TextureNode (abi.TEX_CONSTANT / TEX_IMAGE / TEX_CHECKER / TEX_NOISE / TEX_MIX); the
    defaults are the reference loader's (noise: frequency 4, 5 octaves, world space)."""
    n = abi.TextureNode()
    n.type, n.a, n.b, n.t, n.channel, n.value = kind, a, b, t, channel, value
    n.frequency, n.octaves = frequency, octaves
    n.flags = (abi.TEX_NOISE_TURBULENCE if turbulence else 0) | (abi.TEX_NOISE_WORLD if world_space else 0)
    n.offset[:] = [float(v) for v in offset]
    n.scaleU, n.scaleV = float(uv_scale[0]), float(uv_scale[1])
    n.offsetU, n.offsetV = float(uv_offset[0]), float(uv_offset[1])
    return n


def image_texture(rgb: np.ndarray, wrap: int = abi.WRAP_REPEAT, flip_v: bool = True, uv_scale=(1.0, 1.0),
                  uv_offset=(0.0, 0.0), multiplier=(1.0, 1.0, 1.0)) -> abi.ImageTextureDesc:
    """An ImageTextureDesc over rgb ((height, width, 3) float32 linear, row 0 first; kept alive by
    the record)."""
    img = np.ascontiguousarray(rgb, np.float32)
    t = abi.ImageTextureDesc()
    t.height, t.width = img.shape[0], img.shape[1]
    t.rgb = img.ctypes.data
    t.wrap, t.flipV = wrap, 1 if flip_v else 0
    t.scaleU, t.scaleV = float(uv_scale[0]), float(uv_scale[1])
    t.offsetU, t.offsetV = float(uv_offset[0]), float(uv_offset[1])
    for i in range(3):
        t.rgbScale[i] = float(multiplier[i])
    t._keep = img
    return t


def render_batch(items, config: abi.BatchConfig | None = None, stats: bool = False, device: int = 0):
    """prgpu_render_batch. items: sequence of (scene, ext or None, RenderParams-like dict, film)
    where film is a (height, width, 3) float64 C-contiguous array the samples are ADDED to, and
    the dict holds spp, first_sample, seed, max_depth, clamp. Returns BatchStats when stats."""
    arr = (abi.BatchItem * len(items))()
    keep = []
    for i, (scene, ext, p, film) in enumerate(items):
        assert film.dtype == np.float64 and film.flags["C_CONTIGUOUS"]
        arr[i].scene = _desc_ptr(scene).value
        arr[i].ext = C.addressof(ext) if ext is not None else None
        arr[i].params = abi.RenderParams(p.get("spp", 1), p.get("first_sample", 0), p.get("seed", 0),
                                         p.get("max_depth", 0), p.get("clamp", 0.0))
        arr[i].outXYZ = film.ctypes.data
        keep.append((scene, ext, film))
    st = abi.BatchStats()
    err = abi.err_buf()
    cfg = C.cast(C.pointer(config), C.c_void_p) if config is not None else None
    rc = abi.gpu_lib().prgpu_render_batch(device, len(items), C.cast(arr, C.c_void_p), cfg,
                                          C.cast(C.pointer(st), C.c_void_p), err, len(err))
    abi.check(rc, err, "prgpu_render_batch")
    return st if stats else None


def batch_config(wavefront_paths: int = 0, shade_block: int = 0, host_loop: bool = False) -> abi.BatchConfig:
    """BatchConfig; zero settings are autotuned. host_loop: the loop driven from the host (profiling)."""
    c = abi.BatchConfig()
    c.structSize = C.sizeof(abi.BatchConfig)
    c.wavefrontPaths = wavefront_paths
    c.shadeBlock = shade_block
    c.flags = 1 if host_loop else 0
    return c


def autotune_batch(items, device: int = 0) -> abi.BatchConfig:
    """prgpu_autotune_batch over the same item tuples as render_batch (films are not touched)."""
    arr = (abi.BatchItem * len(items))()
    for i, (scene, ext, p, film) in enumerate(items):
        arr[i].scene = _desc_ptr(scene).value
        arr[i].ext = C.addressof(ext) if ext is not None else None
        arr[i].params = abi.RenderParams(p.get("spp", 1), p.get("first_sample", 0), p.get("seed", 0),
                                         p.get("max_depth", 0), p.get("clamp", 0.0))
        arr[i].outXYZ = film.ctypes.data if film is not None else None
    out = abi.BatchConfig()
    err = abi.err_buf()
    rc = abi.gpu_lib().prgpu_autotune_batch(device, len(items), C.cast(arr, C.c_void_p),
                                            C.cast(C.pointer(out), C.c_void_p), err, len(err))
    abi.check(rc, err, "prgpu_autotune_batch")
    return out


AOV_ALBEDO, AOV_NORMAL, AOV_DEPTH, AOV_POSITION = range(4)


def render_aov(scene, width: int, height: int, kind: int, spp: int, seed: int = 0, through_specular: bool = False,
               d65_spectrum: int = -1, white_adaptation=None, xyz_to_rgb=None, ext: abi.SceneExt | None = None,
               device: int = 0) -> np.ndarray:
    """prgpu_render_aov: (height, width, 3) float32 guide buffer. Albedo needs the SceneDesc index
    of a D65 spectrum and the host's colour matrices (white adaptation, XYZ -> linear sRGB)."""
    p = abi.AovParams()
    p.type, p.spp, p.seed, p.throughSpecular, p.d65Spectrum = kind, spp, seed, 1 if through_specular else 0, d65_spectrum
    for dst, src in ((p.whiteAdaptation, white_adaptation), (p.xyzToRGB, xyz_to_rgb)):
        vals = np.eye(3).ravel() if src is None else np.asarray(src, np.float64).ravel()
        for i in range(9):
            dst[i] = float(vals[i])
    out = np.zeros((height, width, 3), np.float32)
    err = abi.err_buf()
    extp = C.cast(C.pointer(ext), C.c_void_p) if ext is not None else None
    rc = abi.gpu_lib().prgpu_render_aov(device, _desc_ptr(scene), extp, C.cast(C.pointer(p), C.c_void_p), abi.ptr(out),
                                        err, len(err))
    abi.check(rc, err, "prgpu_render_aov")
    return out
