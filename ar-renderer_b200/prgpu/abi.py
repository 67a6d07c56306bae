"""ctypes/numpy mirror of include/prgpu_api.h and include/prhost_api.h.

Array-valued fields (BVH nodes, primitives, materials, lights, spectra, media, light-BVH nodes)
are numpy structured arrays with the exact byte layout of the C structs; the fixed-size structs
(SceneDesc, Camera, Filter, RenderParams, ...) are ctypes Structures. The libraries are loaded
from the package directory; a missing library raises -- there is no fallback path.
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GPU_LIB_PATH = os.path.join(PKG, "libprender_gpu.so")
HOST_LIB_PATH = os.path.join(PKG, "libprender_host.so")

API_VERSION = 4
EXT_VERSION = 5
SPECTRUM_SAMPLES = 95
SPECTRUM_MIN = 360.0
SPECTRUM_STEP = 5.0
FILTER_BINS = 64
SHEEN_MU, SHEEN_ALPHA = 32, 16

PRIM_TRIANGLE, PRIM_SPHERE = 0, 1
MAT_DIFFUSE, MAT_CONDUCTOR, MAT_DIELECTRIC, MAT_BLACK, MAT_INTERFACE, MAT_COATED_DIFFUSE, MAT_COATED_CONDUCTOR = range(7)
FILTER_BOX, FILTER_GAUSSIAN, FILTER_BLACKMAN_HARRIS = range(3)
LIGHT_AREA, LIGHT_POINT = range(2)

# ---------------------------------------------------------------------------------------------
# numpy layouts of the array structs

F3 = ("<f4", (3,))
BVH_NODE = np.dtype({"names": ["bmin", "bmax", "offset", "nPrims", "axis", "pad"],
                     "formats": [F3, F3, "<i4", "<u2", "u1", "u1"],
                     "offsets": [0, 12, 24, 28, 30, 31], "itemsize": 32})
PRIMITIVE = np.dtype({"names": ["type", "material", "light", "mediumInside", "mediumOutside", "pad",
                                "p0", "p1", "p2", "n0", "n1", "n2", "uv", "r", "flip"],
                      "formats": ["<u4", "<i4", "<i4", "<i4", "<i4", "<u4", F3, F3, F3, F3, F3, F3,
                                  ("<f4", (6,)), "<f4", "<u4"],
                      "offsets": [0, 4, 8, 12, 16, 20, 24, 36, 48, 60, 72, 84, 96, 120, 124],
                      "itemsize": 128})
MATERIAL = np.dtype({"names": ["type", "albedo", "albedoB", "checkerScale", "eta", "k", "alphaX", "alphaY",
                               "dispersive", "thin", "coatEta", "coatAlpha", "thickness", "coatG", "coatAlbedo",
                               "coatDispersive", "coatMaxDepth", "coatSamples", "sheenColor", "sheenRoughness",
                               "sheenWeight", "pad"],
                     "formats": ["<u4", "<i4", "<i4", "<f4", "<i4", "<i4", "<f4", "<f4", "<u4", "<u4", "<i4",
                                 "<f4", "<f4", "<f4", "<i4", "<u4", "<i4", "<i4", "<i4", "<f4", "<f4", "<u4"],
                     "offsets": [4 * i for i in range(22)], "itemsize": 88})
MEDIUM = np.dtype({"names": ["sigmaA", "sigmaS", "scale", "g"], "formats": ["<i4", "<i4", "<f4", "<f4"],
                   "offsets": [0, 4, 8, 12], "itemsize": 16})
LIGHT = np.dtype({"names": ["type", "primitive", "spectrum", "scale", "position", "twoSided", "cosPower", "area",
                            "pmf", "pad"],
                  "formats": ["<u4", "<i4", "<i4", "<f4", F3, "<u4", "<f4", "<f4", "<f4", "<u4"],
                  "offsets": [0, 4, 8, 12, 16, 28, 32, 36, 40, 44], "itemsize": 48})
SPECTRUM = np.dtype(("<f4", (SPECTRUM_SAMPLES,)))
LIGHT_BVH_NODE = np.dtype({"names": ["bmin", "bmax", "w", "phi", "cosThetaO", "cosThetaE", "twoSided", "child1",
                                     "light", "parent", "pad"],
                           "formats": [F3, F3, F3, "<f4", "<f4", "<f4", "<i4", "<i4", "<i4", "<i4", ("<i4", (2,))],
                           "offsets": [0, 12, 24, 36, 40, 44, 48, 52, 56, 60, 64], "itemsize": 72})
RAY = np.dtype({"names": ["o", "tMax", "d", "pad"], "formats": [F3, "<f4", F3, "<f4"],
                "offsets": [0, 12, 16, 28], "itemsize": 32})


# ---------------------------------------------------------------------------------------------
# ctypes structs

class Float3(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float)]


class Camera(C.Structure):
    _fields_ = [("cameraToWorld", C.c_float * 12), ("tanHalfFov", C.c_float), ("aspect", C.c_float),
                ("lensRadius", C.c_float), ("focalDistance", C.c_float), ("width", C.c_int32),
                ("height", C.c_int32), ("margin", C.c_int32), ("pad", C.c_uint32)]


class Filter(C.Structure):
    _fields_ = [("type", C.c_uint32), ("radius", C.c_float), ("sigma", C.c_float), ("norm", C.c_float),
                ("cdf", C.c_float * (FILTER_BINS + 1))]


class SceneDesc(C.Structure):
    _fields_ = [("apiVersion", C.c_int32), ("nodes", C.c_void_p), ("nodeCount", C.c_int32),
                ("primOrder", C.c_void_p), ("prims", C.c_void_p), ("primCount", C.c_int32),
                ("materials", C.c_void_p), ("materialCount", C.c_int32), ("lights", C.c_void_p),
                ("lightCount", C.c_int32), ("spectra", C.c_void_p), ("spectrumCount", C.c_int32),
                ("media", C.c_void_p), ("mediumCount", C.c_int32), ("cameraMedium", C.c_int32),
                ("envSpectrum", C.c_int32), ("envScale", C.c_float), ("envPmf", C.c_float),
                ("worldCenter", Float3), ("worldRadius", C.c_float), ("camera", Camera), ("filter", Filter),
                ("sheenAlbedo", C.c_void_p), ("cie", C.c_void_p), ("cieYIntegral", C.c_float)]


class RenderParams(C.Structure):
    _fields_ = [("spp", C.c_int32), ("firstSample", C.c_int32), ("seed", C.c_uint64), ("maxDepth", C.c_int32),
                ("clampLuminance", C.c_float)]


class DeviceInfo(C.Structure):
    _fields_ = [("name", C.c_char * 256), ("globalMemory", C.c_uint64), ("computeUnits", C.c_int32),
                ("isGpu", C.c_int32), ("backend", C.c_char * 32)]


class GridMediumDesc(C.Structure):
    _fields_ = [("sigmaA", C.c_int32), ("sigmaS", C.c_int32), ("scale", C.c_float), ("g", C.c_float),
                ("worldToMedium", C.c_float * 12), ("boundsMin", C.c_float * 3), ("boundsMax", C.c_float * 3),
                ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("maxDensity", C.c_float),
                ("density", C.c_void_p), ("field", C.c_uint32), ("noiseOctaves", C.c_int32),
                ("noiseFrequency", C.c_float), ("noiseThreshold", C.c_float), ("noiseSharpness", C.c_float),
                ("noiseFalloff", C.c_uint32), ("noiseOffset", C.c_float * 3), ("indexOrigin", C.c_int32 * 3)]


GRID_VOXELS, GRID_NOISE, GRID_INDEXED = 0, 1, 2


class EnvMapDesc(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("texels", C.c_void_p), ("illuminant", C.c_int32),
                ("scale", C.c_float), ("rotationDeg", C.c_float), ("pmf", C.c_float)]


class SunDesc(C.Structure):
    _fields_ = [("direction", C.c_float * 3), ("cosThetaMax", C.c_float), ("spectrum", C.c_int32),
                ("scale", C.c_float), ("pmf", C.c_float)]


DELTA_SPOT, DELTA_DISTANT, DELTA_GONIOMETRIC = range(3)


class DeltaLightDesc(C.Structure):
    _fields_ = [("type", C.c_uint32), ("spectrum", C.c_int32), ("scale", C.c_float), ("pmf", C.c_float),
                ("position", C.c_float * 3), ("direction", C.c_float * 3), ("cosFalloffStart", C.c_float),
                ("cosFalloffEnd", C.c_float), ("frame", C.c_float * 9), ("nV", C.c_int32), ("nH", C.c_int32),
                ("pad", C.c_int32), ("profile", C.c_void_p)]


WRAP_REPEAT, WRAP_CLAMP, WRAP_MIRROR = range(3)


class ImageTextureDesc(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("rgb", C.c_void_p), ("wrap", C.c_uint32),
                ("flipV", C.c_uint32), ("scaleU", C.c_float), ("scaleV", C.c_float), ("offsetU", C.c_float),
                ("offsetV", C.c_float), ("rgbScale", C.c_float * 3), ("pad", C.c_uint32)]


class MaterialTextures(C.Structure):
    _fields_ = [("reflectance", C.c_int32), ("normalMap", C.c_int32), ("normalStrength", C.c_float),
                ("normalFlipGreen", C.c_uint32), ("bumpMap", C.c_int32), ("bumpChannel", C.c_int32),
                ("bumpScale", C.c_float), ("reflectanceNode", C.c_int32), ("bumpNode", C.c_int32),
                ("roughnessNodeU", C.c_int32), ("roughnessNodeV", C.c_int32), ("coatRoughnessNode", C.c_int32),
                ("thicknessNode", C.c_int32), ("coatAlbedoNode", C.c_int32), ("sheenColorNode", C.c_int32),
                ("sheenRoughnessNode", C.c_int32), ("etaNode", C.c_int32), ("kNode", C.c_int32)]


TEX_CONSTANT, TEX_IMAGE, TEX_CHECKER, TEX_NOISE, TEX_MIX = 0, 1, 2, 3, 4
TEX_NOISE_TURBULENCE, TEX_NOISE_WORLD = 1, 2


class TextureNode(C.Structure):
    _fields_ = [("type", C.c_uint32), ("a", C.c_int32), ("b", C.c_int32), ("t", C.c_int32), ("channel", C.c_int32),
                ("value", C.c_float), ("frequency", C.c_float), ("octaves", C.c_int32), ("flags", C.c_uint32),
                ("offset", C.c_float * 3), ("scaleU", C.c_float), ("scaleV", C.c_float), ("offsetU", C.c_float),
                ("offsetV", C.c_float)]


class SceneExt(C.Structure):
    _fields_ = [("structSize", C.c_uint32), ("lightBVHNodeCount", C.c_int32), ("lightBVH", C.c_void_p),
                ("lightBVHProb", C.c_float), ("wavefrontPaths", C.c_int32), ("blockSize", C.c_int32),
                ("flags", C.c_int32), ("gridMediumCount", C.c_int32), ("gridMedia", C.c_void_p),
                ("envMap", C.c_void_p), ("sun", C.c_void_p), ("deltaLightCount", C.c_int32), ("pad", C.c_int32),
                ("deltaLights", C.c_void_p), ("textureCount", C.c_int32), ("materialTextureCount", C.c_int32),
                ("textures", C.c_void_p), ("materialTextures", C.c_void_p), ("rgbToSpectrum", C.c_void_p),
                ("textureNodes", C.c_void_p), ("textureNodeCount", C.c_int32), ("pad2", C.c_int32),
                ("rayTap", C.c_void_p), ("rayTapPaths", C.c_int32), ("rayTapBounces", C.c_int32)]


class BatchItem(C.Structure):
    _fields_ = [("scene", C.c_void_p), ("ext", C.c_void_p), ("params", RenderParams), ("outXYZ", C.c_void_p)]


class BatchConfig(C.Structure):
    _fields_ = [("structSize", C.c_uint32), ("wavefrontPaths", C.c_int32), ("shadeBlock", C.c_int32),
                ("flags", C.c_int32)]


class AovParams(C.Structure):
    _fields_ = [("type", C.c_int32), ("spp", C.c_int32), ("seed", C.c_uint64), ("throughSpecular", C.c_int32),
                ("d65Spectrum", C.c_int32), ("whiteAdaptation", C.c_float * 9), ("xyzToRGB", C.c_float * 9)]


class CheckpointHeader(C.Structure):
    _fields_ = [("integrator", C.c_uint32), ("maxDepth", C.c_int32), ("width", C.c_int32), ("height", C.c_int32),
                ("chains", C.c_int32), ("fingerprint", C.c_uint64), ("seed", C.c_uint64)]


class BatchStats(C.Structure):
    _fields_ = [("pathSamples", C.c_uint64), ("closestRays", C.c_uint64), ("shadowRays", C.c_uint64),
                ("waves", C.c_uint64), ("loopIterations", C.c_uint64), ("deviceMs", C.c_double),
                ("hostMs", C.c_double), ("wavefrontPaths", C.c_int32), ("shadeBlock", C.c_int32),
                ("graphBuilt", C.c_int32), ("tuned", C.c_int32)]


class GuideOptions(C.Structure):
    _fields_ = [("maxSelect", C.c_float), ("logKappaMax", C.c_float), ("selectLoss", C.c_int32),
                ("trainPasses", C.c_int32), ("bands", C.c_int32), ("weightClamp", C.c_float)]


class RenderStats(C.Structure):
    _fields_ = [("pathSamples", C.c_uint64), ("closestRays", C.c_uint64), ("shadowRays", C.c_uint64),
                ("bounces", C.c_uint64), ("kernelLaunches", C.c_uint64), ("deviceMs", C.c_double),
                ("traceMs", C.c_double), ("shadowMs", C.c_double), ("shadeMs", C.c_double),
                ("filmMs", C.c_double)]


assert C.sizeof(Camera) == 80 and C.sizeof(Filter) == 276 and C.sizeof(SceneDesc) == 520
assert C.sizeof(RenderParams) == 24 and C.sizeof(DeviceInfo) == 304
assert C.sizeof(GridMediumDesc) == 160 and C.sizeof(SceneExt) == 144 and C.sizeof(DeltaLightDesc) == 104
assert C.sizeof(ImageTextureDesc) == 56 and C.sizeof(MaterialTextures) == 72 and C.sizeof(TextureNode) == 64
assert C.sizeof(AovParams) == 96
assert C.sizeof(EnvMapDesc) == 32 and C.sizeof(SunDesc) == 28
assert C.sizeof(BatchItem) == 48 and C.sizeof(BatchConfig) == 16 and C.sizeof(BatchStats) == 72
assert SceneDesc.camera.offset == 140 and SceneDesc.filter.offset == 220 and SceneDesc.cieYIntegral.offset == 512

# ---------------------------------------------------------------------------------------------
# Library loading

_P = C.c_void_p
_ERR = [C.c_char_p, C.c_int]
_gpu = None
_host = None


def _bind(lib, name, argtypes, restype) -> None:
    """Declare a prototype; symbols the library does not export are left unbound (calling them
    raises AttributeError), and tests/test_abi.py checks the export list against the headers."""
    if hasattr(lib, name):
        f = getattr(lib, name)
        f.argtypes = argtypes
        f.restype = restype


def gpu_lib() -> C.CDLL:
    """The CUDA module. Raises if it has not been built."""
    global _gpu
    if _gpu is None:
        if not os.path.exists(GPU_LIB_PATH):
            raise RuntimeError(f"{GPU_LIB_PATH} is missing: run ar-renderer_b200/build.py")
        lib = C.CDLL(GPU_LIB_PATH)
        _bind(lib, "prgpu_api_version", [], C.c_int)
        _bind(lib, "prgpu_ext_version", [], C.c_int)
        _bind(lib, "prgpu_launch_count", [], C.c_uint64)
        _bind(lib, "prgpu_list_devices", [_P, C.c_int], C.c_int)
        _bind(lib, "prgpu_render", [C.c_int, _P, _P, _P, *_ERR], C.c_int)
        _bind(lib, "prgpu_render_ex", [C.c_int, _P, _P, _P, _P, _P, *_ERR], C.c_int)
        _bind(lib, "prgpu_render_batch", [C.c_int, C.c_int32, _P, _P, _P, *_ERR], C.c_int)
        _bind(lib, "prgpu_autotune_batch", [C.c_int, C.c_int32, _P, _P, *_ERR], C.c_int)
        _bind(lib, "prgpu_guide_set_weights", [C.c_int, _P, *_ERR], C.c_int)
        _bind(lib, "prgpu_guide_get_weights", [C.c_int, _P, *_ERR], C.c_int)
        _bind(lib, "prgpu_guide_infer", [C.c_int, C.c_int64, _P, _P, *_ERR], C.c_int)
        _bind(lib, "prgpu_guide_gradient", [C.c_int, C.c_int64, _P, _P, _P, _P, *_ERR], C.c_int)
        _bind(lib, "prgpu_guide_adam_step", [C.c_int, C.c_float, C.c_float, *_ERR], C.c_int)
        _bind(lib, "prgpu_guide_stats", [C.c_int, _P, *_ERR], C.c_int)
        _bind(lib, "prgpu_guide_set_learning_rate", [C.c_int, C.c_float, *_ERR], C.c_int)
        _bind(lib, "prgpu_guide_set_options", [C.c_int, _P, *_ERR], C.c_int)
        _bind(lib, "prgpu_guide_get_options", [C.c_int, _P, *_ERR], C.c_int)
        _bind(lib, "prgpu_trace_rays", [C.c_int, _P, C.c_int32, _P, _P, C.c_int32, _P, C.c_int64, C.c_int32,
                                        _P, _P, _P, _P, *_ERR], C.c_int)
        _bind(lib, "prgpu_trace_rays_noalloc", [C.c_int, _P, C.c_int32, _P, _P, C.c_int32, _P, C.c_int64,
                                                C.c_int32, _P, _P, _P, _P, *_ERR], C.c_int)
        _bind(lib, "prgpu_accel_create", [C.c_int, _P, C.c_int32, _P, _P, C.c_int32, C.POINTER(_P), *_ERR], C.c_int)
        _bind(lib, "prgpu_accel_trace", [_P, _P, C.c_int64, C.c_int32, _P, _P, _P, *_ERR], C.c_int)
        _bind(lib, "prgpu_accel_trace_host", [_P, _P, C.c_int64, C.c_int32, _P, _P, *_ERR], C.c_int)
        _bind(lib, "prgpu_accel_status", [_P], C.c_int)
        _bind(lib, "prgpu_accel_bytes", [_P], C.c_int64)
        _bind(lib, "prgpu_accel_destroy", [_P], None)
        _bind(lib, "prgpu_eval_bxdf", [C.c_int, C.c_int, _P, C.c_int64, _P, _P, *_ERR], C.c_int)
        _bind(lib, "prgpu_eval_full_bsdf", [C.c_int, _P, _P, C.c_int64, _P, _P, *_ERR], C.c_int)
        _bind(lib, "prgpu_sheen_albedo_table", [_P], None)
        _bind(lib, "prgpu_render_aov", [C.c_int, _P, _P, _P, _P, *_ERR], C.c_int)
        _bind(lib, "prgpu_eval_phase", [C.c_int, C.c_int64, _P, _P, *_ERR], C.c_int)
        _bind(lib, "prgpu_eval_homogeneous", [C.c_int, C.c_int64, _P, _P, *_ERR], C.c_int)
        _bind(lib, "prgpu_eval_light_bvh", [C.c_int, _P, C.c_int32, C.c_int32, C.c_float, C.c_int64, _P, _P, _P,
                                            *_ERR], C.c_int)
        _gpu = lib
    return _gpu


def host_lib() -> C.CDLL:
    global _host
    if _host is None:
        if not os.path.exists(HOST_LIB_PATH):
            raise RuntimeError(f"{HOST_LIB_PATH} is missing: run ar-renderer_b200/build.py")
        lib = C.CDLL(HOST_LIB_PATH)
        lib.prhost_build_bvh.argtypes = [_P, _P, C.c_int64, C.c_int32, C.c_int32, _P, _P]
        lib.prhost_build_bvh.restype = C.c_int64
        lib.prhost_build_bvh_triangles.argtypes = [_P, C.c_int64, C.c_int32, C.c_int32, _P, _P]
        lib.prhost_build_bvh_triangles.restype = C.c_int64
        lib.prhost_build_light_bvh.argtypes = [_P, C.c_int32, _P]
        lib.prhost_build_light_bvh.restype = C.c_int32
        lib.prhost_preetham_sky.argtypes = [_P, C.c_float, C.c_float, C.c_int32, C.c_int32, _P]
        lib.prhost_preetham_sky.restype = C.c_int
        lib.prhost_sun_radiance.argtypes = [_P, C.c_float, C.c_float, C.c_int64, _P, _P]
        lib.prhost_sun_radiance.restype = C.c_int
        lib.prhost_rgb_to_sigmoid.argtypes = [C.c_int64, _P, _P, C.c_int32, _P]
        lib.prhost_rgb_to_sigmoid.restype = C.c_int
        lib.prhost_checkpoint_write.argtypes = [C.c_char_p, _P, _P, C.c_uint64, _P, C.c_uint64, C.c_char_p, C.c_int]
        lib.prhost_checkpoint_write.restype = C.c_int
        lib.prhost_checkpoint_read.argtypes = [C.c_char_p, _P, _P, C.c_uint64, _P, C.c_uint64, C.POINTER(C.c_uint64),
                                               C.c_char_p, C.c_int]
        lib.prhost_checkpoint_read.restype = C.c_int
        _host = lib
    return _host


def ptr(a) -> C.c_void_p | None:
    """Address of a contiguous numpy array (None for None)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "arrays passed across the C ABI must be contiguous"
    return C.c_void_p(a.ctypes.data)


class PrgpuError(RuntimeError):
    pass


def err_buf():
    return C.create_string_buffer(1024)


def check(rc: int, err, what: str) -> None:
    if rc != 0:
        raise PrgpuError(f"{what} failed: {err.value.decode(errors='replace')}")
