"""Image reflectance textures on the GPU against the reference PathIntegrator (pr::ImageData lookup
and ImageSpectrumTexture with the albedo uplift through pr::RGBToSpectrumTable:
src/materials/texture.cpp:8-53, src/core/rgb2spec.cpp:278-305): an outdoor scene whose ground is a
diffuse quad textured by a colour image (repeat wrap, UV scale and offset, an RGB multiplier) and
one sphere with a coated diffuse textured material, from one scene file. The reference loads the
image; the module gets the same texels, the material -> texture table and the reference's own
uplift table (the file its RGBToSpectrumTable caches beside the oracle library)."""

import json
import os
import tempfile

import numpy as np
import pytest

import render_util as ru
from prgpu import abi, render

pytestmark = pytest.mark.gpu


def _uplift_table():
    import ref as oracle_ref

    oracle_ref.ref_lib()  # builds the table (cached) on first load
    path = os.path.join(oracle_ref.REF_DIR, "prender_rgb2spec_srgb_v1.bin")
    raw = np.fromfile(path, np.uint8)
    res = int(raw[8:12].view(np.int32)[0])
    assert res == 64
    return raw[12:].view(np.float32).copy()


def _texture():
    h, w = 24, 32
    v, u = np.meshgrid((np.arange(h) + 0.5) / h, (np.arange(w) + 0.5) / w, indexing="ij")
    img = np.zeros((h, w, 3), np.float32)
    check = ((np.floor(u * 4) + np.floor(v * 3)) % 2).astype(np.float32)
    img[..., 0] = 0.15 + 0.75 * check * u
    img[..., 1] = 0.2 + 0.6 * (1 - check) * v
    img[..., 2] = 0.1 + 0.5 * (u * v)
    return img


def _write_pfm(path, img):
    h, w, _ = img.shape
    with open(path, "wb") as f:
        f.write(f"PF\n{w} {h}\n-1.0\n".encode())
        f.write(np.ascontiguousarray(img[::-1], dtype="<f4").tobytes())


def test_image_textures_agree_with_reference(gpu, oracle):
    """48 x 32, depth 6: per-pixel z of the mean over 16 renders of 256 spp each side, |z| < 4 on
    >= 99.5 % of values; mean luminance within 4 standard errors."""
    w, h = 48, 32
    d = os.path.join(tempfile.gettempdir(), "prb_scenes")
    os.makedirs(d, exist_ok=True)
    img = _texture()
    pfm = os.path.join(d, "ground_tex.pfm")
    _write_pfm(pfm, img)
    doc = ru_outdoor_doc(w, h, pfm)
    path = os.path.join(d, "textures.prscene.json")
    with open(path, "w") as f:
        json.dump(doc, f)
    rs = oracle.RefScene(path)
    desc = rs.export()
    sd = abi.SceneDesc.from_address(desc)
    names = list(doc["materials"])
    # The exported material order follows first use by the objects (ground, then the spheres).
    used = []
    for o in doc["objects"]:
        if o["material"] not in used:
            used.append(o["material"])
    assert sd.materialCount == len(used), (sd.materialCount, used)
    tex_of = {"ground": 0, "tex_coat": 1}
    mat_tex = [tex_of.get(n, -1) for n in used]
    textures = [render.image_texture(img, uv_scale=(3.0, 2.0), uv_offset=(0.25, 0.1), multiplier=(1.0, 0.9, 1.1)),
                render.image_texture(img, wrap=abi.WRAP_MIRROR, uv_scale=(2.0, 2.0))]
    ext = render.make_ext(textures=textures, material_textures=mat_tex, rgb_to_spectrum=_uplift_table())
    g = np.stack([render.render_ex(desc, w, h, 256, seed=1000 + k, max_depth=6, ext=ext) / 256 for k in range(16)])
    c = np.stack([rs.render(256, 2000 + k, 6)[0].astype(np.float64) / 256 for k in range(16)])
    z = ru.z_scores(g, c)
    frac = np.mean(np.abs(z) < 4)
    mg, mc = g[..., 1].mean(axis=(1, 2)), c[..., 1].mean(axis=(1, 2))
    se = np.sqrt(mg.var(ddof=1) / len(mg) + mc.var(ddof=1) / len(mc))
    print(f"textures: frac {frac:.4f}, mean Y gpu {mg.mean():.5f} cpu {mc.mean():.5f} se {se:.5f}")
    assert frac >= 0.995, f"only {frac:.4f} of values within |z| < 4"
    assert abs(mg.mean() - mc.mean()) < 4 * se, f"mean Y gpu {mg.mean()} cpu {mc.mean()} (se {se})"
    # The textures matter: without them the module renders the exporter's average colours.
    flat = np.stack([render.render_ex(desc, w, h, 256, seed=1000 + k, max_depth=6) / 256 for k in range(4)])
    assert np.mean(np.abs(ru.z_scores(flat, c[:4])) < 4) < 0.9


def ru_outdoor_doc(w, h, pfm):
    """Ground quad (UVs 0..1) with the image texture, a plain sphere, a coated diffuse sphere with a
    mirrored-wrap texture, lit by a constant sky and a distant-free point light."""
    return {
        "textures": {"groundtex": {"type": "image", "file": pfm, "colorspace": "linear", "wrap": "repeat",
                                   "flip_v": True, "uv_scale": [3.0, 2.0], "uv_offset": [0.25, 0.1],
                                   "multiplier": [1.0, 0.9, 1.1]},
                     "coattex": {"type": "image", "file": pfm, "colorspace": "linear", "wrap": "mirror",
                                 "flip_v": True, "uv_scale": [2.0, 2.0]}},
        "materials": {"ground": {"type": "diffuse", "reflectance": {"texture": "groundtex"}},
                      "red": {"type": "diffuse", "reflectance": [0.7, 0.2, 0.15]},
                      "tex_coat": {"type": "coated_diffuse", "reflectance": {"texture": "coattex"},
                                   "coat_roughness": 0.1}},
        "media": {},
        "geometry": {"ground": {"type": "mesh", "positions": [-3, 0, -3, -3, 0, 3, 3, 0, 3, 3, 0, -3],
                                "uvs": [0, 0, 0, 1, 1, 1, 1, 0], "indices": [0, 1, 2, 0, 2, 3]},
                     "s0": {"type": "sphere", "center": [-0.8, 0.5, 0], "radius": 0.5},
                     "s1": {"type": "sphere", "center": [0.8, 0.5, 0.2], "radius": 0.5}},
        "objects": [{"name": "ground", "geometry": "ground", "material": "ground"},
                    {"name": "s0", "geometry": "s0", "material": "red"},
                    {"name": "s1", "geometry": "s1", "material": "tex_coat"}],
        "lights": {"sky": {"type": "environment", "color": [0.6, 0.7, 0.9], "intensity": 1.0},
                   "lamp": {"type": "point", "position": [0.5, 2.5, 1.5], "intensity": 3.0, "temperature": 4500}},
        "cameras": {"cam": {"type": "pinhole", "position": [0, 1.8, 3.5], "look_at": [0, 0.2, 0], "fov_y": 50}},
        "render": {"camera": "cam", "seed": 0, "film": {"width": w, "height": h, "filter": "box"},
                   "integrator": {"type": "path", "spp": 16, "max_depth": 6}},
    }


def _normal_image():
    h, w = 32, 32
    v, u = np.meshgrid((np.arange(h) + 0.5) / h, (np.arange(w) + 0.5) / w, indexing="ij")
    n = np.stack([0.6 * np.sin(2 * np.pi * 3 * u), 0.5 * np.cos(2 * np.pi * 2 * v), np.ones_like(u)], -1)
    n /= np.linalg.norm(n, axis=-1, keepdims=True)
    return ((n + 1) * 0.5).astype(np.float32)


def test_normal_maps_agree_with_reference(gpu, oracle):
    """A normal-mapped diffuse ground (strength 0.8) and a normal-mapped rough gold sphere (green
    flipped, mirror wrap), lit by a point light and a constant sky: the same z statistics as above."""
    w, h = 48, 32
    d = os.path.join(tempfile.gettempdir(), "prb_scenes")
    os.makedirs(d, exist_ok=True)
    nimg = _normal_image()
    pfm = os.path.join(d, "normal_map.pfm")
    _write_pfm(pfm, nimg)
    doc = ru_outdoor_doc(w, h, pfm)
    doc["textures"] = {"nmap": {"type": "image", "file": pfm, "colorspace": "linear", "wrap": "repeat",
                                "flip_v": True, "uv_scale": [2.0, 2.0]},
                       "nmap2": {"type": "image", "file": pfm, "colorspace": "linear", "wrap": "mirror",
                                 "flip_v": True, "uv_scale": [3.0, 1.5]}}
    doc["materials"] = {"ground": {"type": "diffuse", "reflectance": [0.6, 0.55, 0.5],
                                   "normal_map": {"texture": "nmap", "strength": 0.8}},
                        "red": {"type": "diffuse", "reflectance": [0.7, 0.2, 0.15]},
                        "tex_coat": {"type": "conductor", "metal": "Au", "roughness": 0.35,
                                     "normal_map": {"texture": "nmap2", "flip_green": True}}}
    path = os.path.join(d, "normal_maps.prscene.json")
    with open(path, "w") as f:
        json.dump(doc, f)
    rs = oracle.RefScene(path)
    desc = rs.export()
    used = []
    for o in doc["objects"]:
        if o["material"] not in used:
            used.append(o["material"])
    maps = {"ground": (-1, 0, 0.8, False), "tex_coat": (-1, 1, 1.0, True)}
    mat_tex = [maps.get(n, (-1, -1, 1.0, False)) for n in used]
    textures = [render.image_texture(nimg, uv_scale=(2.0, 2.0)),
                render.image_texture(nimg, wrap=abi.WRAP_MIRROR, uv_scale=(3.0, 1.5))]
    ext = render.make_ext(textures=textures, material_textures=mat_tex)
    g = np.stack([render.render_ex(desc, w, h, 256, seed=1000 + k, max_depth=6, ext=ext) / 256 for k in range(16)])
    c = np.stack([rs.render(256, 2000 + k, 6)[0].astype(np.float64) / 256 for k in range(16)])
    z = ru.z_scores(g, c)
    frac = np.mean(np.abs(z) < 4)
    mg, mc = g[..., 1].mean(axis=(1, 2)), c[..., 1].mean(axis=(1, 2))
    se = np.sqrt(mg.var(ddof=1) / len(mg) + mc.var(ddof=1) / len(mc))
    print(f"normal maps: frac {frac:.4f}, mean Y gpu {mg.mean():.5f} cpu {mc.mean():.5f} se {se:.5f}")
    assert frac >= 0.995, f"only {frac:.4f} of values within |z| < 4"
    assert abs(mg.mean() - mc.mean()) < 4 * se, f"mean Y gpu {mg.mean()} cpu {mc.mean()} (se {se})"
    flat = np.stack([render.render_ex(desc, w, h, 256, seed=1000 + k, max_depth=6) / 256 for k in range(4)])
    assert np.mean(np.abs(ru.z_scores(flat, c[:4])) < 4) < 0.95


def _height_image():
    h, w = 32, 32
    v, u = np.meshgrid((np.arange(h) + 0.5) / h, (np.arange(w) + 0.5) / w, indexing="ij")
    img = np.zeros((h, w, 3), np.float32)
    img[..., 0] = 0.5 + 0.5 * np.sin(2 * np.pi * 3 * u) * np.cos(2 * np.pi * 2 * v)
    img[..., 1] = 0.5 + 0.4 * np.cos(2 * np.pi * 4 * v)
    img[..., 2] = u * v
    return img


def test_bump_maps_agree_with_reference(gpu, oracle):
    """A bump-mapped diffuse ground (mean of the channels, scale 0.2, multiplier 1.5) and a rough gold
    sphere with a bump map (red channel) under a normal map (both perturbations in the reference's
    order), lit by a point light and a constant sky: the same z statistics as above."""
    w, h = 48, 32
    d = os.path.join(tempfile.gettempdir(), "prb_scenes")
    os.makedirs(d, exist_ok=True)
    himg, nimg = _height_image(), _normal_image()
    hpfm, npfm = os.path.join(d, "height_map.pfm"), os.path.join(d, "normal_map2.pfm")
    _write_pfm(hpfm, himg)
    _write_pfm(npfm, nimg)
    doc = ru_outdoor_doc(w, h, hpfm)
    doc["textures"] = {"height": {"type": "image", "file": hpfm, "wrap": "repeat", "flip_v": True,
                                  "uv_scale": [2.0, 2.0], "multiplier": 1.5},
                       "height2": {"type": "image", "file": hpfm, "wrap": "mirror", "flip_v": True,
                                   "uv_scale": [3.0, 1.5]},
                       "nmap": {"type": "image", "file": npfm, "colorspace": "linear", "wrap": "repeat",
                                "flip_v": True, "uv_scale": [1.0, 1.0]}}
    doc["materials"] = {"ground": {"type": "diffuse", "reflectance": [0.6, 0.55, 0.5],
                                   "bump_map": {"texture": "height", "scale": 0.2}},
                        "red": {"type": "diffuse", "reflectance": [0.7, 0.2, 0.15]},
                        "tex_coat": {"type": "conductor", "metal": "Au", "roughness": 0.3,
                                     "bump_map": {"texture": "height2", "channel": "r", "scale": 0.05},
                                     "normal_map": {"texture": "nmap", "strength": 0.5}}}
    path = os.path.join(d, "bump_maps.prscene.json")
    with open(path, "w") as f:
        json.dump(doc, f)
    rs = oracle.RefScene(path)
    desc = rs.export()
    used = []
    for o in doc["objects"]:
        if o["material"] not in used:
            used.append(o["material"])
    maps = {"ground": (-1, -1, 1.0, False, 0, -1, 0.2), "tex_coat": (-1, 2, 0.5, False, 1, 0, 0.05)}
    mat_tex = [maps.get(n, -1) for n in used]
    textures = [render.image_texture(himg, uv_scale=(2.0, 2.0), multiplier=(1.5, 1.5, 1.5)),
                render.image_texture(himg, wrap=abi.WRAP_MIRROR, uv_scale=(3.0, 1.5)),
                render.image_texture(nimg)]
    ext = render.make_ext(textures=textures, material_textures=mat_tex)
    g = np.stack([render.render_ex(desc, w, h, 256, seed=1000 + k, max_depth=6, ext=ext) / 256 for k in range(16)])
    c = np.stack([rs.render(256, 2000 + k, 6)[0].astype(np.float64) / 256 for k in range(16)])
    z = ru.z_scores(g, c)
    frac = np.mean(np.abs(z) < 4)
    mg, mc = g[..., 1].mean(axis=(1, 2)), c[..., 1].mean(axis=(1, 2))
    se = np.sqrt(mg.var(ddof=1) / len(mg) + mc.var(ddof=1) / len(mc))
    print(f"bump maps: frac {frac:.4f}, mean Y gpu {mg.mean():.5f} cpu {mc.mean():.5f} se {se:.5f}")
    assert frac >= 0.995, f"only {frac:.4f} of values within |z| < 4"
    assert abs(mg.mean() - mc.mean()) < 4 * se, f"mean Y gpu {mg.mean()} cpu {mc.mean()} (se {se})"
    flat = np.stack([render.render_ex(desc, w, h, 256, seed=1000 + k, max_depth=6) / 256 for k in range(4)])
    assert np.mean(np.abs(ru.z_scores(flat, c[:4])) < 4) < 0.95


def _with_albedo_spectra(rs, rgbs, kinds=None):
    """The exported scene with the RGBAlbedoSpectrum of each colour (kind 1: RGBUnboundedSpectrum)
    appended to its spectra; the appended rows' indices."""
    import ctypes as C

    import ref as oracle_ref
    from prgpu import spectra

    base = abi.SceneDesc.from_address(rs.export())
    sd = abi.SceneDesc()
    C.memmove(C.addressof(sd), C.addressof(base), C.sizeof(sd))
    old = np.ctypeslib.as_array((C.c_float * (95 * base.spectrumCount)).from_address(base.spectra)).reshape(-1, 95)
    lam = spectra.LAMBDA.astype(np.float32)
    rows = []
    for j, rgb in enumerate(rgbs):
        out = np.zeros(95, np.float32)
        kind = 0 if kinds is None else kinds[j]
        assert oracle_ref.ref_lib().prref_spectrum(kind, *[float(v) for v in rgb], None, 95, oracle_ref._p(lam),
                                                   oracle_ref._p(out)) == 0
        rows.append(out)
    table = np.ascontiguousarray(np.concatenate([old, np.stack(rows)]), np.float32)
    sd.spectra = table.ctypes.data
    sd.spectrumCount = table.shape[0]
    sd._keep = table
    return sd, list(range(base.spectrumCount, base.spectrumCount + len(rgbs)))


def test_procedural_textures_agree_with_reference(gpu, oracle):
    """Texture trees against the reference's checker / noise / mix textures: a ground whose
    reflectance is a checker of a colour and a world-space noise blend of two colours, bump-mapped by
    world-space fBm noise; a sphere whose reflectance blends an image and a colour by uv-space noise;
    a gold sphere whose roughness is a turbulence blend of 0.1 and 0.6. The same z statistics as
    above."""
    w, h = 48, 32
    d = os.path.join(tempfile.gettempdir(), "prb_scenes")
    os.makedirs(d, exist_ok=True)
    img = _texture()
    pfm = os.path.join(d, "proc_img.pfm")
    _write_pfm(pfm, img)
    doc = ru_outdoor_doc(w, h, pfm)
    c0, c1, c2, c3 = [0.8, 0.3, 0.2], [0.1, 0.2, 0.7], [0.9, 0.9, 0.6], [0.2, 0.5, 0.3]
    doc["textures"] = {
        "chk": {"type": "checker", "a": c0, "b": {"texture": "blend"}, "uv_scale": [4.0, 4.0]},
        "blend": {"type": "noise", "a": c1, "b": c2, "frequency": 3.0, "octaves": 4, "offset": [0.3, 0.1, -0.2]},
        "bump": {"type": "noise", "frequency": 2.5},
        "img": {"type": "image", "file": pfm, "colorspace": "linear", "wrap": "repeat", "flip_v": True,
                "uv_scale": [2.0, 2.0]},
        "mixed": {"type": "noise", "a": {"texture": "img"}, "b": c3, "frequency": 8.0, "octaves": 2, "space": "uv"},
        "rough": {"type": "noise", "a": 0.1, "b": 0.6, "frequency": 5.0, "octaves": 3, "space": "uv",
                  "turbulence": True},
    }
    doc["materials"] = {"ground": {"type": "diffuse", "reflectance": {"texture": "chk"},
                                   "bump_map": {"texture": "bump", "scale": 0.2}},
                        "red": {"type": "diffuse", "reflectance": {"texture": "mixed"}},
                        "tex_coat": {"type": "conductor", "metal": "Au", "roughness": {"texture": "rough"}}}
    path = os.path.join(d, "procedural.prscene.json")
    with open(path, "w") as f:
        json.dump(doc, f)
    rs = oracle.RefScene(path)
    sd, (s0, s1, s2, s3) = _with_albedo_spectra(rs, [c0, c1, c2, c3])
    T = render.texture_node
    nodes = [T(abi.TEX_CONSTANT, a=s0), T(abi.TEX_CONSTANT, a=s1), T(abi.TEX_CONSTANT, a=s2),
             T(abi.TEX_NOISE, frequency=3.0, octaves=4, offset=(0.3, 0.1, -0.2)),
             T(abi.TEX_MIX, a=1, b=2, t=3), T(abi.TEX_CHECKER, a=0, b=4, uv_scale=(4.0, 4.0)),
             T(abi.TEX_NOISE, frequency=2.5),
             T(abi.TEX_IMAGE, a=0), T(abi.TEX_CONSTANT, a=s3), T(abi.TEX_NOISE, frequency=8.0, octaves=2, world_space=False),
             T(abi.TEX_MIX, a=7, b=8, t=9),
             T(abi.TEX_CONSTANT, value=0.1), T(abi.TEX_CONSTANT, value=0.6),
             T(abi.TEX_NOISE, frequency=5.0, octaves=3, world_space=False, turbulence=True), T(abi.TEX_MIX, a=11, b=12, t=13)]
    used = []
    for o in doc["objects"]:
        if o["material"] not in used:
            used.append(o["material"])
    slots = {"ground": {"reflectanceNode": 5, "bumpNode": 6, "bumpScale": 0.2}, "red": {"reflectanceNode": 10},
             "tex_coat": {"roughnessNodeU": 14, "roughnessNodeV": 14}}
    ext = render.make_ext(textures=[render.image_texture(img, uv_scale=(2.0, 2.0))],
                          material_textures=[slots.get(n, {}) for n in used], texture_nodes=nodes,
                          rgb_to_spectrum=_uplift_table())
    g = np.stack([render.render_ex(sd, w, h, 256, seed=1000 + k, max_depth=6, ext=ext) / 256 for k in range(16)])
    c = np.stack([rs.render(256, 2000 + k, 6)[0].astype(np.float64) / 256 for k in range(16)])
    z = ru.z_scores(g, c)
    frac = np.mean(np.abs(z) < 4)
    mg, mc = g[..., 1].mean(axis=(1, 2)), c[..., 1].mean(axis=(1, 2))
    se = np.sqrt(mg.var(ddof=1) / len(mg) + mc.var(ddof=1) / len(mc))
    print(f"procedural textures: frac {frac:.4f}, mean Y gpu {mg.mean():.5f} cpu {mc.mean():.5f} se {se:.5f}")
    assert frac >= 0.995, f"only {frac:.4f} of values within |z| < 4"
    assert abs(mg.mean() - mc.mean()) < 4 * se, f"mean Y gpu {mg.mean()} cpu {mc.mean()} (se {se})"
    flat = np.stack([render.render_ex(sd, w, h, 256, seed=1000 + k, max_depth=6) / 256 for k in range(4)])
    assert np.mean(np.abs(ru.z_scores(flat, c[:4])) < 4) < 0.95


def test_textured_coats_and_sheen_agree_with_reference(gpu, oracle):
    """Texture trees in the coat and sheen slots: a coated-diffuse ground whose coat roughness (uv
    noise blend), thickness (float checker) and scattering albedo (world noise blend of two colours)
    are textured; a diffuse sphere under a sheen with a checker colour and noise roughness; a coated
    gold sphere with noise base and coat roughness. The same z statistics as above."""
    w, h = 48, 32
    d = os.path.join(tempfile.gettempdir(), "prb_scenes")
    os.makedirs(d, exist_ok=True)
    pfm = os.path.join(d, "unused_tex.pfm")
    _write_pfm(pfm, _texture())
    doc = ru_outdoor_doc(w, h, pfm)
    ca, cb, sa, sb = [0.9, 0.5, 0.3], [0.2, 0.6, 0.9], [1.0, 0.8, 0.9], [0.3, 0.9, 0.4]
    doc["textures"] = {
        "crough": {"type": "noise", "a": 0.0, "b": 0.4, "frequency": 5.0, "octaves": 3, "space": "uv"},
        "thick": {"type": "checker", "a": 0.01, "b": 0.3, "uv_scale": [3.0, 3.0]},
        "calb": {"type": "noise", "a": ca, "b": cb, "frequency": 2.0, "octaves": 4},
        "scol": {"type": "checker", "a": sa, "b": sb, "uv_scale": [4.0, 4.0]},
        "srough": {"type": "noise", "a": 0.1, "b": 0.8, "frequency": 6.0, "octaves": 3, "space": "uv"},
        "broug": {"type": "noise", "a": 0.05, "b": 0.5, "frequency": 3.0, "octaves": 2},
    }
    doc["materials"] = {
        "ground": {"type": "coated_diffuse", "reflectance": [0.6, 0.55, 0.5], "coat_roughness": {"texture": "crough"},
                   "thickness": {"texture": "thick"}, "albedo": {"texture": "calb"}, "g": 0.3},
        "red": {"type": "diffuse", "reflectance": [0.7, 0.2, 0.15],
                "sheen": {"color": {"texture": "scol"}, "roughness": {"texture": "srough"}, "weight": 1.0}},
        "tex_coat": {"type": "coated_conductor", "metal": "Au", "roughness": {"texture": "broug"},
                     "coat_roughness": {"texture": "crough"}},
    }
    path = os.path.join(d, "textured_coats.prscene.json")
    with open(path, "w") as f:
        json.dump(doc, f)
    rs = oracle.RefScene(path)
    sd, (ia, ib, isa, isb) = _with_albedo_spectra(rs, [ca, cb, sa, sb])
    T = render.texture_node
    nodes = [T(abi.TEX_CONSTANT, value=0.0), T(abi.TEX_CONSTANT, value=0.4),
             T(abi.TEX_NOISE, frequency=5.0, octaves=3, world_space=False), T(abi.TEX_MIX, a=0, b=1, t=2),
             T(abi.TEX_CONSTANT, value=0.01), T(abi.TEX_CONSTANT, value=0.3), T(abi.TEX_CHECKER, a=4, b=5, uv_scale=(3.0, 3.0)),
             T(abi.TEX_CONSTANT, a=ia), T(abi.TEX_CONSTANT, a=ib), T(abi.TEX_NOISE, frequency=2.0, octaves=4),
             T(abi.TEX_MIX, a=7, b=8, t=9),
             T(abi.TEX_CONSTANT, a=isa), T(abi.TEX_CONSTANT, a=isb), T(abi.TEX_CHECKER, a=11, b=12, uv_scale=(4.0, 4.0)),
             T(abi.TEX_CONSTANT, value=0.1), T(abi.TEX_CONSTANT, value=0.8),
             T(abi.TEX_NOISE, frequency=6.0, octaves=3, world_space=False), T(abi.TEX_MIX, a=14, b=15, t=16),
             T(abi.TEX_CONSTANT, value=0.05), T(abi.TEX_CONSTANT, value=0.5), T(abi.TEX_NOISE, frequency=3.0, octaves=2),
             T(abi.TEX_MIX, a=18, b=19, t=20)]
    used = []
    for o in doc["objects"]:
        if o["material"] not in used:
            used.append(o["material"])
    slots = {"ground": {"coatRoughnessNode": 3, "thicknessNode": 6, "coatAlbedoNode": 10},
             "red": {"sheenColorNode": 13, "sheenRoughnessNode": 17},
             "tex_coat": {"roughnessNodeU": 21, "roughnessNodeV": 21, "coatRoughnessNode": 3}}
    ext = render.make_ext(material_textures=[slots.get(n, {}) for n in used], texture_nodes=nodes)
    g = np.stack([render.render_ex(sd, w, h, 256, seed=1000 + k, max_depth=6, ext=ext) / 256 for k in range(16)])
    c = np.stack([rs.render(256, 2000 + k, 6)[0].astype(np.float64) / 256 for k in range(16)])
    z = ru.z_scores(g, c)
    frac = np.mean(np.abs(z) < 4)
    mg, mc = g[..., 1].mean(axis=(1, 2)), c[..., 1].mean(axis=(1, 2))
    se = np.sqrt(mg.var(ddof=1) / len(mg) + mc.var(ddof=1) / len(mc))
    print(f"textured coats and sheen: frac {frac:.4f}, mean Y gpu {mg.mean():.5f} cpu {mc.mean():.5f} se {se:.5f}")
    assert frac >= 0.995, f"only {frac:.4f} of values within |z| < 4"
    assert abs(mg.mean() - mc.mean()) < 4 * se, f"mean Y gpu {mg.mean()} cpu {mc.mean()} (se {se})"
    flat = np.stack([render.render_ex(sd, w, h, 256, seed=1000 + k, max_depth=6) / 256 for k in range(4)])
    assert np.mean(np.abs(ru.z_scores(flat, c[:4])) < 4) < 0.95


def test_textured_conductor_n_k_agree_with_reference(gpu, oracle):
    """Conductor n and k from texture trees of unbounded spectra: a rough conductor sphere whose n and
    k are checkers of two colours each, and a coated-conductor ground whose n and k are world-space
    noise blends (relative to the coat's IOR on the device, as the reference divides them). The
    same z statistics as above."""
    w, h = 48, 32
    d = os.path.join(tempfile.gettempdir(), "prb_scenes")
    os.makedirs(d, exist_ok=True)
    pfm = os.path.join(d, "unused_tex2.pfm")
    _write_pfm(pfm, _texture())
    doc = ru_outdoor_doc(w, h, pfm)
    ea, eb, ka, kb = [0.2, 0.4, 1.2], [1.5, 1.0, 0.5], [3.5, 2.7, 2.2], [2.0, 2.5, 3.0]
    doc["textures"] = {
        "eta_chk": {"type": "checker", "a": ea, "b": eb, "uv_scale": [4.0, 4.0]},
        "k_chk": {"type": "checker", "a": ka, "b": kb, "uv_scale": [4.0, 4.0]},
        "eta_nz": {"type": "noise", "a": ea, "b": eb, "frequency": 2.0, "octaves": 3},
        "k_nz": {"type": "noise", "a": ka, "b": kb, "frequency": 2.0, "octaves": 3},
    }
    doc["materials"] = {
        "ground": {"type": "coated_conductor", "eta": {"texture": "eta_nz"}, "k": {"texture": "k_nz"},
                   "roughness": 0.2, "coat_roughness": 0.1},
        "red": {"type": "diffuse", "reflectance": [0.7, 0.2, 0.15]},
        "tex_coat": {"type": "conductor", "eta": {"texture": "eta_chk"}, "k": {"texture": "k_chk"}, "roughness": 0.3},
    }
    path = os.path.join(d, "textured_nk.prscene.json")
    with open(path, "w") as f:
        json.dump(doc, f)
    rs = oracle.RefScene(path)
    sd, (iea, ieb, ika, ikb) = _with_albedo_spectra(rs, [ea, eb, ka, kb], kinds=[1, 1, 1, 1])
    T = render.texture_node
    nodes = [T(abi.TEX_CONSTANT, a=iea), T(abi.TEX_CONSTANT, a=ieb), T(abi.TEX_CHECKER, a=0, b=1, uv_scale=(4.0, 4.0)),
             T(abi.TEX_CONSTANT, a=ika), T(abi.TEX_CONSTANT, a=ikb), T(abi.TEX_CHECKER, a=3, b=4, uv_scale=(4.0, 4.0)),
             T(abi.TEX_NOISE, frequency=2.0, octaves=3), T(abi.TEX_MIX, a=0, b=1, t=6), T(abi.TEX_MIX, a=3, b=4, t=6)]
    used = []
    for o in doc["objects"]:
        if o["material"] not in used:
            used.append(o["material"])
    slots = {"ground": {"etaNode": 7, "kNode": 8}, "tex_coat": {"etaNode": 2, "kNode": 5}}
    ext = render.make_ext(material_textures=[slots.get(n, {}) for n in used], texture_nodes=nodes)
    g = np.stack([render.render_ex(sd, w, h, 256, seed=1000 + k, max_depth=6, ext=ext) / 256 for k in range(16)])
    c = np.stack([rs.render(256, 2000 + k, 6)[0].astype(np.float64) / 256 for k in range(16)])
    z = ru.z_scores(g, c)
    frac = np.mean(np.abs(z) < 4)
    mg, mc = g[..., 1].mean(axis=(1, 2)), c[..., 1].mean(axis=(1, 2))
    se = np.sqrt(mg.var(ddof=1) / len(mg) + mc.var(ddof=1) / len(mc))
    print(f"textured n, k: frac {frac:.4f}, mean Y gpu {mg.mean():.5f} cpu {mc.mean():.5f} se {se:.5f}")
    assert frac >= 0.998, f"only {frac:.4f} of values within |z| < 4"
    assert abs(mg.mean() - mc.mean()) < 4 * se, f"mean Y gpu {mg.mean()} cpu {mc.mean()} (se {se})"
    flat = np.stack([render.render_ex(sd, w, h, 256, seed=1000 + k, max_depth=6) / 256 for k in range(4)])
    assert np.mean(np.abs(ru.z_scores(flat, c[:4])) < 4) < 0.95


def test_textured_conductor_reflectance_agrees_with_reference(gpu, oracle):
    """The artist reflectance of reflectance-parameterised conductors from texture trees
    (ConductorMaterial::MakeBxDF, material.cpp:90-96): a rough conductor sphere whose reflectance is
    a checker of two colours and a coated-conductor ground whose reflectance is a world-space noise
    blend (not divided by the coat's IOR, material.cpp:159-163). The exported v4 materials carry
    only the first checker colour or the average colour; the trees reach the module through
    SceneExt. The same z statistics as above, and without the trees the images differ."""
    w, h = 48, 32
    d = os.path.join(tempfile.gettempdir(), "prb_scenes")
    os.makedirs(d, exist_ok=True)
    pfm = os.path.join(d, "unused_tex3.pfm")
    _write_pfm(pfm, _texture())
    doc = ru_outdoor_doc(w, h, pfm)
    ra, rb = [0.95, 0.6, 0.2], [0.3, 0.5, 0.9]
    doc["textures"] = {
        "r_chk": {"type": "checker", "a": ra, "b": rb, "uv_scale": [4.0, 4.0]},
        "r_nz": {"type": "noise", "a": ra, "b": rb, "frequency": 2.0, "octaves": 3},
    }
    doc["materials"] = {
        "ground": {"type": "coated_conductor", "reflectance": {"texture": "r_nz"}, "roughness": 0.2,
                   "coat_roughness": 0.1},
        "red": {"type": "diffuse", "reflectance": [0.7, 0.2, 0.15]},
        "tex_coat": {"type": "conductor", "reflectance": {"texture": "r_chk"}, "roughness": 0.3},
    }
    path = os.path.join(d, "textured_reflectance_conductor.prscene.json")
    with open(path, "w") as f:
        json.dump(doc, f)
    rs = oracle.RefScene(path)
    sd, (ia, ib) = _with_albedo_spectra(rs, [ra, rb])
    T = render.texture_node
    nodes = [T(abi.TEX_CONSTANT, a=ia), T(abi.TEX_CONSTANT, a=ib), T(abi.TEX_CHECKER, a=0, b=1, uv_scale=(4.0, 4.0)),
             T(abi.TEX_NOISE, frequency=2.0, octaves=3), T(abi.TEX_MIX, a=0, b=1, t=3)]
    used = []
    for o in doc["objects"]:
        if o["material"] not in used:
            used.append(o["material"])
    slots = {"ground": {"reflectanceNode": 4}, "tex_coat": {"reflectanceNode": 2}}
    ext = render.make_ext(material_textures=[slots.get(n, {}) for n in used], texture_nodes=nodes)
    g = np.stack([render.render_ex(sd, w, h, 256, seed=1000 + k, max_depth=6, ext=ext) / 256 for k in range(16)])
    c = np.stack([rs.render(256, 2000 + k, 6)[0].astype(np.float64) / 256 for k in range(16)])
    z = ru.z_scores(g, c)
    frac = np.mean(np.abs(z) < 4)
    mg, mc = g[..., 1].mean(axis=(1, 2)), c[..., 1].mean(axis=(1, 2))
    se = np.sqrt(mg.var(ddof=1) / len(mg) + mc.var(ddof=1) / len(mc))
    print(f"textured conductor reflectance: frac {frac:.4f}, mean Y gpu {mg.mean():.5f} cpu {mc.mean():.5f} se {se:.5f}")
    assert frac >= 0.998, f"only {frac:.4f} of values within |z| < 4"
    assert abs(mg.mean() - mc.mean()) < 4 * se, f"mean Y gpu {mg.mean()} cpu {mc.mean()} (se {se})"
    flat = np.stack([render.render_ex(sd, w, h, 256, seed=1000 + k, max_depth=6) / 256 for k in range(4)])
    assert np.mean(np.abs(ru.z_scores(flat, c[:4])) < 4) < 0.95
