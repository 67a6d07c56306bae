"""The drop-in through the reference's own host program: PRender's CLI (src/cli/main.cpp and pr_core,
compiled from the reference sources by oracle/Makefile's `prender` target) with the dlopen branch
of INTEGRATION.md in its module loader, running `--integrator path --device gpu` on this
repository's libprender_gpu.so. The reference's own exporter (gpu_path.cpp:106-456) flattens the
scene and its own progressive loop (gpu_path.cpp:458-509) calls prgpu_render; the images are
compared with `--device cpu` renders of the same scene by the same binary (PathIntegrator,
src/integrators/path.cpp:113-238), per-pixel z over independent seeds (the pattern of the
reference's tests/test_quality.cpp:146-173)."""

import os
import shutil
import subprocess

import numpy as np
import pytest

import render_util as ru

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PRENDER = os.path.join(ROOT, "oracle", "_ref", "prender")
TABLE = os.path.join(ROOT, "oracle", "_ref", "prender_rgb2spec_srgb_v1.bin")


def read_pfm(path: str) -> np.ndarray:
    with open(path, "rb") as f:
        kind = f.readline().strip()
        w, h = (int(x) for x in f.readline().split())
        scale = float(f.readline().strip())
        data = np.frombuffer(f.read(), dtype="<f4" if scale < 0 else ">f4")
    assert kind == b"PF"
    return data.reshape(h, w, 3)[::-1].astype(np.float64)


@pytest.fixture(scope="module")
def cli_env(tmp_path_factory):
    if not os.path.exists(PRENDER):
        pytest.fail(f"{PRENDER} is missing: build it with `make -C oracle prender` where the reference tree exists")
    cache = tmp_path_factory.mktemp("prender_cache")
    os.makedirs(cache / "prender", exist_ok=True)
    if os.path.exists(TABLE):  # the reference's RGB -> spectrum table, so each run skips rebuilding it
        shutil.copy(TABLE, cache / "prender" / os.path.basename(TABLE))
    env = dict(os.environ, LOCALAPPDATA=str(cache),
               LD_LIBRARY_PATH=os.path.join(ROOT, "ar-renderer_b200") + os.pathsep + os.environ.get("LD_LIBRARY_PATH", ""))
    return env


def _run(env, *args):
    r = subprocess.run([PRENDER, *args], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout + r.stderr


def test_list_devices_shows_the_cuda_module(gpu, cli_env):
    out = _run(cli_env, "--list-devices")
    assert "gpu:0" in out and "cuda" in out, out
    assert "GPU:" not in out, out  # the loader's status line appears only when the module failed


def test_reference_cli_gpu_render_agrees_with_its_cpu_render(gpu, cli_env, tmp_path):
    w = h = 48
    scene = ru.scene_file("cli_box", seed=0, width=w, height=h)
    seeds, spp = 12, 256
    g, c = [], []
    for k in range(seeds):
        out = str(tmp_path / f"g{k}.pfm")
        log = _run(cli_env, scene, "--integrator", "path", "--device", "gpu", "--spp", str(spp), "--seed", str(100 + k),
                   "--max-depth", "8", "--out", out, "--quiet")
        assert "rendering on the CPU" not in log and "failed" not in log, log
        g.append(read_pfm(out))
        out = str(tmp_path / f"c{k}.pfm")
        _run(cli_env, scene, "--integrator", "path", "--device", "cpu", "--spp", str(spp), "--seed", str(500 + k),
             "--max-depth", "8", "--out", out, "--quiet")
        c.append(read_pfm(out))
    g, c = np.stack(g), np.stack(c)
    assert g.shape == (seeds, h, w, 3) and np.isfinite(g).all()
    z = ru.z_scores(g, c)
    frac = np.mean(np.abs(z) < 4)
    lum = np.array([0.2126729, 0.7151522, 0.0721750])
    mg, mc = (g @ lum).mean(axis=(1, 2)), (c @ lum).mean(axis=(1, 2))
    se = np.sqrt(mg.var(ddof=1) / seeds + mc.var(ddof=1) / seeds)
    print(f"prender --device gpu vs cpu: frac {frac:.4f}, mean Y {mg.mean():.5f} vs {mc.mean():.5f} (se {se:.5f})")
    assert frac >= 0.995, f"only {frac:.4f} of values within |z| < 4"
    assert abs(mg.mean() - mc.mean()) < 4 * se, (mg.mean(), mc.mean(), se)
