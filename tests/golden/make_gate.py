"""Writes tests/golden/gate_c0.npz: the 65,536-spp CPU reference of the unbiasedness gate.

The reference PathIntegrator (src/integrators/path.cpp:113-238, compiled from the reference sources
into oracle/_ref/libprref.so) renders the box-and-spheres scene at 256 x 256, depth 8, box filter,
16 times with seeds 9000..9015 at 4,096 spp each (16 x 4,096 = 65,536 spp). The fixture keeps, per
pixel and XYZ channel, the mean of the 16 per-seed mean images and their variance across seeds
(ddof 1): the statistics tests/test_quality.cpp:146-173 of the reference forms from independent
seeds, since the film stores no second moment. A GPU test then compares its own 16 seeds against
these without re-running the CPU render (which takes about 75 minutes on 8 cores).

Run from the repository root:  python tests/golden/make_gate.py  [--spp 4096 --seeds 16]
Per-seed partial images are cached under the system temp directory, so an interrupted run resumes.
"""

import argparse
import hashlib
import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "ar-renderer_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]

import ref  # noqa: E402
import render_util as ru  # noqa: E402

SIDE = 256
DEPTH = 8
SEED0 = 9000


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--spp", type=int, default=4096)
    ap.add_argument("--seeds", type=int, default=16)
    ap.add_argument("--out", default=os.path.join(HERE, "gate_c0.npz"))
    args = ap.parse_args()
    ref.set_threads(0)
    path = ru.scene_file("gate_c0", seed=0, width=SIDE, height=SIDE)
    with open(path, "rb") as f:
        scene_sha = hashlib.sha256(f.read()).hexdigest()[:16]
    cache = os.path.join(tempfile.gettempdir(), "prb_gate_c0", f"{scene_sha}_{args.spp}")
    os.makedirs(cache, exist_ok=True)
    rs = ref.RefScene(path)
    imgs = []
    for k in range(args.seeds):
        part = os.path.join(cache, f"seed{SEED0 + k}.npy")
        if os.path.exists(part):
            imgs.append(np.load(part))
            continue
        t0 = time.time()
        img, _ = rs.render(args.spp, SEED0 + k, DEPTH)
        img = img.astype(np.float64) / args.spp
        np.save(part, img)
        imgs.append(img)
        print(f"seed {SEED0 + k}: {time.time() - t0:.0f} s", flush=True)
    rs.close()
    c = np.stack(imgs)
    np.savez_compressed(args.out, mean=c.mean(0).astype(np.float32), var=c.var(0, ddof=1).astype(np.float32),
                        mean_y=np.float64(c[..., 1].mean()), seeds=np.int32(args.seeds), spp=np.int32(args.spp),
                        first_seed=np.int32(SEED0), side=np.int32(SIDE), depth=np.int32(DEPTH),
                        threads=np.int32(ref.thread_count()), scene_sha=scene_sha)
    print("wrote", args.out, "mean Y", c[..., 1].mean())


if __name__ == "__main__":
    main()
