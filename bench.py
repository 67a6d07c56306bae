"""Benchmark of the B200 path-tracing module (one JSON line on stdout, rank 0).

Workload (default): the traversal microbenchmark -- 2^24 rays against a 1,048,576-triangle soup
(centroids uniform in the unit cube, vertex offsets uniform in [-0.01, 0.01]^3; ray origins
uniform in [-0.5, 1.5]^3, directions uniform on the sphere), one closest-hit pass (tMax = inf,
primitive id + distance out) and one any-hit pass (tMax uniform in [0, 2]) per step. Synthetic,
seeded inputs; the BVH is this library's own SAH build (libprender_host.so).

  value  -- Mrays/s of both passes with rays resident in HBM (device time, CUDA events on the
            launching stream, max over ranks); inputs are 1 GiB per step, larger than L2.
  e2e    -- the same through prgpu_accel_trace_host with pinned HOST rays and results: the
            host->device copy of the rays and device->host copy of the hits are inside the
            timed region.
  roofline -- the closest-hit kernel: algorithmic bytes per launch (per-ray node, triangle, ray
            and hit bytes with per-ray work counts measured once on the CPU oracle) over its
            CUDA-event duration, against the measured HBM copy bandwidth.
  cpu_baseline -- the reference's own BVH::Intersect / IntersectP (oracle/_ref, compiled from the
            reference sources) on a bounded sample of the same rays, all host threads.

--impl reference prints the reference CPU traversal as its own arm (rank 0 only).
Multi-GPU (torchrun): each rank traces its own 2^24 rays (weak scaling, no data-path collective).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.join(ROOT, "ar-renderer_b200"), os.path.join(ROOT, "oracle")]

import numpy as np  # noqa: E402

N_TRIS = 1 << 20
N_RAYS = 1 << 24
METRIC = "path samples/s; equal-time relMSE guided vs plain (same B200); Mrays/s"

# Per-ray work of the closest-hit pass on this workload: the reference's own BVH traversal
# (pr::BVH::Intersect over the reference's tree), counted once with the oracle's counting traversal
# (oracle/restate.c) over 2^18 of the benchmark rays by oracle/measure_trace_work.py: mean node
# visits and triangle tests per ray. The device kernel, whatever tree it runs on, is credited with
# this work.
NODES_PER_RAY = 28.86
TRIS_PER_RAY = 2.92
# Algorithmic bytes per closest-hit ray: every visited node (32 B in the reference layout) and
# every tested triangle (36 B) read once, the 32-byte ray read and an 8-byte hit written.
BYTES_PER_RAY = 32 * NODES_PER_RAY + 36 * TRIS_PER_RAY + 32 + 8
# DRAM bytes per closest-hit launch: dram__bytes_read.sum + dram__bytes_write.sum of this kernel
# in one ncu capture of a 2^22-ray launch of this workload (a full 2^24-ray launch is too large to
# capture), scaled by the rays of a full launch. Not measured by this run; the JSON says so.
NCU_TRAFFIC_PER_LAUNCH = (664.852480e6 + 42.621440e6) * 4
# Plain path tracer (box scene, 256^2, depth 8): algorithmic bytes per path sample,
# N_closest B_ray + N_shadow B_shadow + 24 B of film, with the reference traversal's per-ray node
# and triangle counts on the rays the GPU traces for a seeded 2^16-path subset
# (oracle/measure_path_work.py): 4.266 closest rays of 1,567 B and 2.805 shadow rays of 755 B.
PT_BYTES_PER_SAMPLE = 4.266 * 1567.27 + 2.805 * 754.97 + 24
# L2 hit rate of the path tracer's closest-hit kernel on that scene (ncu lts__t_sector_hit_rate of
# k_extend, first bounce of a 128^2 x 64 spp render): the scene (about 9 MB) stays in L2.
PT_L2_HIT_RATE = 0.708


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown," \
             "clocks_event_reasons.sw_power_cap"

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "50"], stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        try:
            self.file.flush()
            rows = [l.split(", ") for l in open(self.file.name).read().splitlines() if l.strip()]
        except Exception:
            rows = []
        rows = [r for r in rows if len(r) >= 9 and r[0].strip() == str(self.gpu)]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def bench_config(world: int) -> dict:
    """The workload both arms run (ours on the GPU, the reference's on the host cores): the same
    triangles and rays per pass; each arm traverses its own BVH."""
    return {"workload": "traversal microbenchmark: 2^24 rays vs 1,048,576-triangle soup, closest + any-hit",
            "rays_per_pass": N_RAYS, "triangles": N_TRIS, "l2": "inputs larger than L2 (1 GiB of rays per step)",
            "parallelism": f"replicas x{world}"}


def max_over_ranks(values, world: int, device: str = "cuda"):
    """Element-wise maximum of this rank's timings over all ranks: a multi-GPU step takes as long as
    its slowest rank. One all-reduce on the process group (NCCL for the GPUs, gloo in the CPU test)."""
    vals = [float(v) for v in values]
    if world <= 1:
        return vals
    import torch
    import torch.distributed as dist

    x = torch.tensor(vals, device=device, dtype=torch.float64)
    dist.all_reduce(x, op=dist.ReduceOp.MAX)
    return [float(v) for v in x.tolist()]


def whole_job_mrays(world: int, rays_per_rank: int, seconds: float) -> float:
    """Mrays/s of the whole job: every rank traces its own rays_per_rank in `seconds` (the maximum
    over ranks), so the job's rate is world times one rank's rays over that time (weak scaling)."""
    return world * rays_per_rank / seconds / 1e6


def make_inputs(rank: int):
    from prgpu import trace, workloads

    verts = workloads.triangle_soup(N_TRIS, seed=1)
    closest = workloads.soup_rays(N_RAYS, seed=2 + 1000 * rank)
    anyhit = workloads.soup_rays(N_RAYS, seed=3 + 1000 * rank, any_hit=True)
    return verts, closest, anyhit, trace


def cpu_reference(verts, closest, anyhit, rays_per_pass: int):
    """Reference CPU traversal (oracle/_ref) on the first rays_per_pass rays of each pass."""
    import ref
    from prgpu import workloads

    ref.set_threads(0)
    b = ref.SoupBVH(verts)
    c = workloads.rays_as_f8(closest[:rays_per_pass])
    a = workloads.rays_as_f8(anyhit[:rays_per_pass])
    b.trace(c[: 1 << 14])  # warm the pool
    *_, t1 = b.trace(c)
    _, t2 = b.trace(a, any_hit=True)
    b.close()
    return 2 * rays_per_pass / (t1 + t2) / 1e6, ref.thread_count(), t1 + t2


def path_tracer_bench(args, device: int, cpu: bool):
    """The plain path tracer on the box scene (256 x 256, 64 spp, 4 hero wavelengths, max depth 8,
    44,814 primitives), built by this library's host side (prgpu.hostscene) and rendered through
    prgpu_render_ex. value = path samples/s of device time; e2e = the v4 prgpu_render call with a
    host SceneDesc and host film (scene upload cached after the first call, film copied out each
    step); cpu_baseline = the reference PathIntegrator (oracle/_ref) on the same scene."""
    from prgpu import abi, hostscene, render, scenes

    s = scenes.box_scene(seed=0, width=args.pt_res, height=args.pt_res, spp=64, max_depth=8)
    h = hostscene.build_box_scene(s)
    desc = h.desc()
    w, hh, spp = s.width, s.height, s.spp
    for _ in range(args.warmup):
        render.render_ex(desc, w, hh, spp, seed=1, max_depth=8)
    dev_ms, wall = [], []
    for k in range(args.steps):
        t0 = time.perf_counter()
        _, st = render.render_ex(desc, w, hh, spp, first_sample=k * spp, seed=1, max_depth=8, stats=True)
        wall.append(time.perf_counter() - t0)
        dev_ms.append(st.deviceMs)
    samples = w * hh * spp
    film = np.zeros((hh, w, 3), np.float32)
    render.render_v4(desc, w, hh, spp, seed=1, max_depth=8, out=film)
    t0 = time.perf_counter()
    for k in range(args.steps):
        render.render_v4(desc, w, hh, spp, first_sample=k * spp, seed=1, max_depth=8, out=film)
    e2e_s = (time.perf_counter() - t0) / args.steps
    out = {
        "workload": "plain path tracer, box + 35 icospheres (44,814 triangles), 256x256, 64 spp, depth 8, 4 hero wavelengths",
        "metric": "path samples/s", "value": samples / (statistics.mean(dev_ms) * 1e-3), "unit": "path samples/s",
        "ms_per_step": statistics.mean(dev_ms), "steps": args.steps,
        "kernel_ms": {"closest": st.traceMs, "shade": st.shadeMs, "shadow": st.shadowMs, "film": st.filmMs},
        "rays_per_step": {"closest": int(st.closestRays), "shadow": int(st.shadowRays)},
        "e2e": {"value": samples / e2e_s, "unit": "path samples/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": int(w * hh * 3 * 8)},
    }
    peak, peak_kind = _peaks()
    achieved = PT_BYTES_PER_SAMPLE * out["value"] / 1e9
    out["roofline"] = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                       "peak_source": peak_kind, "bytes_per_path_sample": PT_BYTES_PER_SAMPLE,
                       "l2_hit_rate_closest": PT_L2_HIT_RATE,
                       "note": "algorithmic bytes of the reference traversal's node / triangle visits per path sample; "
                               "the scene is L2-resident, so DRAM moves far less"}
    if cpu:
        import tempfile

        import ref

        ref.set_threads(0)
        jp = os.path.join(tempfile.gettempdir(), "prb_bench", "box_c0.prscene.json")
        rs = ref.RefScene(scenes.write_reference_json(scenes.box_scene(seed=0, width=256, height=256), jp))
        rs.render(1, 0, 8)
        cspp = 256
        _, dt = rs.render(cspp, 1, 8)
        out["cpu_baseline"] = {"value": w * hh * cspp / dt, "unit": "path samples/s", "cores": ref.thread_count(),
                               "kind": "reference",
                               "sample": f"reference PathIntegrator, same scene from its JSON form, {cspp} spp at 256x256 ({dt:.1f} s)"}
    return out


def batch_bench(args, device: int, cpu: bool):
    """The uneven batch: 48 renders of the box family (scene seeds 0..47; resolution uniform over
    {128,256,512,1024}^2, spp over {16,64,256}, depth over {8,16,32}; even seeds with the chromatic
    homogeneous medium) rendered by ONE prgpu_render_batch call -- one CUDA graph launch whose
    device-side loop runs every wave -- with the autotuner's queue capacity and shading block.
    value = path samples/s of the graph's device time; e2e = the same over the whole call (film
    copies in and out, scene residency checks, scheduling)."""
    from prgpu import hostscene, render, scenes

    specs = scenes.uneven_batch(48)[: max(1, min(48, args.batch_renders))]
    t0 = time.perf_counter()
    hosts = [hostscene.build_box_scene(s) for s in specs]
    build_s = time.perf_counter() - t0
    films = [np.zeros((s.height, s.width, 3)) for s in specs]
    div = max(1, args.batch_spp_div)
    items = [(h.desc(), None, dict(spp=max(1, s.spp // div), seed=1, max_depth=s.max_depth), f)
             for h, s, f in zip(hosts, specs, films)]
    t0 = time.perf_counter()
    if args.batch_wave > 0:
        cfg = render.batch_config(args.batch_wave, 256)
    else:
        cfg = render.autotune_batch(items)
    tune_s = time.perf_counter() - t0
    bcfg = render.batch_config(cfg.wavefrontPaths, cfg.shadeBlock, host_loop=args.batch_host_loop)
    for _ in range(args.batch_warmup):
        render.render_batch(items, config=bcfg)
    dev, wall, st = [], [], None
    for k in range(args.batch_steps):
        step = [(d, e, dict(p, first_sample=(k + 1) * p["spp"]), f) for d, e, p, f in items]
        t0 = time.perf_counter()
        st = render.render_batch(step, config=bcfg, stats=True)
        wall.append(time.perf_counter() - t0)
        dev.append(st.deviceMs)
    samples = int(st.pathSamples)
    film_bytes = int(sum(f.nbytes for f in films))
    # The same renders one by one (prgpu_render_ex each), against one batch of them, both at 1/8 of
    # every render's spp: what batching gains over sequential single renders on this workload.
    cmp_div = 8
    cmp_items = [(d, e, dict(p, spp=max(1, p["spp"] // cmp_div)), np.zeros_like(f)) for d, e, p, f in items]
    cst = render.render_batch(cmp_items, config=bcfg, stats=True)
    single_ms = 0.0
    for d, e, p, f in cmp_items:
        _, sst = render.render_ex(d, f.shape[1], f.shape[0], p["spp"], seed=p["seed"], max_depth=p["max_depth"],
                                  out=np.zeros_like(f), stats=True)
        single_ms += sst.deviceMs
    out = {
        "workload": f"uneven batch: {len(specs)} box-family renders, 128^2..1024^2, 16..256 spp, depth 8..32, half with media",
        "metric": "path samples/s", "value": samples / (statistics.mean(dev) * 1e-3), "unit": "path samples/s",
        "ms_per_step": statistics.mean(dev), "steps": args.batch_steps, "warmup": args.batch_warmup,
        "path_samples_per_step": samples, "spp_divided_by": div, "waves": int(st.waves), "loop_iterations": int(st.loopIterations),
        "graph_launches_per_step": 0 if args.batch_host_loop else 1, "kernel_nodes_per_iteration": 14,
        "autotuned": {"wavefrontPaths": cfg.wavefrontPaths, "shadeBlock": cfg.shadeBlock, "seconds": tune_s,
                      "fixed_by_flag": args.batch_wave > 0},
        "vs_sequential_singles": {"spp_divided_by": cmp_div, "batch_ms": cst.deviceMs, "singles_ms": single_ms,
                                  "speedup": single_ms / cst.deviceMs},
        "host_scene_build_s": build_s,
        "rays_per_step": {"closest": int(st.closestRays), "shadow": int(st.shadowRays)},
        "e2e": {"value": samples / statistics.mean(wall), "unit": "path samples/s",
                "h2d_bytes_per_step": film_bytes, "d2h_bytes_per_step": film_bytes},
    }
    if cpu:
        import ref

        ref.set_threads(0)
        tot, secs = 0, 0.0
        for k in range(min(2, len(specs))):
            s = specs[k]
            jp = os.path.join(tempfile.gettempdir(), "prb_bench", f"batch_{k}.prscene.json")
            rs = ref.RefScene(scenes.write_reference_json(s, jp))
            cspp = 2
            _, dt = rs.render(cspp, 1, s.max_depth)
            tot += s.width * s.height * cspp
            secs += dt
        out["cpu_baseline"] = {"value": tot / secs, "unit": "path samples/s", "cores": ref.thread_count(),
                               "kind": "reference",
                               "sample": f"reference PathIntegrator on batch scenes 0 (medium) and 1 (plain) at their "
                                         f"resolutions, 2 spp each ({secs:.1f} s)"}
    return out


def guided_vs_plain_bench(args):
    """Equal-time relMSE, guided vs plain, on the guided-vs-plain scene (the box with its light
    behind an occluder with a 0.1-wide slit and 12 subsurface BK7 spheres; 4 hero wavelengths,
    depth 32) at a reduced size (--gvp-res, default 128^2), and on the box lit only indirectly (its
    light facing the ceiling). The reference image is a --gvp-ref-spp plain render on the GPU.
    Plain renders --gvp-spp samples per pixel; its device time is the budget. The guided form
    starts from fresh weights, samples with the guide and trains it online for --gvp-train-frac of
    the budget (default: all of it) in the guided, batched form (one graph launch per 256 spp, Adam
    steps on the samples of every filmed wave of --gvp-train-wave / 2 paths), and samples with the
    trained guide for the rest, if any (prgpu_render_ex); every sample is in its image. Training
    throughout measured best (training share 0.3 / 0.6 / 1.0 of the budget: slit scene 0.89 /
    0.90 / 0.91x, indirectly lit box 1.28 / 1.44 / 1.44x): a few Adam steps per wave cost little and
    the guide keeps improving.
    relMSE is the form of the reference's tests/test_quality.cpp:241-248: mean over pixels and
    channels of (x - ref)^2 / (ref^2 + 1e-2). ratio = relMSE plain / relMSE guided (> 1: the guide
    wins at equal time)."""
    from prgpu import guide, hostscene, render, scenes

    R = args.gvp_res
    out = {"metric": "equal-time relMSE ratio (plain / guided)", "unit": "x",
           "guide_settings": guide.get_options()}
    for name, s in (("slit_sss", scenes.slit_scene(seed=0, width=R, height=R, max_depth=32)),
                    ("indirect", scenes.indirect_scene(seed=0, width=R, height=R, max_depth=32, subdiv=3))):
        depth = s.max_depth
        desc = hostscene.build_box_scene(s).desc()
        t0 = time.perf_counter()
        ref_spp = args.gvp_ref_spp
        ref = render.render_ex(desc, R, R, ref_spp, seed=777, max_depth=depth) / ref_spp
        ref_s = time.perf_counter() - t0

        def relmse(img):
            return float(np.mean((img - ref) ** 2 / (ref ** 2 + 1e-2)))

        spp = args.gvp_spp
        plain, pst = render.render_ex(desc, R, R, spp, seed=11, max_depth=depth, stats=True)
        budget = pst.deviceMs
        guide.set_options()
        guide.set_learning_rate(1e-3)
        train = render.make_ext(guide=render.GUIDE_SAMPLE | render.GUIDE_TRAIN | render.GUIDE_RESET,
                                wavefront_paths=65536)
        use = render.make_ext(guide=render.GUIDE_SAMPLE)
        # Chunk by chunk on one film, counting device time: train while within the training share
        # of the budget, then sample with the trained guide until the budget is spent (the last
        # chunk may overshoot by one chunk's time, which is reported).
        film = np.zeros((R, R, 3))
        done, ms = 0, 0.0
        # Training runs in the guided, batched form: one graph launch per call, Adam steps after
        # every filmed wave (--gvp-train-wave paths in flight, half of them per wave), no host
        # round trip per bounce.
        tcfg = render.batch_config(args.gvp_train_wave, 256)
        # Calls of 256 spp, the last sized from the cost per sample so far to end near the budget.
        per_spp = None
        while ms < args.gvp_train_frac * budget:
            n = 256 if per_spp is None else max(8, min(256, int((args.gvp_train_frac * budget - ms) / per_spp) // 8 * 8))
            st = render.render_batch([(desc, train, dict(spp=n, first_sample=done, seed=13, max_depth=depth), film)],
                                     config=tcfg, stats=True)
            train.flags = render.GUIDE_SAMPLE | render.GUIDE_TRAIN
            ms += st.deviceMs
            done += n
            per_spp = st.deviceMs / n
        n_train = done
        # Sampling with the trained guide: calls sized from the cost per sample measured so far, so
        # that the last one ends close to the budget (chunks as large as plain rendering's).
        per_spp = None
        while ms < budget:
            n = 64 if per_spp is None else max(8, min(8192, int((budget - ms) / per_spp) // 8 * 8))
            _, st = render.render_ex(desc, R, R, n, first_sample=done, seed=13, max_depth=depth, ext=use, out=film,
                                     stats=True)
            ms += st.deviceMs
            done += n
            per_spp = st.deviceMs / n
        n_use = done - n_train
        ep, eg = relmse(plain / spp), relmse(film / done)
        # Equal sample count, for reference: the trained guide sampling only.
        g_eq, _ = render.render_ex(desc, R, R, spp, seed=14, max_depth=depth, ext=use, stats=True)
        out[name] = {"workload": f"{R}x{R}, depth {depth}, 4 hero wavelengths, reference {ref_spp} spp plain "
                                 f"({ref_s:.1f} s)",
                     "ratio": ep / eg, "plain": {"spp": spp, "device_ms": budget, "relmse": ep},
                     "guided": {"spp_training": n_train, "spp_trained": n_use, "device_ms": ms, "relmse": eg},
                     "equal_spp_ratio": ep / relmse(g_eq / spp)}
    out["ratio"] = out["slit_sss"]["ratio"]
    return out


def run_reference_arm(args, rank: int, world: int):
    if rank != 0:
        return
    from prgpu import workloads

    # The whole workload of a step (2^24 + 2^24 rays, about 2 s on 16 host threads).
    verts = workloads.triangle_soup(N_TRIS, seed=1)
    per = N_RAYS
    closest = workloads.soup_rays(per, seed=2)
    anyhit = workloads.soup_rays(per, seed=3, any_hit=True)
    import ref

    ref.set_threads(0)
    b = ref.SoupBVH(verts)
    c8 = workloads.rays_as_f8(closest)
    a8 = workloads.rays_as_f8(anyhit)
    for _ in range(args.warmup):
        b.trace(c8[: 1 << 16])
    times = []
    for _ in range(args.steps):
        *_, t1 = b.trace(c8)
        _, t2 = b.trace(a8, any_hit=True)
        times.append(t1 + t2)
    b.close()
    dt = sum(times)
    value = args.steps * 2 * per / dt / 1e6
    sample = (f"{per} closest-hit + {per} any-hit rays of the benchmark workload per step: the reference's "
              f"BVH::Intersect / IntersectP over its own BVH")
    line = {
        "metric": METRIC, "impl": "reference", "value": value, "unit": "Mrays/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": bench_config(world), "bvh": "the reference's own pr::BVH",
        "cpu_baseline": {"value": value, "unit": "Mrays/s", "cores": ref.thread_count(), "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def large_scene_bench(args, device: int):
    """The large outdoor scene (prgpu.hostscene.build_large_scene): a 4096^2 fBm heightfield
    (33.5M triangles), a 256^3 fBm cloud grid medium, 200 analytic GGX conductor spheres, a sun
    cone and an importance-sampled sky map, 3840 x 2160, depth 64, rendered through
    prgpu_render_ex. One step = --ls-spp samples per pixel; value = path samples/s of device time,
    plain BSDF sampling; guided = the same with the guide network sampling diffuse vertices and
    training online. No CPU baseline: the reference renders this scene at well under 1 spp per
    minute of this bench's budget."""
    from prgpu import hostscene, render

    t0 = time.perf_counter()
    hs, ext = hostscene.build_large_scene(args.ls_width, args.ls_height, terrain_res=args.ls_terrain,
                                          cloud_res=args.ls_cloud)
    build_s = time.perf_counter() - t0
    desc = hs.desc()
    w, h, spp, depth = args.ls_width, args.ls_height, args.ls_spp, 64
    film = np.zeros((h, w, 3))
    t0 = time.perf_counter()
    render.render_ex(desc, w, h, 1, seed=1, max_depth=depth, ext=ext, out=film)
    first_s = time.perf_counter() - t0
    out = {"workload": f"large outdoor scene: {args.ls_terrain}^2 fBm terrain ({2 * (args.ls_terrain - 1) ** 2:,} triangles), "
                       f"{args.ls_cloud}^3 fBm cloud grid, 200 GGX conductor spheres, sun + sky map, {w}x{h}, "
                       f"{spp} spp per step, depth 64",
           "metric": "path samples/s", "unit": "path samples/s", "host_scene_build_s": build_s,
           "first_render_s_with_upload": first_s, "steps": args.ls_steps}
    for name, flags in (("plain", 0), ("guided", render.GUIDE_SAMPLE | render.GUIDE_TRAIN)):
        e = abi_copy_ext(ext, flags | (render.GUIDE_RESET if flags else 0))
        render.render_ex(desc, w, h, 1, seed=2, max_depth=depth, ext=e, out=film)
        e.flags = flags
        dev, st = [], None
        for k in range(args.ls_steps):
            _, st = render.render_ex(desc, w, h, spp, first_sample=(k + 1) * spp, seed=1, max_depth=depth, ext=e,
                                     out=film, stats=True)
            dev.append(st.deviceMs)
        r = {"value": w * h * spp / (statistics.mean(dev) * 1e-3), "ms_per_step": statistics.mean(dev),
             "kernel_ms": {"closest": st.traceMs, "shade": st.shadeMs, "shadow": st.shadowMs, "film": st.filmMs},
             "rays_per_step": {"closest": int(st.closestRays), "shadow": int(st.shadowRays)},
             "closest_rays_per_sample": st.closestRays / (w * h * spp)}
        if name == "plain":
            out.update(r)
        else:
            out["guided"] = r
    return out


def c4_time_to_relmse(args):
    """The north-star comparison on the large outdoor scene (4096^2 fBm terrain, 256^3 cloud, 200
    metal spheres, Preetham sun and sky; depth 64) at a reduced film (--c4-width x --c4-height):
    device time until relMSE <= --c4-target against a plain reference of --c4-ref-spp samples,
    for the plain path tracer (prgpu_render_ex) and for the guided, batched form (prgpu_render_batch,
    the guide sampling diffuse vertices and training online after every filmed wave, fresh weights).
    Both add samples in doubling steps (1, 1, 2, 4, ... spp) onto one film and check relMSE after
    each step; a step's device time counts whole. Opt-in: the reference takes minutes."""
    from prgpu import guide, hostscene, render

    w, h, depth = args.c4_width, args.c4_height, 64
    hs, ext = hostscene.build_large_scene(w, h, terrain_res=args.ls_terrain, cloud_res=args.ls_cloud)
    desc = hs.desc()
    t0 = time.perf_counter()
    ref = render.render_ex(desc, w, h, args.c4_ref_spp, seed=999, max_depth=depth, ext=ext) / args.c4_ref_spp
    ref_s = time.perf_counter() - t0

    def relmse(img):
        return float(np.mean((img - ref) ** 2 / (ref ** 2 + 1e-2)))

    def progress(step):
        film = np.zeros((h, w, 3))
        done, ms, trace = 0, 0.0, []
        n = 1
        while done < args.c4_max_spp:
            ms += step(film, done, n)
            done += n
            e = relmse(film / done)
            trace.append((done, ms, e))
            if e <= args.c4_target:
                break
            n = max(1, done)
        return trace

    plain_ext = abi_copy_ext(ext, 0)

    def plain_step(film, first, n):
        _, st = render.render_ex(desc, w, h, n, first_sample=first, seed=1, max_depth=depth, ext=plain_ext, out=film,
                                 stats=True)
        return st.deviceMs

    guide.set_options()
    gext = abi_copy_ext(ext, render.GUIDE_SAMPLE | render.GUIDE_TRAIN | render.GUIDE_RESET)

    def guided_step(film, first, n):
        st = render.render_batch([(desc, gext, dict(spp=n, first_sample=first, seed=1, max_depth=depth), film)],
                                 config=render.batch_config(args.c4_wave, 256), stats=True)
        gext.flags = render.GUIDE_SAMPLE | render.GUIDE_TRAIN
        return st.deviceMs

    tp, tg = progress(plain_step), progress(guided_step)
    hit = lambda tr: tr[-1][1] if tr[-1][2] <= args.c4_target else None  # noqa: E731
    out = {"workload": f"large outdoor scene, {w}x{h}, depth 64, reference {args.c4_ref_spp} spp plain ({ref_s:.0f} s)",
           "target_relmse": args.c4_target, "plain": {"trace_spp_ms_relmse": tp, "ms_to_target": hit(tp)},
           "guided_batched": {"trace_spp_ms_relmse": tg, "ms_to_target": hit(tg)}}
    if hit(tp) and hit(tg):
        out["guided_time_fraction"] = hit(tg) / hit(tp)
    return out


def abi_copy_ext(ext, flags: int):
    """A copy of a SceneExt with other guide flags (the arrays stay owned by the original)."""
    from prgpu import abi

    e = abi.SceneExt.from_buffer_copy(ext)
    e.flags = flags
    e._keep = [ext]
    return e


def main():
    global N_RAYS
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer pass (profiling runs)")
    ap.add_argument("--no-path-tracer", action="store_true", help="skip the path-tracer workload")
    ap.add_argument("--rays", type=int, default=N_RAYS, help="rays per pass (smaller for profiling captures)")
    ap.add_argument("--path-tracer-only", action="store_true",
                    help="run only the path-tracer workload and print its JSON object (profiling captures)")
    ap.add_argument("--pt-res", type=int, default=256, help="path-tracer image side (256 = the measured workload)")
    ap.add_argument("--no-batch", action="store_true", help="skip the uneven-batch workload")
    ap.add_argument("--batch-only", action="store_true", help="run only the uneven batch and print its JSON object")
    ap.add_argument("--batch-steps", type=int, default=2)
    ap.add_argument("--batch-warmup", type=int, default=1)
    ap.add_argument("--batch-host-loop", action="store_true",
                    help="drive the batch loop from the host (profiling captures: ncu cannot see inside "
                         "conditional graphs)")
    ap.add_argument("--batch-spp-div", type=int, default=1,
                    help="divide every render's spp (profiling captures only; the JSON says so)")
    ap.add_argument("--batch-renders", type=int, default=48,
                    help="render only the first K of the 48 batch scenes (profiling captures only; the JSON says so)")
    ap.add_argument("--batch-wave", type=int, default=0,
                    help="paths in flight instead of the autotuner's choice, shading blocks of 256 (profiling captures)")
    ap.add_argument("--no-guided", action="store_true", help="skip the guided-vs-plain comparison")
    ap.add_argument("--guided-only", action="store_true",
                    help="run only the guided-vs-plain comparison and print its JSON object (profiling captures)")
    ap.add_argument("--gvp-res", type=int, default=128, help="guided-vs-plain image side (1024 = the full C3 size)")
    ap.add_argument("--gvp-spp", type=int, default=32768, help="plain samples per pixel of the equal-time comparison")
    ap.add_argument("--gvp-ref-spp", type=int, default=65536, help="samples per pixel of the plain reference image")
    ap.add_argument("--gvp-train-frac", type=float, default=1.0,
                    help="share of the guided run's time budget spent training online")
    ap.add_argument("--gvp-train-wave", type=int, default=1 << 22,
                    help="paths in flight in the guided run's batched training calls (two waves of half)")
    ap.add_argument("--large-scene", action="store_true",
                    help="also run the large outdoor scene (33.5M-triangle terrain, cloud grid, 4K film; opt-in: "
                         "about a minute of host scene build)")
    ap.add_argument("--large-scene-only", action="store_true", help="run only the large outdoor scene")
    ap.add_argument("--c4-time-to-relmse", action="store_true",
                    help="run only the large scene's time to relMSE, guided + batched vs plain (opt-in, minutes)")
    ap.add_argument("--c4-width", type=int, default=480)
    ap.add_argument("--c4-height", type=int, default=270)
    ap.add_argument("--c4-ref-spp", type=int, default=16384)
    ap.add_argument("--c4-target", type=float, default=0.01)
    ap.add_argument("--c4-wave", type=int, default=1 << 22,
                    help="paths in flight in the guided, batched run (two waves of half)")
    ap.add_argument("--c4-max-spp", type=int, default=4096)
    ap.add_argument("--ls-spp", type=int, default=4)
    ap.add_argument("--ls-steps", type=int, default=2)
    ap.add_argument("--ls-width", type=int, default=3840)
    ap.add_argument("--ls-height", type=int, default=2160)
    ap.add_argument("--ls-terrain", type=int, default=4096)
    ap.add_argument("--ls-cloud", type=int, default=256)
    args = ap.parse_args()
    N_RAYS = args.rays
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference_arm(args, rank, world)
    if args.path_tracer_only:
        print(json.dumps(path_tracer_bench(args, local, cpu=not args.no_cpu_baseline)))
        return
    if args.batch_only:
        print(json.dumps(batch_bench(args, local, cpu=not args.no_cpu_baseline)))
        return
    if args.large_scene_only:
        print(json.dumps(large_scene_bench(args, local)))
        return
    if args.guided_only:
        print(json.dumps(guided_vs_plain_bench(args)))
        return
    if args.c4_time_to_relmse:
        print(json.dumps(c4_time_to_relmse(args)))
        return

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))

    from prgpu import abi

    verts, closest, anyhit, trace = make_inputs(rank)
    nodes, order = trace.build_bvh_triangles(verts, max_leaf=1)
    acc = trace.Accel(nodes, order, verts, device=local)
    lib = abi.gpu_lib()

    dc = torch.from_numpy(closest.view(np.uint8)).cuda()
    da = torch.from_numpy(anyhit.view(np.uint8)).cuda()
    prim = torch.empty(N_RAYS, dtype=torch.int32, device="cuda")
    tdist = torch.empty(N_RAYS, dtype=torch.float32, device="cuda")
    occ = torch.empty(N_RAYS, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()

    def step(ev=None):
        if ev is not None:
            ev[0].record(stream)
        acc.trace_device(dc.data_ptr(), N_RAYS, prim.data_ptr(), tdist.data_ptr(), False, stream.cuda_stream)
        if ev is not None:
            ev[1].record(stream)
        acc.trace_device(da.data_ptr(), N_RAYS, occ.data_ptr(), 0, True, stream.cuda_stream)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    t_start, t_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # The clock sampler runs from the warm-up through the timed region (both under full load).
    with ClockSampler(local) as clocks:
        for _ in range(max(args.warmup, 8)):
            step()
        barrier()
        launches0 = lib.prgpu_launch_count()
        barrier()
        t_start.record(stream)
        for k in range(args.steps):
            step(evs[k])
        t_end.record(stream)
        barrier()
    launches = int(lib.prgpu_launch_count() - launches0)
    ms = t_start.elapsed_time(t_end)
    closest_ms = statistics.mean(a.elapsed_time(b) for a, b in evs)
    ms, closest_ms = max_over_ranks([ms, closest_ms], world)
    ms_per_step = ms / args.steps
    value = whole_job_mrays(world, 2 * N_RAYS, ms_per_step * 1e-3)
    assert acc.status() == 0, "traversal stack overflow"

    # End to end through the C ABI with pinned host buffers (the copies are inside the region).
    e2e_value = None
    if not args.no_e2e:
        hc = torch.from_numpy(closest.view(np.uint8)).pin_memory().numpy().view(abi.RAY)
        ha = torch.from_numpy(anyhit.view(np.uint8)).pin_memory().numpy().view(abi.RAY)
        hprim = torch.empty(N_RAYS, dtype=torch.int32).pin_memory().numpy()
        ht = torch.empty(N_RAYS, dtype=torch.float32).pin_memory().numpy()
        hocc = torch.empty(N_RAYS, dtype=torch.int32).pin_memory().numpy()
        e2e_steps = max(3, min(args.steps, 5))
        for _ in range(2):
            acc.trace_host(hc, hprim, ht, False)
            acc.trace_host(ha, hocc, None, True)
        barrier()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            acc.trace_host(hc, hprim, ht, False)
            acc.trace_host(ha, hocc, None, True)
        barrier()
        e2e_s = (time.perf_counter() - t0) / e2e_steps
        (e2e_s,) = max_over_ranks([e2e_s], world)
        e2e_value = whole_job_mrays(world, 2 * N_RAYS, e2e_s)
        np.testing.assert_array_equal(hprim, prim.cpu().numpy())

    peak, peak_kind = _peaks()
    achieved = BYTES_PER_RAY * N_RAYS / (closest_ms * 1e-3) / 1e9
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        per = 1 << 24
        v, cores, secs = cpu_reference(verts, closest, anyhit, per)
        cpu = {"value": v, "unit": "Mrays/s", "cores": cores, "kind": "reference",
               "sample": f"{per} closest-hit + {per} any-hit rays of this workload through the reference "
                         f"BVH::Intersect/IntersectP on its own BVH ({secs:.1f} s)"}
    pt = None
    if world == 1 and not args.no_path_tracer:
        pt = path_tracer_bench(args, local, cpu=not args.no_cpu_baseline)
    bt = None
    if world == 1 and not args.no_batch:
        bt = batch_bench(args, local, cpu=not args.no_cpu_baseline)
    gvp = None
    if world == 1 and not args.no_guided:
        gvp = guided_vs_plain_bench(args)
    ls = None
    if world == 1 and args.large_scene:
        ls = large_scene_bench(args, local)
    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": bench_config(world), "bvh": "own binned SAH, 1 triangle per leaf, collapsed 4-wide",
        "e2e": None if e2e_value is None else
        {"value": e2e_value, "unit": "Mrays/s", "h2d_bytes_per_step": int(2 * N_RAYS * 32),
         "d2h_bytes_per_step": int(N_RAYS * 8 + N_RAYS * 4)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_kind, "kernel": "k_trace<closest>",
                     "bytes_per_ray": BYTES_PER_RAY, "launch_ms": closest_ms,
                     "traffic": NCU_TRAFFIC_PER_LAUNCH,
                     "traffic_source": "ncu dram read + write of this kernel on a 2^22-ray launch of this workload, "
                                       "scaled x4; not measured in this run"},
        "cpu_baseline": cpu,
        "clocks": clocks.summary(),
        "gpu_launches": launches,
        "closest_hit_mrays": N_RAYS / (closest_ms * 1e3),
        "any_hit_mrays": N_RAYS / ((ms_per_step - closest_ms) * 1e3),
        "path_tracer": pt,
        "uneven_batch": bt,
        "guided_vs_plain": gvp,
    }
    if ls is not None:
        line["large_scene"] = ls
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
