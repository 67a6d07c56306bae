"""Checkpointed progressive rendering: the reference's GPU render loop with checkpoint and resume
(src/integrators/gpu_path.cpp:458-513), over this module's FP64 film.

Checkpoint files use the reference's PRCKPT02 layout (libprender_host.so,
prhost_checkpoint_write / _read), so the files a PRender build writes for a GPU path-tracer render
resume here and the other way round. Sample streams are addressed by sample index and the film
sums each pixel's samples in sample order in FP64, so a render resumed from a checkpoint is
bit-identical to the same render done in one go.
"""

from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import abi, render

PATH_INTEGRATOR, GPU_DEVICE_BIT = 0, 0x100
DEFAULT_CHAINS = 1024  # pr::IntegratorSettings::chains, written into every header


def header(width: int, height: int, seed: int, max_depth: int, fingerprint: int = 0, gpu: bool = True,
           integrator: int = PATH_INTEGRATOR, chains: int = DEFAULT_CHAINS) -> abi.CheckpointHeader:
    """The header a PRender GPU path-tracer render writes (integrator.cpp:18-28): max depth <= 0
    is stored as 0 (unlimited, as CreateIntegrator normalises it)."""
    h = abi.CheckpointHeader()
    h.integrator = integrator | (GPU_DEVICE_BIT if gpu else 0)
    h.maxDepth = max(0, max_depth)
    h.width, h.height, h.chains = width, height, chains
    h.fingerprint, h.seed = fingerprint, seed
    return h


def write(path: str, hdr: abi.CheckpointHeader, film: np.ndarray, passes: int) -> None:
    """film: (height, width, 3) float64 XYZ sums; passes: samples per pixel rendered."""
    f = np.ascontiguousarray(film, np.float64)
    body = np.array([passes], np.int32)
    err = abi.err_buf()
    rc = abi.host_lib().prhost_checkpoint_write(path.encode(), C.byref(hdr), abi.ptr(f), f.size, abi.ptr(body),
                                                body.nbytes, err, len(err))
    if rc != 0:
        raise abi.PrgpuError(err.value.decode())


def read(path: str, hdr: abi.CheckpointHeader) -> tuple[np.ndarray, int]:
    """(film (height, width, 3) float64, passes) of a checkpoint made for exactly hdr."""
    film = np.zeros((hdr.height, hdr.width, 3), np.float64)
    body = np.zeros(16, np.uint8)
    size = C.c_uint64(0)
    err = abi.err_buf()
    rc = abi.host_lib().prhost_checkpoint_read(path.encode(), C.byref(hdr), abi.ptr(film), film.size, abi.ptr(body),
                                               body.nbytes, C.byref(size), err, len(err))
    if rc != 0:
        raise abi.PrgpuError(err.value.decode())
    if size.value != 4:
        raise abi.PrgpuError(f"{path} is truncated or corrupt")
    return film, int(body[:4].view(np.int32)[0])


def progressive_render(scene, width: int, height: int, spp: int, seed: int = 0, max_depth: int = 0, ext=None,
                       checkpoint: str | None = None, resume: str | None = None, fingerprint: int = 0,
                       checkpoint_interval: float = 60.0, stop_after: int | None = None, device: int = 0):
    """Renders spp samples per pixel in progressive batches (the batch doubles while a call takes
    under 0.15 s, halves above 0.5 s, at most 256: gpu_path.cpp:486-500). resume: continue from
    that checkpoint (its samples are kept, rendering restarts at its sample count). checkpoint:
    written every checkpoint_interval seconds and at the end. stop_after: stop once that many
    samples per pixel are done (a render cut short, as by a cancel). Returns (film, done)."""
    hdr = header(width, height, seed, max_depth, fingerprint)
    film = np.zeros((height, width, 3), np.float64)
    done = 0
    if resume:
        film, done = read(resume, hdr)
    target = spp if stop_after is None else min(spp, stop_after)
    batch, last = 1, time.perf_counter()
    while done < target:
        n = min(batch, target - done)
        t0 = time.perf_counter()
        render.render_ex(scene, width, height, n, first_sample=done, seed=seed, max_depth=max_depth, out=film, ext=ext,
                         device=device)
        dt = time.perf_counter() - t0
        done += n
        if dt < 0.15:
            batch = min(batch * 2, 256)
        elif dt > 0.5 and batch > 1:
            batch //= 2
        if checkpoint and time.perf_counter() - last >= checkpoint_interval:
            write(checkpoint, hdr, film, done)
            last = time.perf_counter()
    if checkpoint:
        write(checkpoint, hdr, film, done)
    return film, done
