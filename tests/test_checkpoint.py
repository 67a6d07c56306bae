"""Checkpoint files against the reference's own WriteCheckpoint / ReadCheckpoint
(src/integrators/integrator.cpp:16-90, film.cpp:61-84): the module's host library writes the same
bytes for the same render state, reads the reference's files, and refuses the same files with the
same messages (wrong magic, another header, truncation)."""

import ctypes as C
import os

import numpy as np
import pytest

from prgpu import abi, checkpoint

W, H, SEED, DEPTH, FP = 7, 5, 1234567, 8, 0x9E3779B97F4A7C15


def _film(seed=0):
    rng = np.random.default_rng(seed)
    return rng.normal(size=(H, W, 3)) * 10.0 ** rng.integers(-3, 6, size=(H, W, 3))


def _ref_write(oracle, path, film, passes, seed=SEED, device=0):
    err = C.create_string_buffer(512)
    f = np.ascontiguousarray(film, np.float64)
    assert oracle.ref_lib().prref_checkpoint_write(path.encode(), W, H, device, DEPTH, FP, seed, oracle._p(f), passes,
                                                   err, len(err)) == 0, err.value


def _ref_read(oracle, path, seed=SEED, device=0):
    err = C.create_string_buffer(512)
    film = np.zeros((H, W, 3), np.float64)
    passes = C.c_int32(0)
    rc = oracle.ref_lib().prref_checkpoint_read(path.encode(), W, H, device, DEPTH, FP, seed, oracle._p(film),
                                                C.byref(passes), err, len(err))
    return rc, film, passes.value, err.value.decode()


def test_same_bytes_as_the_reference(oracle, tmp_path):
    film = _film()
    ref_path, our_path = str(tmp_path / "ref.ckpt"), str(tmp_path / "ours.ckpt")
    _ref_write(oracle, ref_path, film, 37)
    checkpoint.write(our_path, checkpoint.header(W, H, SEED, DEPTH, FP), film, 37)
    assert open(ref_path, "rb").read() == open(our_path, "rb").read()
    assert not os.path.exists(our_path + ".tmp")


def test_reads_reference_files_and_the_reference_reads_ours(oracle, tmp_path):
    film = _film(1)
    ref_path, our_path = str(tmp_path / "ref.ckpt"), str(tmp_path / "ours.ckpt")
    _ref_write(oracle, ref_path, film, 5)
    got, passes = checkpoint.read(ref_path, checkpoint.header(W, H, SEED, DEPTH, FP))
    assert passes == 5 and np.array_equal(got, film)
    checkpoint.write(our_path, checkpoint.header(W, H, SEED, DEPTH, FP), film, 9)
    rc, got, passes, _ = _ref_read(oracle, our_path)
    assert rc == 0 and passes == 9 and np.array_equal(got, film)


def test_refusals_match_the_reference(oracle, tmp_path):
    film = _film(2)
    path = str(tmp_path / "a.ckpt")
    checkpoint.write(path, checkpoint.header(W, H, SEED, DEPTH, FP), film, 3)
    cases = {}
    # Another seed: the header differs.
    cases["header"] = (path, SEED + 1)
    # Truncated film.
    trunc = str(tmp_path / "t.ckpt")
    open(trunc, "wb").write(open(path, "rb").read()[:200])
    cases["truncated"] = (trunc, SEED)
    # Not a checkpoint at all.
    junk = str(tmp_path / "j.ckpt")
    open(junk, "wb").write(b"PRCKPT01" + bytes(100))
    cases["magic"] = (junk, SEED)
    for name, (p, seed) in cases.items():
        rc, _, _, ref_msg = _ref_read(oracle, p, seed=seed)
        assert rc != 0, name
        with pytest.raises(abi.PrgpuError) as e:
            checkpoint.read(p, checkpoint.header(W, H, seed, DEPTH, FP))
        assert str(e.value) == ref_msg, (name, str(e.value), ref_msg)


def test_gpu_bit_in_the_header(oracle, tmp_path):
    """A CPU render's checkpoint (no device bit) does not resume a GPU render."""
    path = str(tmp_path / "cpu.ckpt")
    _ref_write(oracle, path, _film(3), 4, device=-1)
    with pytest.raises(abi.PrgpuError, match="different scene, integrator, device"):
        checkpoint.read(path, checkpoint.header(W, H, SEED, DEPTH, FP))
    film, passes = checkpoint.read(path, checkpoint.header(W, H, SEED, DEPTH, FP, gpu=False))
    assert passes == 4
