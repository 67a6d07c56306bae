"""Checkpoint and resume of a progressive GPU render (the reference's loop,
src/integrators/gpu_path.cpp:458-513): a render stopped part-way, written to a PRCKPT02 file and
resumed, ends bit-identical to the same render done in one go; a checkpoint made for another seed
is refused."""

import numpy as np
import pytest

import render_util as ru
from prgpu import abi, checkpoint

pytestmark = pytest.mark.gpu


def test_resumed_render_is_bit_identical(gpu, oracle, tmp_path):
    w = h = 48
    rs = oracle.RefScene(ru.scene_file("ckpt_box", seed=2, width=w, height=h, medium=True))
    desc = rs.export()
    whole, done = checkpoint.progressive_render(desc, w, h, 96, seed=7, max_depth=8)
    assert done == 96
    path = str(tmp_path / "render.ckpt")
    part, done = checkpoint.progressive_render(desc, w, h, 96, seed=7, max_depth=8, checkpoint=path, stop_after=37)
    assert done == 37 and not np.array_equal(part, whole)
    resumed, done = checkpoint.progressive_render(desc, w, h, 96, seed=7, max_depth=8, resume=path, checkpoint=path)
    assert done == 96
    assert np.array_equal(resumed, whole)
    film, passes = checkpoint.read(path, checkpoint.header(w, h, 7, 8))
    assert passes == 96 and np.array_equal(film, whole)
    with pytest.raises(abi.PrgpuError, match="different scene"):
        checkpoint.progressive_render(desc, w, h, 96, seed=8, max_depth=8, resume=path)
