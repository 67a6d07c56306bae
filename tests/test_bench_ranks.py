"""The benchmark's multi-GPU bookkeeping, run on CPU with the gloo backend (world size 2).

`bench.py --gpus N` runs one rank per GPU, each tracing its own rays (replicas: no data-path
collective). The only cross-rank steps are a barrier around the timed region and the reduction of
each rank's timings to the slowest rank's (`max_over_ranks`, an all-reduce with MAX); the
whole-job rate then counts every rank's rays over that time (`whole_job_mrays`). Here two gloo
ranks run exactly those functions with different local timings. The reference arm runs on rank 0
only; the other ranks return at once without work."""

import os
import socket
from datetime import timedelta

import pytest

WORLD = 2


def _free_port() -> int:
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, q) -> None:
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        import bench

        # Per-rank step time, closest-hit time, end-to-end seconds: rank 1 is slower on the first
        # two, rank 0 on the third.
        local = [7.0 + rank, 4.0 + 0.5 * rank, 0.03 - 0.01 * rank]
        dist.barrier()
        out = bench.max_over_ranks(local, world, device="cpu")
        q.put((rank, out, bench.whole_job_mrays(world, 2 * bench.N_RAYS, out[0] * 1e-3)))
    finally:
        dist.destroy_process_group()


def test_timings_reduce_to_the_slowest_rank_over_gloo():
    import torch.multiprocessing as mp

    import bench

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, WORLD, port, q)) for r in range(WORLD)]
    for p in procs:
        p.start()
    try:
        results = sorted(q.get(timeout=120) for _ in range(WORLD))
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    expect = [8.0, 4.5, 0.03]
    for rank, out, mrays in results:
        assert out == pytest.approx(expect), (rank, out)
        # Two ranks of 2 x 2^24 rays each in the slowest rank's 8 ms.
        assert mrays == pytest.approx(2 * 2 * bench.N_RAYS / 8e-3 / 1e6)


def test_single_rank_needs_no_process_group():
    import bench

    assert bench.max_over_ranks([3.0, 1.5], 1) == [3.0, 1.5]
    assert bench.whole_job_mrays(1, 1_000_000, 0.5) == pytest.approx(2.0)


def test_reference_arm_runs_on_rank_zero_only():
    import bench

    # Any rank but 0 returns before touching its arguments or the oracle.
    assert bench.run_reference_arm(None, rank=1, world=WORLD) is None
