"""The per-ray work the benchmark's roofline credits (bench.py NODES_PER_RAY, TRIS_PER_RAY) is
the reference traversal's own, counted by the oracle over the reference's tree on the benchmark's
rays (oracle/measure_trace_work.py): the frozen constants must equal a fresh count."""

import pytest


def test_frozen_trace_work_equals_the_oracle_count(oracle):
    import bench
    import measure_trace_work as mtw

    w = mtw.trace_work(1 << 18)
    assert round(w["closest_nodes"], 2) == pytest.approx(bench.NODES_PER_RAY)
    assert round(w["closest_tris"], 2) == pytest.approx(bench.TRIS_PER_RAY)
    assert bench.BYTES_PER_RAY == pytest.approx(32 * w["closest_nodes"] + 36 * w["closest_tris"] + 40, rel=1e-3)
