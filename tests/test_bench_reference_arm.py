"""`bench.py --impl reference` on the host cores (no GPU): the reference's own BVH::Intersect /
IntersectP over its own tree (oracle/_ref) on the benchmark's workload, here at 2^16 rays per pass,
printing one JSON line with the benchmark contract's keys, the same `config` as the GPU arm's
and a positive rate."""

import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_the_contract_line(oracle, monkeypatch):
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "2",
                          "--warmup", "3", "--rays", str(1 << 16)], capture_output=True, text=True, timeout=600,
                         cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["unit"] == "Mrays/s" and line["value"] > 0
    assert line["steps"] == 2 and line["warmup"] == 3 and line["higher_is_better"] is True
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["value"] == line["value"]
    import bench

    monkeypatch.setattr(bench, "N_RAYS", 1 << 16)
    assert line["config"] == bench.bench_config(1)
