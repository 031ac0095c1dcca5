"""bench.py --impl reference (no GPU): the reference's own program
(oracle/_ref/ref_runnable_group, mpi/main.cc with the stock BfsBase) runs on
the host cores and bench.py prints one JSON line in the bench contract --
same metric and unit as the GPU arm, cpu_baseline of kind "reference", e2e
without copies, and a config naming the SCALE and options that actually
ran."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_line(built):
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_runnable_group")
    if not os.path.exists(exe):
        pytest.fail("oracle/_ref/ref_runnable_group missing: `make -C oracle/ref` where the "
                    "reference tree is")
    env = dict(os.environ, OMP_NUM_THREADS=str(min(os.cpu_count() or 1, 8)))
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--steps", "4", "--warmup", "2", "--ref-scale", "12"],
                       capture_output=True, text=True, timeout=600, env=env, cwd=ROOT)
    assert p.returncode == 0, p.stderr[-3000:]
    lines = [l for l in p.stdout.splitlines() if l.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"].startswith("harmonic-mean GTEPS, SCALE 28")
    assert d["unit"] == "GTEPS" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 4 and d["warmup"] == 2
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": "GTEPS", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    c = d["config"]
    assert c["scale"] == 12 and c["gpu_arm_scale"] == 28
    assert c["corebfs"] and c["group_reorder"] and c["auto_tune"]
    assert "-A -C group reordering" in c["workload"]
    # no library of this repository in the process that ran the reference
    assert "b200bfs" not in p.stderr
