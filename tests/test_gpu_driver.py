"""The C++ drop-in (bfs_on_b200.hpp via the runnable driver) and the -A
alpha/beta tuner on the device."""
import os
import re
import subprocess

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RUNNABLE = os.path.join(ROOT, "graph500-bfs_b200", "runnable")


def run_driver(*args):
    out = subprocess.run([RUNNABLE, *map(str, args)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    fields = dict(re.findall(r"^(\w+):\s+(\S+)$", out.stdout, re.M))
    return fields, out.stderr


@pytest.mark.parametrize("opts", [[], ["-C"], ["-G"], ["-A"], ["-A", "-C", "-G"]])
def test_runnable_reports_reference_counts(built, opts):
    f, err = run_driver(18, "-n", 8, *opts)
    assert int(f["SCALE"]) == 18 and int(f["NBFS"]) == 8
    # every root is validated and counts pf_nedge edges (mpi/utils.hpp:3687-3733)
    assert float(f["min_nedge"]) == float(f["max_nedge"]) == O.PF_NEDGE[18]
    assert float(f["harmonic_mean_TEPS"]) > 0
    if "-A" in opts:
        assert "Estimated Performance" in err


def test_auto_tune_keeps_results_exact(built):
    import b200bfs

    e = b200bfs.Engine(0)
    e.generate_graph(18, 16)
    e.prepare(16)
    roots = e.find_roots(8)
    edges = O.generate_edges(18)
    g = O.Graph(edges)
    nedge = []
    for r in roots:
        e.run(int(r), 16)
        err, cnt = e.validate(int(r))
        assert err == 0
        nedge.append(cnt)
    a, b, teps = e.auto_tune(roots, nedge, 16, 10.0, 14.0)
    assert a > 0 and b > 0 and teps > 0
    for r in roots[:3]:
        at = e.run(int(r), 16, a, b)
        lv = e.get_levels()[: g.nverts]
        assert np.array_equal(lv, g.levels(int(r)))
        ref_pred, ref_at, _ = g.bfs(int(r), alpha=a, beta=b)
        assert np.array_equal(at, ref_at)
    e.close()
