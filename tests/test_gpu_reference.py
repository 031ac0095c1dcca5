"""The B200 engine against the reference's own CPU BFS, and the reference's own
driver running the engine.

1. Golden fixtures (tests/golden/reference_bfs_*.npz, written from the
   reference's stock BfsBase by make_reference_golden.py): on the same seeded
   graph, with the same flags (-C, group reordering) and α/β, the engine must
   pick the same roots (find_roots_in_large_graph, main.cc:334-359) and give,
   per search, the same auto_tuning_data slots (bfs.hpp:3413-3457), the same
   level for every vertex, the same CoreBFS tree entries (parents of the
   pruned forest, corebfs_adaptor.hpp:290-296) and a pred that the oracle's
   and the device's Graph500 validators accept with the reference's
   traversed-edge count.
2. Drop-in: oracle/_ref/b200_runnable is the reference's mpi/main.cc,
   unchanged, built with graph500-bfs_b200/dropin/bfs_cpu.hpp in place of
   mpi/bfs_cpu.hpp.  Its own find_roots, timing, validate.hpp and result
   printing run on the engine; every search must validate with
   pf_nedge[SCALE] traversed edges.
"""
import glob
import os
import re
import subprocess

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
REF_BIN = os.path.join(ROOT, "oracle", "_ref")
FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "reference_bfs_*.npz")))
NAMES = [os.path.basename(f)[len("reference_bfs_"):-4] for f in FIXTURES]


@pytest.fixture(scope="module")
def engine(built):
    import b200bfs

    e = b200bfs.Engine(0)
    yield e
    e.close()


@pytest.mark.parametrize("name", NAMES)
def test_engine_reproduces_reference(engine, name):
    import b200bfs

    d = dict(np.load(os.path.join(GOLDEN, "reference_bfs_%s.npz" % name)))
    scale = int(d["scale"])
    alpha, beta = float(d["alpha"]), float(d["beta"])
    corebfs = bool(int(d["corebfs"]))
    n = 1 << scale
    flags = (b200bfs.BUILD_COREBFS if corebfs else 0) | (
        b200bfs.BUILD_GROUP_REORDER if int(d["group"]) else 0)
    engine.generate_graph(scale, 16, flags=flags)
    gi = engine.info()
    assert gi.num_global_edges == int(d["num_global_edges"])
    assert gi.num_global_verts == int(d["num_global_verts"])
    assert gi.pred_size == int(d["pred_size"])
    if int(d["group"]):
        assert gi.reorder_bits == int(d["reorder_bits"])
    engine.prepare(16, 10.0, 14.0)
    has_edge = engine.has_edge_all()[:n]
    roots = O.find_roots_in_large_graph(has_edge, n, len(d["roots"]),
                                        lambda r: int(engine.run(r, 16, 10.0, 14.0)[8]))
    assert np.array_equal(roots, d["roots"])
    edges = O.generate_edges(scale)
    engine.prepare(16, alpha, beta)
    for i, r in enumerate(roots):
        at = engine.run(int(r), 16, alpha, beta)
        assert np.array_equal(at, d["atd"][i]), (i, at, d["atd"][i])
        pred = engine.get_pred()
        assert (pred[n:] == -1).all()
        lv, tree = O.resolve_levels(pred[:n])
        assert np.array_equal(lv, d["levels"][i].astype(np.int64)), i
        assert np.array_equal(engine.get_levels()[:n], d["levels"][i].astype(np.int32)), i
        if corebfs:
            want = d["forest_parent"].astype(np.int64).copy()
            climb = d["climb"][i]
            want[climb[climb >= 0]] = -1
            assert np.array_equal(tree, want), i
        else:
            assert (tree < 0).all()
        err, cnt = O.validate(edges, n, pred[:n], int(r), corebfs=corebfs, nlocalverts=n)
        assert err == 0 and cnt == int(d["nedge"][i]), (i, err, cnt)
        assert engine.validate(int(r)) == (0, int(d["nedge"][i]))
    engine.end()


def _run_driver(exe, args, timeout=600):
    env = dict(os.environ, OMP_NUM_THREADS=str(min(os.cpu_count() or 1, 16)))
    p = subprocess.run([os.path.join(REF_BIN, exe)] + args, capture_output=True, text=True,
                       timeout=timeout, env=env)
    assert p.returncode == 0, (p.returncode, p.stdout[-2000:], p.stderr[-2000:])
    return p.stdout + p.stderr


def _result(out):
    fields = {}
    for k in ("SCALE", "NBFS", "min_nedge", "max_nedge", "harmonic_mean_TEPS", "alpha", "beta"):
        m = re.search(r"^%s:\s+(\S+)" % k, out, re.M)
        if m:
            fields[k] = float(m.group(1))
    return fields


@pytest.mark.parametrize("exe,args", [
    ("b200_runnable", ["16", "-n", "8"]),
    ("b200_runnable", ["16", "-A", "-C", "-n", "8"]),
    ("b200_runnable_group", ["16", "-A", "-C", "-n", "8"]),
    ("b200_runnable_group", ["20", "-C", "-n", "4"]),
])
def test_reference_driver_runs_engine(built, exe, args):
    if not os.path.exists(os.path.join(REF_BIN, exe)):
        pytest.fail("%s missing: build it with `make -C oracle/ref` where the reference is" % exe)
    out = _run_driver(exe, args)
    assert "No results printed for invalid run" not in out
    res = _result(out)
    scale = int(args[0])
    assert res["SCALE"] == scale and res["NBFS"] == int(args[args.index("-n") + 1])
    assert res["min_nedge"] == res["max_nedge"] == O.PF_NEDGE[scale], res
    assert res["harmonic_mean_TEPS"] > 0
    # the engine, not the reference's BfsBase, ran the searches
    assert "B200" in out or "b200" in out
