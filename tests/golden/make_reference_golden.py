"""Writes golden fixtures of the reference's own CPU BFS.

Runs oracle/_ref/ref_dump and ref_dump_group (the reference's mpi/main.cc flow
with its stock BfsBase, built unchanged by oracle/ref/Makefile against the
single-rank MPI runtime) for each configuration below and stores, per
configuration, tests/golden/reference_bfs_<name>.npz with:

  scale, edgefactor, alpha, beta     the α/β the searches ran with (after the
                                     -A tuner when auto_tune is set; the tuner
                                     times searches, so its α/β vary by machine
                                     and are recorded rather than re-derived)
  corebfs, group, auto_tune, reorder_bits, pred_size,
  num_global_edges, num_global_verts graph_ fields after construct
  roots        int64[n]     find_roots_in_large_graph's roots (main.cc:334-359)
  atd          int64[n, 9]  auto_tuning_data of each search (bfs.hpp:3413-3457)
  nedge        int64[n]     validate_bfs_result's traversed-edge count
  valid        int8[n]      validate_bfs_result's verdict
  levels       int8/int16[n, 2^scale]  exact level of every vertex, -1 unreached;
               CoreBFS tree entries (level field 0xFFFF, corebfs_adaptor.hpp:
               290-296) resolved from their parents as validate.hpp does
  forest_parent int32[2^scale]  (CoreBFS only) the pruned forest's parent of
               every vertex whose entry has level field 0xFFFF in some search,
               -1 elsewhere; unique for a given graph
  climb        int64[n, 64]  (CoreBFS only) per search, the forest vertices
               whose entry is NOT a tree entry (the root's climb to the core,
               written with real levels), -1 padded: a search's tree entries
               are exactly forest_parent's vertices minus its climb

Parents of core vertices are not stored: BFS trees are not unique, so those
are checked through validation only.

usage: python tests/golden/make_reference_golden.py   (needs oracle/_ref built
from the reference tree: `make -C oracle/ref`)
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle"))
import oracle  # noqa: E402
REF_BIN = os.path.join(REPO, "oracle", "_ref")

# name, scale, roots, flags, group reordering
CONFIGS = [
    ("s12_plain", 12, 16, [], False),
    ("s12_A", 12, 16, ["-A"], False),
    ("s12_AC", 12, 16, ["-A", "-C"], False),
    ("s12_AC_group", 12, 16, ["-A", "-C"], True),
    ("s16_plain", 16, 8, [], False),
    ("s16_C", 16, 8, ["-C"], False),
    ("s16_AC_group", 16, 8, ["-A", "-C"], True),
    ("s20_plain", 20, 2, [], False),
    ("s20_AC_group", 20, 2, ["-A", "-C"], True),
]

def levels_from_pred(pred, nverts):
    """Exact levels and tree parents of a reference pred (oracle.resolve_levels)."""
    lv, tree = oracle.resolve_levels(pred[:nverts])
    return lv.astype(np.int16), tree.astype(np.int32), bool((tree >= 0).any())


def run_config(name, scale, nroots, flags, group, out_dir):
    exe = os.path.join(REF_BIN, "ref_dump_group" if group else "ref_dump")
    with tempfile.TemporaryDirectory() as tmp:
        cmd = [exe, str(scale), tmp, "-n", str(nroots)] + flags
        env = dict(os.environ)
        env.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
        subprocess.run(cmd, check=True, env=env, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        meta = {}
        for line in open(os.path.join(tmp, "meta.txt")):
            k, v = line.split()
            meta[k] = float(v) if k in ("alpha", "beta") else int(v)
        roots = np.fromfile(os.path.join(tmp, "roots.bin"), np.int64)
        atd = np.fromfile(os.path.join(tmp, "atd.bin"), np.int64).reshape(-1, 9)
        nedge = np.fromfile(os.path.join(tmp, "nedge.bin"), np.int64)
        valid = np.fromfile(os.path.join(tmp, "valid.bin"), np.int8)
        nverts = 1 << scale
        levels, trees, any_tree = [], [], False
        for i in range(len(roots)):
            pred = np.fromfile(os.path.join(tmp, "pred_%02d.bin" % i), np.int64)
            assert pred.size == meta["pred_size"]
            assert (pred[nverts:] == -1).all()
            lv, tp, has_tree = levels_from_pred(pred, nverts)
            levels.append(lv)
            trees.append(tp)
            any_tree |= has_tree
    assert valid.all(), (name, valid)
    arrays = dict(
        scale=scale, edgefactor=meta["edgefactor"], alpha=meta["alpha"], beta=meta["beta"],
        corebfs=meta["corebfs"], group=int(group), auto_tune=meta["auto_tune"],
        reorder_bits=meta["reorder_bits"], pred_size=meta["pred_size"],
        num_global_edges=meta["num_global_edges"], num_global_verts=meta["num_global_verts"],
        roots=roots, atd=atd, nedge=nedge, valid=valid,
        levels=np.stack(levels).astype(np.int8 if max(int(l.max()) for l in levels) < 127 else np.int16))
    if meta["corebfs"]:
        assert any_tree, name
        trees = np.stack(trees)
        forest = trees.max(axis=0)
        # a vertex's tree parent is the same in every search that writes it
        assert ((trees == -1) | (trees == forest[None, :])).all(), name
        climb = np.full((len(roots), 64), -1, np.int64)
        for i in range(len(roots)):
            c = np.nonzero((forest >= 0) & (trees[i] < 0))[0]
            assert c.size <= 64, (name, i, c.size)
            climb[i, : c.size] = c
        arrays["forest_parent"] = forest
        arrays["climb"] = climb
    path = os.path.join(out_dir, "reference_bfs_%s.npz" % name)
    np.savez_compressed(path, **arrays)
    return path


def main():
    only = set(sys.argv[1:])
    for name, scale, nroots, flags, group in CONFIGS:
        if only and name not in only:
            continue
        path = run_config(name, scale, nroots, flags, group, HERE)
        print("wrote", os.path.relpath(path, REPO), os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
