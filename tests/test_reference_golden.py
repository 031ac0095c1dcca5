"""The oracle against the reference's own CPU BFS (no GPU).

tests/golden/reference_bfs_*.npz hold what the reference's mpi/main.cc flow
with its stock BfsBase produced (tests/golden/make_reference_golden.py over
oracle/_ref/ref_dump*): roots from find_roots_in_large_graph, the
auto_tuning_data slots of every search, validate_bfs_result's traversed-edge
counts, the exact level of every vertex and, with CoreBFS, the pruned
forest's parents.  The oracle restatement must reproduce all of them bit for
bit from the same seeds and α/β.
"""
import glob
import os

import numpy as np
import pytest

import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "reference_bfs_*.npz")))
NAMES = [os.path.basename(f)[len("reference_bfs_"):-4] for f in FIXTURES]


def load(name):
    return dict(np.load(os.path.join(GOLDEN, "reference_bfs_%s.npz" % name)))


def test_fixtures_present():
    assert {"s12_plain", "s12_A", "s12_AC", "s12_AC_group", "s16_plain", "s16_C",
            "s16_AC_group", "s20_plain", "s20_AC_group"} <= set(NAMES)


_graphs = {}


def graph(scale):
    if scale not in _graphs:
        e = O.generate_edges(scale)
        _graphs[scale] = (e, O.Graph(e))
    return _graphs[scale]


@pytest.mark.parametrize("name", NAMES)
def test_oracle_reproduces_reference(built, name):
    d = load(name)
    scale = int(d["scale"])
    alpha, beta = float(d["alpha"]), float(d["beta"])
    edges, g = graph(scale)
    n = 1 << scale
    assert g.scale == scale
    if int(d["corebfs"]):
        core = O.Core(g, 16, alpha, beta)
        # with CoreBFS graph_ describes the 2-core (corebfs_adaptor.hpp:328-357)
        assert core.core_num_edges == int(d["num_global_edges"])
        assert core.core_num_verts == int(d["num_global_verts"])
        has_edge = core.has_edge()
        search = core.bfs
    else:
        assert g.num_edges == int(d["num_global_edges"])
        assert g.num_verts == int(d["num_global_verts"])
        has_edge = g.has_edge()
        search = g.bfs
    # root selection, including the re-pick of roots reaching <= 3 levels
    roots = O.find_roots_in_large_graph(has_edge, n, len(d["roots"]),
                                        lambda r: int(search(r, 16, 10.0, 14.0)[1][8]))
    assert np.array_equal(roots, d["roots"])
    for i, r in enumerate(roots):
        pred, at, _ = search(int(r), 16, alpha, beta)
        assert np.array_equal(at, d["atd"][i]), (i, at, d["atd"][i])
        lv, tree = O.resolve_levels(pred[:n])
        assert np.array_equal(lv, d["levels"][i].astype(np.int64)), i
        if int(d["corebfs"]):
            want = d["forest_parent"].astype(np.int64).copy()
            climb = d["climb"][i]
            want[climb[climb >= 0]] = -1
            assert np.array_equal(tree, want), i
        else:
            assert (tree < 0).all()
        err, cnt = O.validate(edges, n, pred[:n], int(r), corebfs=bool(int(d["corebfs"])),
                              nlocalverts=n)
        assert err == 0 and cnt == int(d["nedge"][i]), (i, err, cnt)


def test_reference_counts_are_pf_nedge():
    """validate_bfs_result's counts are the pf_nedge known answers
    (mpi/utils.hpp:3687-3733) for every fixture root."""
    for name in NAMES:
        d = load(name)
        assert (d["nedge"] == O.PF_NEDGE[int(d["scale"])]).all(), name
        assert d["valid"].all(), name


def test_resolve_levels_handles_tree_chains():
    # root 0 (level 0), core vertex 1 (level 1), tree chain 2 <- 3 <- 4
    # hanging off 1, vertex 5 unreached
    def enc(lv, p):
        return np.array((lv << 48) | p, np.uint64).view(np.int64)

    pred = np.array([enc(0, 0), enc(1, 0), enc(0xFFFF, 1), enc(0xFFFF, 2), enc(0xFFFF, 3), -1],
                    np.int64)
    lv, tree = O.resolve_levels(pred)
    assert lv.tolist() == [0, 1, 2, 3, 4, -1]
    assert tree.tolist() == [-1, -1, 1, 2, 3, -1]
    with pytest.raises(ValueError):
        O.resolve_levels(np.array([enc(0xFFFF, 1), enc(0xFFFF, 0)], np.int64))
