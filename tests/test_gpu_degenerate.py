"""Degenerate and ragged inputs.

What the host refuses before any kernel runs (an empty edge list, an edge
list of self-loops only, which leaves no row, ids outside [0, 2^30), a
CoreBFS graph whose 2-core is empty), and that the engine stays usable
afterwards; and small ragged graphs -- one edge, duplicates and self-loops,
two components, a star, a random graph of skewed degrees -- whose levels
and parents from every kind of root (a hub, a leaf, a root in the smaller
component, a vertex without edges) must equal the oracle's and pass its
validator, with the bottom-up levels forced too (force_direction 2), where
the last bitmap word of a graph of a few rows is mostly padding.  A root
without edges past the last used vertex is a Graph500 range error, and the
device validator must report what the oracle does."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _cases():
    rng = np.random.default_rng(7)
    n, m = 300, 900
    ragged = np.stack([rng.integers(0, n, m), (rng.integers(0, n, m) ** 2) % n], axis=1)
    return {
        "single_edge": np.array([[0, 1]]),
        "duplicates_and_loops": np.array([[0, 1], [1, 0], [0, 1], [1, 1], [2, 2], [1, 2], [2, 1]]),
        "two_components": np.array([[0, 1], [1, 2], [2, 3], [10, 11], [11, 12]]),
        "star": np.array([[0, i] for i in range(1, 101)]),
        "ragged": ragged,
    }


CASES = _cases()


def test_refused_inputs_leave_the_engine_usable(built):
    import b200bfs

    e = b200bfs.Engine(0)
    bad = [np.zeros((0, 2), np.int64),                   # no edges at all
           np.array([[0, 0], [3, 3], [7, 7]]),           # self-loops only: no row
           np.array([[0, 1], [2, -1]]),                  # negative id
           np.array([[0, 1 << 30]])]                     # id beyond 2^30
    for edges in bad:
        with pytest.raises(b200bfs.B200BfsError) as ei:
            e.build_from_edges(edges)
        assert ei.value.code == 1, edges
    with pytest.raises(b200bfs.B200BfsError) as ei:  # a star has an empty 2-core
        e.build_from_edges(CASES["star"], flags=b200bfs.BUILD_COREBFS)
    assert ei.value.code == 1
    e.build_from_edges(np.array([[0, 1], [1, 2]]))
    e.prepare(16)
    e.run(0, 16)
    assert list(e.get_levels()[:3]) == [0, 1, 2]
    e.close()


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("force", [0, 2])
def test_small_ragged_graphs_match_oracle(built, name, force):
    import b200bfs

    edges = CASES[name].astype(np.int64)
    g = O.Graph(edges)
    e = b200bfs.Engine(0)
    e.build_from_edges(edges)
    gi = e.info()
    assert gi.scale == g.scale and gi.num_global_edges == g.num_edges
    e.set_option("force_direction", force)
    e.prepare(16)
    he = g.has_edge()
    with_edges = np.nonzero(he)[0]
    roots = list(with_edges[:3]) + [int(with_edges[-1])]
    if (he[: g.nverts] == 0).any():
        roots.append(int(np.nonzero(he == 0)[0][0]))  # a root without edges
    # main.cc validates against max_used_vertex + 1 vertices (find_max_used_vertex,
    # benchmark_helper.hpp:564-582, main.cc:647): a root past the last vertex
    # with an edge is a range error there, in the oracle and on the device alike
    nglobal = int(with_edges.max()) + 1
    try:
        for r in roots:
            r = int(r)
            e.run(r, 16)
            pred = e.get_pred()
            assert np.all(pred[g.nverts:] == -1)
            assert np.array_equal(e.get_levels()[: g.nverts], g.levels(r)), (name, r)
            err, cnt = O.validate(edges, nglobal, pred[: g.nverts], r)
            assert (err == 0) == (r < nglobal), (name, r, err)
            derr, dcnt = e.validate(r)
            assert (derr, dcnt) == (err, cnt), (name, r)
    finally:
        e.close()
