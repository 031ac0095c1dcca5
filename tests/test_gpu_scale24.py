"""SCALE 24 (a benchmark configuration) against the CPU oracle on the same
graph: the device's per-vertex levels equal the oracle's queue BFS for every
mode of the search -- plain with the reference's default alpha/beta, with
-A-tuned switch points, with CoreBFS on a group-reordered graph, and batched
-- and every parent array passes the Graph500 rules with the reference's
known traversed-edge count pf_nedge[24] (mpi/utils.hpp:3687-3733).
"""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

SCALE = 24
NROOTS = 4


@pytest.fixture(scope="module")
def reference_levels(built):
    edges = O.generate_edges(SCALE)
    g = O.Graph(edges)
    roots = [int(r) for r in O.find_roots(g.has_edge(), 1 << SCALE, NROOTS)]
    levels = {r: g.levels(r) for r in roots}
    return g.nverts, roots, levels


def _check(e, r, n, ref):
    assert np.array_equal(e.get_levels()[:n], ref), r
    err, cnt = e.validate(r)
    assert err == 0 and cnt == O.PF_NEDGE[SCALE], (r, err, cnt)


def test_scale24_plain_tuned_and_batch(reference_levels):
    import b200bfs

    n, roots, levels = reference_levels
    e = b200bfs.Engine(0)
    try:
        e.generate_graph(SCALE, 16)
        e.prepare(16)
        for r in roots:
            e.run(r)
            _check(e, r, n, levels[r])
        nedge = np.full(len(roots), float(O.PF_NEDGE[SCALE]))
        alpha, beta, _ = e.auto_tune(roots, nedge)
        for r in roots:
            e.run(r, 16, alpha, beta)
            _check(e, r, n, levels[r])
        e.run_batch(roots)
        for i, r in enumerate(roots):
            e.batch_select(i)
            _check(e, r, n, levels[r])
    finally:
        e.close()


def test_scale24_corebfs_group_reorder(reference_levels):
    import b200bfs

    n, roots, levels = reference_levels
    e = b200bfs.Engine(0)
    try:
        e.generate_graph(SCALE, 16, flags=b200bfs.BUILD_COREBFS | b200bfs.BUILD_GROUP_REORDER)
        e.prepare(16)
        nedge = np.full(len(roots), float(O.PF_NEDGE[SCALE]))
        alpha, beta, _ = e.auto_tune(roots, nedge)
        rep = e.tune_engine(roots, 16, alpha, beta,
                            b200bfs.TUNE_FORMS | b200bfs.TUNE_BATCH_ALPHA | b200bfs.TUNE_SWITCH)
        for r in roots:
            e.run(r, 16, rep.alpha, rep.beta)
            _check(e, r, n, levels[r])
        e.run_batch(roots, 16, 0.0, rep.beta)
        for i, r in enumerate(roots):
            e.batch_select(i)
            _check(e, r, n, levels[r])
    finally:
        e.close()
