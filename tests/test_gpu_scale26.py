"""SCALE 26 single-source searches run three ways -- plain, with -A tuned
switch points, and -A -C (CoreBFS) with group reordering -- plus a 64-root
batch on the same graph.

Anchors: the CPU oracle generates the SCALE 26 graph itself on the host
(about 50 GB of host memory, a minute or two on the box's cores), builds its
own CSR and searches it; the engine's CSR sizes, root sample, per-vertex
levels and auto_tuning_data slots (plain α/β) must equal the oracle's for
the first roots, and the device validator's traversed-edge count must equal
the oracle validator's.  Levels depend only on the graph and the root, so the
-A, -A -C (group reordering) and batched searches must give the same levels
again; every parent array passes the Graph500 rules on the device with the
reference's known answer pf_nedge[26] (mpi/utils.hpp:3687-3733).
"""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

SCALE = 26
NROOTS = 8
NORACLE = 4  # roots also searched by the CPU oracle


@pytest.fixture(scope="module")
def plain_levels(built):
    import b200bfs

    e = b200bfs.Engine(0)
    e.generate_graph(SCALE, 16)
    e.prepare(16)
    roots = [int(r) for r in e.find_roots(NROOTS)]
    levels = {}
    for r in roots:
        e.run(r)
        err, cnt = e.validate(r)
        assert err == 0 and cnt == O.PF_NEDGE[SCALE], r
        levels[r] = e.get_levels()
    # -A: tuned alpha/beta move the switch levels, not the levels
    nedge = np.full(len(roots), float(O.PF_NEDGE[SCALE]))
    alpha, beta, _ = e.auto_tune(roots, nedge)
    for r in roots:
        e.run(r, 16, alpha, beta)
        assert np.array_equal(e.get_levels(), levels[r]), r
        err, cnt = e.validate(r)
        assert err == 0 and cnt == O.PF_NEDGE[SCALE]
    # 64-root batch (roots repeated to fill it)
    batch = (roots * 8)[:64]
    e.run_batch(batch)
    for i in (0, 5, 13, 63):
        e.batch_select(i)
        assert np.array_equal(e.get_levels(), levels[batch[i]]), i
        err, cnt = e.validate(batch[i])
        assert err == 0 and cnt == O.PF_NEDGE[SCALE]
    e.close()
    return roots, levels


@pytest.fixture(scope="module")
def oracle26(plain_levels):
    """The oracle's own graph, generated and built on the host."""
    edges = O.generate_edges(SCALE)
    g = O.Graph(edges)
    yield edges, g
    del g, edges


def test_scale26_matches_oracle_graph(plain_levels, oracle26):
    import b200bfs

    roots, levels = plain_levels
    edges, g = oracle26
    e = b200bfs.Engine(0)
    e.generate_graph(SCALE, 16)
    gi = e.info()
    assert gi.num_global_edges == g.num_edges and gi.num_global_verts == g.num_verts
    e.prepare(16)
    assert np.array_equal(e.find_roots(NROOTS), O.find_roots(g.has_edge(), 1 << SCALE, NROOTS))
    n = 1 << SCALE
    for r in roots[:NORACLE]:
        at = e.run(r, 16)
        pred, ref_at, _ = g.bfs(r)
        assert np.array_equal(at, ref_at), (r, at, ref_at)
        assert np.array_equal(levels[r][:n], O.pred_levels(pred)), r
        err, cnt = O.validate(edges, n, e.get_pred()[:n], r)
        assert err == 0 and cnt == O.PF_NEDGE[SCALE], r
        assert e.validate(r) == (0, cnt)
    e.close()


def test_scale26_plain_tuned_and_batch(plain_levels):
    roots, levels = plain_levels
    assert len(roots) == NROOTS and all(int(lv.max()) >= 4 for lv in levels.values())


def test_scale26_corebfs_group_reorder(plain_levels):
    import b200bfs

    roots, levels = plain_levels
    e = b200bfs.Engine(0)
    e.generate_graph(SCALE, 16, flags=b200bfs.BUILD_COREBFS | b200bfs.BUILD_GROUP_REORDER)
    e.prepare(16)
    nedge = np.full(len(roots), float(O.PF_NEDGE[SCALE]))
    alpha, beta, _ = e.auto_tune(roots, nedge)
    for r in roots:
        e.run(r, 16, alpha, beta)
        assert np.array_equal(e.get_levels(), levels[r]), r
        err, cnt = e.validate(r)
        assert err == 0 and cnt == O.PF_NEDGE[SCALE], r
    e.run_batch(roots)
    for i, r in enumerate(roots):
        e.batch_select(i)
        assert np.array_equal(e.get_levels(), levels[r]), r
    e.close()
