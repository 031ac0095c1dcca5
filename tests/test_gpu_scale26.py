"""SCALE 26 single-source searches run three ways -- plain, with -A tuned
switch points, and -A -C (CoreBFS) with group reordering -- plus a 64-root
batch on the same graph.

At this size the CPU oracle is too slow to run here, so parity rests on
size-independent properties: per-vertex levels depend only on the graph and
the root, so all four ways must give identical levels; every parent array
must pass the Graph500 rules on the device; and the traversed-edge count of
every root in the giant component equals the reference's known answer
pf_nedge[26] (mpi/utils.hpp:3687-3733).
"""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

SCALE = 26
NROOTS = 8


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
