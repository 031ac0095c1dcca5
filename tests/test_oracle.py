"""CPU oracle checks against the reference's known answers (no GPU)."""
import numpy as np
import pytest

import oracle as O


@pytest.fixture(scope="module")
def graphs(built):
    out = {}
    for s in (10, 12, 14, 16):
        e = O.generate_edges(s)
        out[s] = (e, O.Graph(e))
    return out


def test_mrg_constants():
    # the double conversion constants are (2^31-1)^-1 and (2^31-1)^-2
    assert 4.656612875245796924105750827e-10 == 1.0 / 2147483647.0
    assert abs(2.168404346990492787e-19 - 1.0 / 2147483647.0 ** 2) < 1e-33


def test_mrg_matrix_powers(built):
    p = 0x7FFFFFFF
    a1 = O.mrg_pow2_matrix(1).astype(object)
    a0 = O.mrg_pow2_matrix(0).astype(object)
    assert ((a0.dot(a0)) % p == a1).all()
    assert a0[0, 0] == 107374182 and a0[0, 4] == 104480


@pytest.mark.parametrize("scale", [10, 12, 14, 16])
def test_pf_nedge_known_answer(graphs, scale):
    """generate -> symmetrize -> BFS -> validate reproduces pf_nedge[SCALE]
    (mpi/utils.hpp:3687-3733) for every sampled root in the giant component."""
    edges, g = graphs[scale]
    assert g.scale == scale
    roots = O.find_roots(g.has_edge(), 1 << g.scale, 4)
    assert len(roots) == 4 and len(set(roots.tolist())) == 4
    counts = set()
    for r in roots:
        pred, at, st = g.bfs(int(r))
        err, cnt = O.validate(edges, 1 << g.scale, pred, int(r))
        assert err == 0
        assert np.array_equal(O.pred_levels(pred), g.levels(int(r)))
        counts.add(cnt)
    assert O.PF_NEDGE[scale] in counts


def test_pf_nedge_scale18(built):
    e = O.generate_edges(18)
    g = O.Graph(e)
    r = int(O.find_roots(g.has_edge(), 1 << g.scale, 1)[0])
    pred, _, _ = g.bfs(r)
    err, cnt = O.validate(e, 1 << g.scale, pred, r)
    assert err == 0 and cnt == O.PF_NEDGE[18]


def test_direction_switch_slots(graphs):
    """auto_tuning_data slots follow bfs.hpp:3413-3457 (T2B before B2T)."""
    _, g = graphs[16]
    r = int(O.find_roots(g.has_edge(), 1 << g.scale, 1)[0])
    _, at, st = g.bfs(r)
    assert at[8] == st.levels
    assert at[2] >= 1 and at[1] == g.num_edges
    assert at[0] > g.num_edges / 10.0
    if at[5] != -1:
        assert at[5] > at[2] and at[4] == g.num_verts
    # a tiny alpha (threshold num_edges / alpha never reached) keeps the
    # whole search top-down with the same levels
    pred_td, at_td, st_td = g.bfs(r, alpha=1e-9)
    assert st_td.edges_bu == 0 and at_td[2] == -1
    assert np.array_equal(O.pred_levels(pred_td), g.levels(r))


def test_validator_rejects_corruption(graphs):
    """Host-side fault injection: corrupted parent arrays must fail the
    Graph500 rules (validate.hpp:607-976)."""
    edges, g = graphs[14]
    r = int(O.find_roots(g.has_edge(), 1 << g.scale, 1)[0])
    pred, _, _ = g.bfs(r)
    assert O.validate(edges, 1 << g.scale, pred, r)[0] == 0
    reached = np.nonzero((pred != -1) & (np.arange(pred.size) != r))[0]
    v = int(reached[len(reached) // 2])
    bad = pred.copy()
    bad[v] = (bad[v] & ~0xFFFFFFFFFFFF) | ((v + 1) % g.nverts)  # parent without an edge / wrong
    assert O.validate(edges, 1 << g.scale, bad, r)[0] > 0
    bad = pred.copy()
    bad[v] = int(bad[v]) + (1 << 48)  # wrong level
    assert O.validate(edges, 1 << g.scale, bad, r)[0] > 0
    bad = pred.copy()
    bad[r] = -1  # root not its own parent
    assert O.validate(edges, 1 << g.scale, bad, r)[0] > 0
    bad = pred.copy()
    bad[v] = -1  # reachable vertex left unreached
    assert O.validate(edges, 1 << g.scale, bad, r)[0] > 0


@pytest.mark.parametrize("scale", [12, 16])
def test_corebfs_oracle(graphs, scale):
    """CoreBFS (-C): pruned trees + 2-core search validate with the CoreBFS
    depth rebuild and give the same traversed-edge count and levels."""
    edges, g = graphs[scale]
    core = O.Core(g)
    assert 0 < core.rounds <= 32
    he = core.has_edge()
    roots = O.find_roots(he, 1 << g.scale, 3)
    for r in roots:
        r = int(r)
        pred, at, st = core.bfs(r)
        err, cnt = O.validate(edges, 1 << g.scale, pred, r, corebfs=True)
        assert err == 0
        lv_plain = g.levels(r)
        if lv_plain[r] == 0 and (lv_plain >= 0).sum() > 100:
            assert cnt == O.PF_NEDGE[scale]
        # levels of core vertices are exact; tree vertices carry 0xFFFF
        lv = O.pred_levels(pred)
        known = (lv >= 0) & (lv != 0xFFFF)
        assert np.array_equal(lv[known], lv_plain[known])


def test_find_roots_deterministic(graphs):
    _, g = graphs[14]
    a = O.find_roots(g.has_edge(), 1 << g.scale, 16)
    b = O.find_roots(g.has_edge(), 1 << g.scale, 16)
    assert np.array_equal(a, b)
    assert all(g.has_edge()[a] == 1)
    c = O.find_roots(g.has_edge(), 1 << g.scale, 16, r1=1)
    assert not np.array_equal(a, c)
