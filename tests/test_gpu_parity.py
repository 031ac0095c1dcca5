"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Bit-exact: generated edges, CSR sizes, per-vertex levels, direction-switch
slots (auto_tuning_data), CoreBFS tree parents.  Parents are checked with the
Graph500 rules (oracle validator and the device validator) since BFS trees
are not unique.
"""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

SCALES = [10, 14, 16, 18, 20]


@pytest.fixture(scope="module")
def engine(built):
    import b200bfs

    e = b200bfs.Engine(0)
    yield e
    e.close()


@pytest.fixture(scope="module")
def oracle_graphs(built):
    cache = {}

    def get(scale):
        if scale not in cache:
            e = O.generate_edges(scale)
            cache[scale] = (e, O.Graph(e))
        return cache[scale]

    return get


@pytest.mark.parametrize("scale", [10, 16, 20])
def test_generator_bit_exact(engine, scale):
    m = (1 << scale) * 16
    for a, b in [(0, min(m, 100000)), (m - 5000, m)]:
        dev = engine.generate_edges(scale, a, b)
        ref = O.generate_edges(scale, start=a, end=b)
        assert np.array_equal(dev, ref)


def test_generator_bit_exact_scale28_sample(engine):
    m = (1 << 28) * 16
    for a in (0, 1 << 31, m - 4096):
        dev = engine.generate_edges(28, a, a + 4096)
        ref = O.generate_edges(28, start=a, end=a + 4096)
        assert np.array_equal(dev, ref)


def _check_search(engine, edges, g, roots, alpha=10.0, beta=14.0):
    for r in roots:
        r = int(r)
        at = engine.run(r, 16, alpha, beta)
        pred = engine.get_pred()
        n = g.nverts
        assert np.all(pred[n:] == -1)
        ref_pred, ref_at, ref_st = g.bfs(r, alpha=alpha, beta=beta)
        assert np.array_equal(O.pred_levels(pred[:n]), O.pred_levels(ref_pred)), r
        assert np.array_equal(at, ref_at), (r, at, ref_at)
        err, cnt = O.validate(edges, 1 << g.scale, pred[:n], r)
        assert err == 0, r
        derr, dcnt = engine.validate(r)
        assert derr == 0 and dcnt == cnt
        lv = engine.get_levels()
        assert np.array_equal(lv[:n], g.levels(r))
        st = engine.run_stats()
        assert st.levels == ref_st.levels and st.visited == ref_st.visited


@pytest.mark.parametrize("scale", SCALES)
def test_bfs_levels_bit_exact(engine, oracle_graphs, scale):
    edges, g = oracle_graphs(scale)
    engine.generate_graph(scale, 16)
    gi = engine.info()
    assert gi.scale == g.scale
    assert gi.num_global_edges == g.num_edges
    assert gi.num_global_verts == g.num_verts
    assert gi.pred_size == max(1 << scale, 1 << 16)
    assert np.array_equal(engine.has_edge_all()[: g.nverts], g.has_edge())
    roots = O.find_roots(g.has_edge(), 1 << g.scale, 8)
    engine.prepare(16)
    _check_search(engine, edges, g, roots)
    # the traversed-edge count of a giant-component root is pf_nedge
    # (mpi/utils.hpp:3687-3733); the sampled roots include such a root
    counts = set()
    for r in roots[:4]:
        engine.run(int(r), 16)
        err, cnt = engine.validate(int(r))
        assert err == 0
        counts.add(cnt)
    assert O.PF_NEDGE[scale] in counts
    engine.end()


def test_bfs_pf_nedge_scale20(engine, oracle_graphs):
    edges, g = oracle_graphs(20)
    engine.generate_graph(20, 16)
    engine.prepare(16)
    roots = O.find_roots(g.has_edge(), 1 << 20, 16)
    counts = []
    for r in roots:
        engine.run(int(r), 16)
        err, cnt = engine.validate(int(r))
        assert err == 0
        counts.append(cnt)
    assert counts.count(O.PF_NEDGE[20]) >= 12
    engine.end()


@pytest.mark.parametrize("alpha,beta", [(10.0, 14.0), (1e-9, 14.0), (1e9, 14.0), (2.0, 100.0),
                                        (30.0, 2.0)])
def test_switch_parameters(engine, oracle_graphs, alpha, beta):
    """Other alpha/beta (the -A tuner's knobs) keep levels exact and the
    switch levels equal to the reference rule."""
    edges, g = oracle_graphs(16)
    engine.generate_graph(16, 16)
    engine.prepare(16, alpha, beta)
    roots = O.find_roots(g.has_edge(), 1 << 16, 4)
    _check_search(engine, edges, g, roots, alpha, beta)
    engine.end()


def test_input_paths_match(engine, oracle_graphs):
    """Host int64 pairs, packed 12-byte records and a pre-symmetrised list
    build the same graph as the device generator."""
    import b200bfs

    edges, g = oracle_graphs(14)
    roots = O.find_roots(g.has_edge(), 1 << 14, 4)
    engine.build_from_edges(edges, 14)
    gi = engine.info()
    assert (gi.num_global_edges, gi.num_global_verts) == (g.num_edges, g.num_verts)
    engine.prepare(16)
    _check_search(engine, edges, g, roots)
    packed = np.zeros((edges.shape[0], 3), np.uint32)
    packed[:, 0] = edges[:, 0] & 0xFFFFFFFF
    packed[:, 1] = edges[:, 1] & 0xFFFFFFFF
    packed[:, 2] = ((edges[:, 0] >> 32) & 0xFFFF) | (((edges[:, 1] >> 32) & 0xFFFF) << 16)
    engine.build_from_packed(packed, 14)
    engine.prepare(16)
    _check_search(engine, edges, g, roots)
    loops = edges[:, 0] == edges[:, 1]
    sym = np.concatenate([edges[~loops], edges[~loops][:, ::-1]])
    engine.build_from_edges(sym, 14, b200bfs.BUILD_INPUT_SYMMETRIC)
    gi = engine.info()
    assert (gi.num_global_edges, gi.num_global_verts) == (g.num_edges, g.num_verts)
    engine.prepare(16)
    for r in roots:
        engine.run(int(r), 16)
        pred = engine.get_pred()[: g.nverts]
        assert np.array_equal(O.pred_levels(pred), g.levels(int(r)))
        assert O.validate(edges, 1 << 14, pred, int(r))[0] == 0
    engine.end()


def test_group_reorder(engine, oracle_graphs):
    import b200bfs

    edges, g = oracle_graphs(18)
    engine.generate_graph(18, 16, flags=b200bfs.BUILD_GROUP_REORDER)
    gi = engine.info()
    assert gi.reorder_bits == 16
    assert (gi.num_global_edges, gi.num_global_verts) == (g.num_edges, g.num_verts)
    engine.prepare(16)
    _check_search(engine, edges, g, O.find_roots(g.has_edge(), 1 << 18, 4))
    # neighbour lists: the oracle's neighbour sets, highest degree first
    row_ptr, col, inv, mdeg = engine.get_csr()
    rng = np.random.default_rng(3)
    for r in rng.integers(0, len(inv), 200):
        nb = col[row_ptr[r]:row_ptr[r + 1]]
        assert np.all(np.diff(mdeg[nb]) <= 0)
        v = int(inv[r])
        assert np.array_equal(np.sort(inv[nb]), g.col[g.row_ptr[v]:g.row_ptr[v + 1]])
    engine.end()


@pytest.mark.parametrize("scale,assemble", [(12, 0), (16, 0), (18, 0), (12, 1), (16, 1)])
def test_corebfs_parity(engine, oracle_graphs, scale, assemble):
    """assemble 1: tree parents come from the assembly pass's map, the climb
    is written after it."""
    import b200bfs

    edges, g = oracle_graphs(scale)
    core = O.Core(g)
    engine.generate_graph(scale, 16, flags=b200bfs.BUILD_COREBFS)
    engine.prepare(16)
    engine.set_option("pred_assemble", assemble)
    gi = engine.info()
    assert gi.corebfs == 1 and gi.prune_rounds == core.rounds
    assert gi.num_global_verts == core.core_num_verts
    assert gi.num_global_edges == core.core_num_edges
    assert gi.tree_vertices == int((core.tree_parent >= 0).sum())
    he = engine.has_edge_all()[: g.nverts]
    assert np.array_equal(he, core.has_edge())
    roots = O.find_roots(core.has_edge(), 1 << scale, 6)
    for r in roots:
        r = int(r)
        at = engine.run(r, 16)
        pred = engine.get_pred()[: g.nverts]
        ref_pred, ref_at, _ = core.bfs(r)
        # tree parents and path entries are unique, so those entries match
        tree = O.pred_levels(ref_pred) == 0xFFFF
        assert np.array_equal(pred[tree], ref_pred[tree])
        assert np.array_equal(O.pred_levels(pred), O.pred_levels(ref_pred))
        assert np.array_equal(at, ref_at)
        err, cnt = O.validate(edges, 1 << scale, pred, r, corebfs=True)
        assert err == 0
        derr, dcnt = engine.validate(r)
        assert derr == 0 and dcnt == cnt
        # exact levels, tree vertices filled in
        assert np.array_equal(engine.get_levels()[: g.nverts], g.levels(r))
    # tree parents are rewritten only along the climbs: after a batch result
    # and across roots they must still equal the reference's
    engine.run_batch([int(x) for x in roots[:3]])
    engine.batch_select(2)
    for r in roots[::-1]:
        r = int(r)
        engine.run(r, 16)
        pred = engine.get_pred()[: g.nverts]
        ref_pred, _, _ = core.bfs(r)
        tree = O.pred_levels(ref_pred) == 0xFFFF
        assert np.array_equal(pred[tree], ref_pred[tree])
        assert np.array_equal(O.pred_levels(pred), O.pred_levels(ref_pred))
    engine.set_option("pred_assemble", 1)
    engine.end()


def test_sparse_assembly_restores_climbs(engine, oracle_graphs):
    """After a search that used the assembly pass, the next pass writes only
    the groups of four ids that hold a searched row; the previous root's
    entry and the previous CoreBFS climb must go back to their values.
    Roots at the ends of the deepest climbs, alternating with core roots
    and with each other, leave tree entries and levels equal to the oracle's
    after every search."""
    import b200bfs

    scale = 14
    edges, g = oracle_graphs(scale)
    core = O.Core(g)
    engine.generate_graph(scale, 16, flags=b200bfs.BUILD_COREBFS)
    engine.prepare(16)
    engine.set_option("pred_assemble", 1)
    tp = core.tree_parent
    depth = np.zeros(g.nverts, dtype=np.int64)
    for v in np.nonzero(tp >= 0)[0]:
        d, u = 0, int(v)
        while tp[u] >= 0:
            u = int(tp[u])
            d += 1
        depth[v] = d
    deep = [int(v) for v in np.argsort(-depth, kind="stable")[:3] if depth[v] > 0]
    assert len(deep) == 3 and depth[deep[0]] >= 2
    he = core.has_edge()
    core_roots = [int(r) for r in O.find_roots(he, 1 << scale, 8) if tp[int(r)] < 0][:2]
    assert len(core_roots) == 2
    seq = [deep[0], core_roots[0], deep[1], deep[2], deep[0], core_roots[1], deep[1]]
    for r in seq:
        engine.run(r, 16)
        pred = engine.get_pred()[: g.nverts]
        ref_pred, _, _ = core.bfs(r)
        tree = O.pred_levels(ref_pred) == 0xFFFF
        assert np.array_equal(pred[tree], ref_pred[tree]), r
        assert np.array_equal(O.pred_levels(pred), O.pred_levels(ref_pred)), r
        err, cnt = O.validate(edges, 1 << scale, pred, r, corebfs=True)
        assert err == 0, r
        assert np.array_equal(engine.get_levels()[: g.nverts], g.levels(r)), r
    engine.end()


def test_errors_are_status_codes(engine):
    import b200bfs

    with pytest.raises(b200bfs.B200BfsError) as ei:
        engine.generate_graph(31, 16)
    assert ei.value.code == 1
    engine.generate_graph(10, 16)
    engine.end()
    with pytest.raises(b200bfs.B200BfsError) as ei:
        engine.run(0, 16)
    assert ei.value.code == 4
    engine.prepare(16)
    with pytest.raises(b200bfs.B200BfsError) as ei:
        engine.run(1 << 12, 16)
    assert ei.value.code == 1
    engine.end()


def test_hbm_budget_admission(built):
    """A graph larger than the HBM budget fails cleanly with ERR_OOM and the
    handle stays usable."""
    import b200bfs

    e = b200bfs.Engine(0, hbm_budget_bytes=64 << 20)
    with pytest.raises(b200bfs.B200BfsError) as ei:
        e.generate_graph(22, 16)
    assert ei.value.code == 3
    e.generate_graph(12, 16)
    e.prepare(16)
    e.run(int(np.nonzero(e.has_edge_all())[0][0]), 16)
    e.close()


@pytest.mark.parametrize("bu,td,first", [(1, 1, 1), (2, 2, 1), (3, 1, 1), (4, 2, 0), (4, 3, 1),
                                         (4, 4, 1), (4, 5, 0), (4, 6, 1), (2, 7, 1)])
def test_kernel_forms_agree(engine, oracle_graphs, bu, td, first):
    """Every bottom-up / top-down kernel form gives the reference levels."""
    edges, g = oracle_graphs(18)
    engine.generate_graph(18, 16)
    engine.set_option("bu_kernel", bu)
    engine.set_option("td_kernel", td)
    engine.set_option("bu_first", first)
    engine.prepare(16)
    try:
        _check_search(engine, edges, g, O.find_roots(g.has_edge(), 1 << 18, 3))
        _check_search(engine, edges, g, O.find_roots(g.has_edge(), 1 << 18, 2), alpha=1e-9)
    finally:
        engine.set_option("bu_kernel", 2)
        engine.set_option("td_kernel", 4)
        engine.set_option("bu_first", 1)
        engine.end()


def test_engine_tuner_keeps_results_exact(engine, oracle_graphs):
    """b200bfs_tune_engine picks kernel forms and the batch alpha by timing;
    searches and batches with its choices still give the oracle's levels."""
    import b200bfs

    edges, g = oracle_graphs(18)
    engine.generate_graph(18, 16)
    engine.prepare(16)
    roots = O.find_roots(g.has_edge(), 1 << 18, 8)
    try:
        rep = engine.tune_engine(roots)
        assert 1 <= rep.bu_kernel <= 4 and rep.td_kernel in (1, 3, 4, 5, 6, 7)
        assert rep.batch_alpha in (10.0, 20.0, 30.0, 50.0, 100.0, 200.0, 400.0)
        assert rep.searches > 0 and rep.batches == 14 and rep.single_ms > 0 and rep.batch_ms > 0
        assert (rep.alpha, rep.beta) == (10.0, 14.0)  # not refined without TUNE_SWITCH
        _check_search(engine, edges, g, roots[:3])
        engine.run_batch(roots, 16, 0.0)  # alpha <= 0: the tuned batch alpha
        for i, r in enumerate(roots):
            engine.batch_select(i)
            assert np.array_equal(engine.get_levels()[: g.nverts], g.levels(int(r)))
        # alpha/beta refinement: each is the input scaled by one of the
        # tried factors; the oracle with the same alpha/beta gives the same
        # switch levels (auto_tuning_data) and levels
        rep = engine.tune_engine(roots, 16, 10.0, 14.0, b200bfs.TUNE_SWITCH)
        assert rep.alpha in [10.0 * f for f in (0.5, 0.7, 1.0, 1.4, 2.0)]
        assert rep.beta in [14.0 * f for f in (0.5, 0.7, 1.0, 1.4, 2.0)]
        _check_search(engine, edges, g, roots[:3], alpha=rep.alpha, beta=rep.beta)
    finally:
        engine.set_option("bu_kernel", 2)
        engine.set_option("td_kernel", 4)
        engine.set_option("batch_alpha", 30)
        engine.end()


@pytest.mark.parametrize("alpha,beta,flags", [(10.0, 14.0, 0), (1e-9, 14.0, 0), (1e9, 14.0, 0),
                                              (2.0, 100.0, 0), (30.0, 2.0, 0), (10.0, 14.0, 3)])
def test_device_level_loop_matches_host_loop(engine, oracle_graphs, alpha, beta, flags):
    """The level loop run on the device (one CUDA graph per search) applies
    the same switch rule: levels, auto_tuning_data, run statistics and
    per-level records equal the host loop's and the oracle's."""
    import b200bfs

    edges, g = oracle_graphs(16)
    engine.generate_graph(16, 16, flags=flags)
    engine.prepare(16, alpha, beta)
    if flags & b200bfs.BUILD_COREBFS:
        roots = O.find_roots(O.Core(g).has_edge(), 1 << 16, 4)
    else:
        roots = O.find_roots(g.has_edge(), 1 << 16, 4)
    keys = ("levels", "num_td_levels", "num_bu_levels", "bu_level_mask", "visited",
            "edges_scanned_td", "edges_scanned_bu", "algorithmic_bytes", "td_bytes", "bu_bytes")
    try:
        engine.run(int(roots[0]), 16, alpha, beta)  # the first search fills pred once
        for r in roots:
            r = int(r)
            engine.set_option("single_graph", 0)
            at_h = engine.run(r, 16, alpha, beta)
            st_h = engine.run_stats()
            lv_h = [{k: v for k, v in x.items() if k != "ms"} for x in engine.level_stats()]
            engine.set_option("single_graph", 1)
            at_d = engine.run(r, 16, alpha, beta)
            st_d = engine.run_stats()
            lv_d = [{k: v for k, v in x.items() if k != "ms"} for x in engine.level_stats()]
            assert np.array_equal(at_h, at_d)
            for k in keys:
                if k == "algorithmic_bytes" and flags & b200bfs.BUILD_COREBFS:
                    continue  # includes the tree rewrite, which depends on the previous climb
                assert getattr(st_h, k) == getattr(st_d, k), k
            assert lv_h == lv_d
            assert np.array_equal(engine.get_levels()[: g.nverts], g.levels(r))
            err, cnt = engine.validate(r)
            assert err == 0
        if not flags:
            engine.set_option("single_graph", 1)
            _check_search(engine, edges, g, roots, alpha, beta)
    finally:
        engine.set_option("single_graph", 0)
        engine.end()


@pytest.mark.parametrize("single_graph,assemble", [(0, 0), (1, 0), (0, 1), (1, 1)])
def test_pred_exact_across_searches(engine, oracle_graphs, single_graph, assemble):
    """Without the assembly pass pred is not refilled with -1 before every
    search: each search resets the rows it leaves unreached and the previous
    root's entry.  With it (pred_assemble 1) every entry is rewritten from the
    row-order buffer, whose rows a search did not reach hold stale entries.
    Searches that reach different vertex sets (giant component, a small
    component, an isolated vertex, a batch result in between, a switch of
    the option) must each leave exactly their own result."""
    edges, g = oracle_graphs(16)
    engine.generate_graph(16, 16)
    engine.prepare(16)
    he = g.has_edge()
    big = [int(r) for r in O.find_roots(he, 1 << 16, 2)]
    small = None
    for v in np.nonzero(he)[0][::-1]:
        lv = g.levels(int(v))
        if 1 < int((lv >= 0).sum()) < 1000:
            small = int(v)
            break
    assert small is not None
    isolated = int(np.nonzero(he == 0)[0][0])
    def check(r):
        engine.run(r)
        assert np.array_equal(engine.get_levels()[: g.nverts], g.levels(r)), r
        pred = engine.get_pred()
        assert np.all(pred[g.nverts:] == -1)
        assert np.all(pred[: g.nverts][g.levels(r) < 0] == -1), r
        err, _ = engine.validate(r)
        assert err == 0, r

    try:
        engine.set_option("single_graph", single_graph)
        engine.set_option("pred_assemble", assemble)
        for r in [big[0], small, big[1], isolated, small, big[0]]:
            check(r)
        engine.run_batch([small, big[1]])
        engine.batch_select(0)
        check(big[0])
        engine.batch_select(1)
        check(small)
        engine.set_option("pred_assemble", 1 - assemble)
        for r in [big[1], small, isolated]:
            check(r)
    finally:
        engine.set_option("single_graph", 0)
        engine.set_option("pred_assemble", 1)
        engine.end()


@pytest.mark.parametrize("scale,flags", [(16, 0), (20, 2)])
def test_find_roots_matches_oracle(engine, oracle_graphs, scale, flags):
    """b200bfs_find_roots against the oracle's find_roots
    (benchmark_helper.hpp:527-562) for several seeds, plain and with group
    reordering (has_edge is by original id either way)."""
    edges, g = oracle_graphs(scale)
    engine.generate_graph(scale, 16, flags=flags)
    for r1, r2 in ((0, 0), (1, 0), (2, 0), (5, 3), (17, 0)):
        dev = engine.find_roots(16, r1, r2)
        ref = O.find_roots(g.has_edge(), 1 << scale, 16, r1, r2)
        assert np.array_equal(dev, ref), (r1, r2)


@pytest.mark.parametrize("bu,sparse,spec", [(2, 0, 0), (2, 1, 0), (2, 1, 1), (2, 0, 1), (3, 1, 0),
                                             (3, 1, 1), (4, 1, 0), (4, 1, 1), (4, 0, 0)])
def test_bottom_up_sparse_levels_agree(engine, oracle_graphs, bu, sparse, spec):
    """Bottom-up forms with (bu_sparse 1) and without the skip of full
    bitmap words on levels with few unvisited rows, and form 2 with and
    without the early first-neighbour loads on levels where most rows are
    unvisited (bu_spec); every level after the first runs bottom-up
    (force_direction 2), so the second level takes the early-load path and
    the last levels the sparse path."""
    edges, g = oracle_graphs(18)
    engine.generate_graph(18, 16)
    engine.set_option("bu_kernel", bu)
    engine.set_option("bu_sparse", sparse)
    engine.set_option("bu_spec", spec)
    engine.set_option("force_direction", 2)
    engine.prepare(16)
    try:
        for r in O.find_roots(g.has_edge(), 1 << 18, 3):
            engine.run(int(r), 16)
            assert np.array_equal(engine.get_levels()[: g.nverts], g.levels(int(r)))
            err, cnt = O.validate(edges, 1 << 18, engine.get_pred()[: g.nverts], int(r))
            assert err == 0
    finally:
        engine.set_option("bu_kernel", 2)
        engine.set_option("bu_sparse", 1)
        engine.set_option("bu_spec", 1)
        engine.set_option("force_direction", 0)
        engine.end()
