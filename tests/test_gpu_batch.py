"""Batched multi-source search (b200bfs_run_batch) through the C ABI.

Every root of a batch must get exactly the per-vertex levels of a
single-source search from that root (the oracle's queue BFS), whatever the
per-root direction choices were; the parents rebuilt by b200bfs_batch_select
must pass the Graph500 rules (oracle validator and device validator) with the
same traversed-edge count as the oracle.
"""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine(built):
    import b200bfs

    e = b200bfs.Engine(0)
    yield e
    e.close()


@pytest.fixture(scope="module")
def graphs(built):
    cache = {}

    def get(scale):
        if scale not in cache:
            e = O.generate_edges(scale)
            cache[scale] = (e, O.Graph(e))
        return cache[scale]

    return get


def _check_batch(engine, edges, g, roots, alpha=30.0, corebfs=False):
    roots = [int(r) for r in roots]
    st = engine.run_batch(roots, 16, alpha)
    assert st.num_roots == len(roots)
    assert st.ms > 0
    nglobal = 1 << g.scale
    for i, r in enumerate(roots):
        engine.batch_select(i)
        lv = engine.get_levels()[: g.nverts]
        assert np.array_equal(lv, g.levels(r)), (i, r)
        pred = engine.get_pred()[: g.nverts]
        err, cnt = O.validate(edges, nglobal, pred, r, corebfs=corebfs)
        assert err == 0, (i, r)
        derr, dcnt = engine.validate(r)
        assert derr == 0 and dcnt == cnt, (i, r)
    return st


@pytest.mark.parametrize("scale,k", [(10, 64), (16, 1), (16, 8), (18, 64), (20, 32)])
def test_batch_levels_bit_exact(engine, graphs, scale, k):
    edges, g = graphs(scale)
    engine.generate_graph(scale, 16)
    engine.prepare(16)
    roots = O.find_roots(g.has_edge(), 1 << scale, k)
    st = _check_batch(engine, edges, g, roots)
    assert st.levels == max(int(g.levels(int(r)).max()) for r in roots)


@pytest.mark.parametrize("alpha", [1e-9, 1e9, 10.0, 30.0])
def test_batch_any_direction_gives_same_levels(engine, graphs, alpha):
    """alpha 1e-9 keeps every root top-down, 1e9 sends each root bottom-up
    after its first level: levels must not change."""
    edges, g = graphs(16)
    engine.generate_graph(16, 16)
    engine.prepare(16)
    roots = O.find_roots(g.has_edge(), 1 << 16, 64)
    st = _check_batch(engine, edges, g, roots, alpha=alpha)
    if alpha == 1e-9:
        assert st.num_bu_levels == 0
    if alpha == 1e9:
        assert st.num_bu_levels > 0


def test_batch_host_loop_and_graph_agree(engine, graphs):
    """The level loop run by the host (with per-level timings) and as a CUDA
    graph on the device give the same levels and statistics."""
    edges, g = graphs(16)
    engine.generate_graph(16, 16)
    engine.prepare(16)
    roots = O.find_roots(g.has_edge(), 1 << 16, 64)
    try:
        engine.set_option("batch_graph", 0)
        a = _check_batch(engine, edges, g, roots)
        lv = engine.level_stats()
        assert lv and all(x["ms"] > 0 for x in lv)
        engine.set_option("batch_graph", 1)
        b = _check_batch(engine, edges, g, roots)
    finally:
        engine.set_option("batch_graph", 1)
    for f in ("levels", "num_td_levels", "num_bu_levels", "edges_scanned_td", "edges_scanned_bu",
              "algorithmic_bytes"):
        assert getattr(a, f) == getattr(b, f), f


def test_batch_duplicate_and_isolated_roots(engine, graphs):
    edges, g = graphs(14)
    engine.generate_graph(14, 16)
    engine.prepare(16)
    he = g.has_edge()
    good = O.find_roots(he, 1 << 14, 4)
    isolated = int(np.nonzero(he == 0)[0][0])
    roots = [good[0], good[1], good[0], isolated, good[2], good[3], good[1]]
    _check_batch(engine, edges, g, roots)


@pytest.mark.parametrize("scale", [12, 16])
def test_batch_corebfs(engine, graphs, scale):
    import b200bfs

    edges, g = graphs(scale)
    core = O.Core(g)
    engine.generate_graph(scale, 16, flags=b200bfs.BUILD_COREBFS)
    engine.prepare(16)
    roots = O.find_roots(core.has_edge(), 1 << scale, 64)
    _check_batch(engine, edges, g, roots, corebfs=True)


def test_batch_group_reorder_corebfs(engine, graphs):
    import b200bfs

    edges, g = graphs(16)
    core = O.Core(g)
    engine.generate_graph(16, 16, flags=b200bfs.BUILD_COREBFS | b200bfs.BUILD_GROUP_REORDER)
    engine.prepare(16)
    roots = O.find_roots(core.has_edge(), 1 << 16, 64, 2)
    _check_batch(engine, edges, g, roots, corebfs=True)


def test_batch_long_path_grows_planes(engine):
    """A 60-vertex path has 60 levels: more than the 16 level planes a batch
    starts with, so the plane pool must grow during the search."""
    n = 60
    edges = np.stack([np.arange(n - 1), np.arange(1, n)], axis=1).astype(np.int64)
    g = O.Graph(edges)
    engine.build_from_edges(edges)
    engine.prepare(16)
    roots = [0, 17, 59, 30]
    st = _check_batch(engine, edges, g, roots)
    assert st.levels == 59


def test_consecutive_batches_different_roots(engine, graphs):
    """Each batch starts from the previous batch's planes: level 0 is cleared
    only at the rows the previous batch seeded there, so batches over
    different root sets (and different batch sizes) must not see each
    other's roots; the probe depth of the sweep must not change levels."""
    edges, g = graphs(16)
    engine.generate_graph(16, 16)
    engine.prepare(16)
    he = g.has_edge()
    sets = [O.find_roots(he, 1 << 16, 64, 7), O.find_roots(he, 1 << 16, 9, 8),
            O.find_roots(he, 1 << 16, 33, 9)]
    try:
        for probe, roots in zip((4, 128, 1024), sets):
            engine.set_option("batch_probe", probe)
            roots = [int(r) for r in roots]
            engine.run_batch(roots)
            for i in (0, len(roots) // 2, len(roots) - 1):
                engine.batch_select(i)
                assert np.array_equal(engine.get_levels()[: g.nverts], g.levels(roots[i])), (probe, i)
    finally:
        engine.set_option("batch_probe", 128)


def test_batch_then_single_root(engine, graphs):
    edges, g = graphs(14)
    engine.generate_graph(14, 16)
    engine.prepare(16)
    roots = O.find_roots(g.has_edge(), 1 << 14, 8)
    engine.run_batch(roots)
    engine.run(int(roots[3]))
    assert np.array_equal(engine.get_levels()[: g.nverts], g.levels(int(roots[3])))
    engine.batch_select(5)
    assert np.array_equal(engine.get_levels()[: g.nverts], g.levels(int(roots[5])))


def test_batch_errors(engine, graphs):
    import b200bfs

    edges, g = graphs(10)
    engine.generate_graph(10, 16)
    with pytest.raises(b200bfs.B200BfsError) as ex:
        engine.run_batch([1])
    assert ex.value.code == 4  # STATE: prepare not called
    engine.prepare(16)
    with pytest.raises(b200bfs.B200BfsError) as ex:
        engine.batch_select(0)
    assert ex.value.code == 4
    for bad in ([], list(range(65)), [1 << 20]):
        with pytest.raises(b200bfs.B200BfsError) as ex:
            engine.run_batch(bad)
        assert ex.value.code == 1
    engine.run_batch([int(r) for r in O.find_roots(g.has_edge(), 1 << 10, 2)])
    with pytest.raises(b200bfs.B200BfsError) as ex:
        engine.batch_select(2)
    assert ex.value.code == 1


@pytest.mark.parametrize("scale,flags", [(16, 0), (20, 0), (16, 3), (20, 3)])
def test_batch_root_levels_match_single_root(engine, scale, flags):
    """b200bfs_batch_root_levels gives, for every root of a batch, the
    AUTO_LEVEL slot b200bfs_run leaves for that root alone, so the re-pick
    test of find_roots_in_large_graph (main.cc:334-359: pick again while a
    root reaches <= 3 levels) can run as one batch.  Plain, and CoreBFS with
    group reordering (roots climbing into the core)."""
    engine.generate_graph(scale, 16, flags=flags)
    engine.prepare(16)
    for seed in range(4):
        roots = engine.find_roots(64, seed, 0)
        engine.run_batch(roots, 16, 0.0)
        lv = engine.batch_root_levels()
        single = np.array([engine.run(int(r), 16)[8] for r in roots])
        assert np.array_equal(lv, single), (seed, lv, single)
        assert (lv <= 3).any() == (single <= 3).any()
    engine.end()
