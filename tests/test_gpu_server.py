"""The BFS server (b200bfs_server_*): continuous batching over resident graphs.

Each request's levels must be those of a single-source search from its root
(the oracle's queue BFS), and identical whether the request was served alone
or in a mix of concurrent requests over several graphs.
"""
import threading
import time

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

GRAPHS = [(12, 16), (14, 16), (14, 8)]


@pytest.fixture(scope="module")
def oracle_graphs(built):
    out = {}
    for scale, ef in GRAPHS:
        g = O.Graph(O.generate_edges(scale, edgefactor=ef))
        out[(scale, ef)] = g
    return out


def _roots(g, scale, n, seed):
    return [int(r) for r in O.find_roots(g.has_edge(), 1 << scale, n, seed)]


def test_alone_and_in_mix_are_identical(built, oracle_graphs):
    import b200bfs

    srv = b200bfs.Server(0, keep_results=True, slots_per_graph=2)
    try:
        gids = [srv.add_graph(s, ef) for s, ef in GRAPHS]
        psize = [srv.graph_info(g).pred_size for g in gids]
        nv = [1 << s for s, _ in GRAPHS]
        probe = (0, _roots(oracle_graphs[GRAPHS[0]], GRAPHS[0][0], 1, 0)[0])
        rid = srv.submit(gids[probe[0]], probe[1])
        info = srv.wait(rid)
        assert info.state == b200bfs.REQ_DONE and info.batch_size == 1
        alone = srv.levels(rid, psize[probe[0]])
        srv.release(rid)
        g0 = oracle_graphs[GRAPHS[0]]
        assert np.array_equal(alone[: nv[0]], g0.levels(probe[1]))

        # the mix: three graphs, two submitting threads, the probe request
        # repeated inside it
        rng = np.random.default_rng(5)
        work = []
        for i, (s, ef) in enumerate(GRAPHS):
            for r in _roots(oracle_graphs[(s, ef)], s, 48, 1 + i):
                work.append((i, r))
        work += [probe] * 6
        order = rng.permutation(len(work))
        work = [work[i] for i in order]
        ids = [None] * len(work)

        def submit(part):
            for j in part:
                ids[j] = srv.submit(gids[work[j][0]], work[j][1])

        threads = [threading.Thread(target=submit, args=(range(k, len(work), 2),))
                   for k in range(2)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        # With keep_results a slot is reused only after every request it
        # served is released, so results are consumed as they finish (in any
        # order), as a client of the server must.
        batch_sizes = []
        outstanding = dict(enumerate(ids))
        deadline = time.time() + 120
        while outstanding:
            assert time.time() < deadline, f"{len(outstanding)} requests unfinished"
            progressed = False
            for j, rid in list(outstanding.items()):
                info = srv.poll(rid)
                if info.state < b200bfs.REQ_DONE:
                    continue
                assert info.state == b200bfs.REQ_DONE
                gi, r = work[j]
                batch_sizes.append(info.batch_size)
                lv = srv.levels(rid, psize[gi])
                ref = oracle_graphs[GRAPHS[gi]].levels(r)
                assert np.array_equal(lv[: nv[gi]], ref), (gi, r)
                assert info.depth == int(ref.max())
                if (gi, r) == probe:
                    assert np.array_equal(lv, alone)
                srv.release(rid)
                del outstanding[j]
                progressed = True
            if not progressed:
                time.sleep(0.002)
        assert max(batch_sizes) > 1  # requests were packed into batches
        st = srv.stats()
        assert st.completed == len(work) + 1 and st.failed == 0
        assert st.p99_ms >= st.p50_ms > 0 and st.bfs_per_s > 0
        assert st.graphs == 3 and st.slots == 6
    finally:
        srv.stop()


def test_results_not_kept_and_stats(built, oracle_graphs):
    import b200bfs

    srv = b200bfs.Server(0, keep_results=False, max_batch=16, slots_per_graph=1)
    try:
        gid = srv.add_graph(12, 16)
        roots = _roots(oracle_graphs[(12, 16)], 12, 40, 3)
        ids = [srv.submit(gid, r) for r in roots]
        for rid, r in zip(ids, roots):
            info = srv.wait(rid)
            assert info.state == b200bfs.REQ_DONE
            assert info.batch_size <= 16
            assert info.depth == int(oracle_graphs[(12, 16)].levels(r).max())
        with pytest.raises(b200bfs.B200BfsError) as ex:
            srv.levels(ids[0], srv.graph_info(gid).pred_size)
        assert ex.value.code == 4
        for rid in ids:
            srv.release(rid)
        st = srv.stats()
        assert st.completed == 40 and st.batches >= 3
        srv.reset_stats()
        assert srv.stats().completed == 0
    finally:
        srv.stop()


def test_hbm_budget_admission(built):
    import b200bfs

    srv = b200bfs.Server(0, hbm_budget_bytes=64 << 20, slots_per_graph=4)
    try:
        gid = srv.add_graph(12, 16)
        st = srv.stats()
        assert 1 <= st.slots <= 4 and st.device_bytes <= 64 << 20
        with pytest.raises(b200bfs.B200BfsError) as ex:
            srv.add_graph(20, 16)
        assert ex.value.code == 3  # OOM: does not fit the budget
        assert srv.stats().graphs == 1
        rid = srv.submit(gid, 1)
        assert srv.wait(rid).state == b200bfs.REQ_DONE
        srv.release(rid)
    finally:
        srv.stop()


def test_server_errors_and_stop(built):
    import b200bfs

    srv = b200bfs.Server(0, slots_per_graph=1)
    gid = srv.add_graph(10, 16)
    with pytest.raises(b200bfs.B200BfsError) as ex:
        srv.submit(gid + 1, 0)
    assert ex.value.code == 7
    with pytest.raises(b200bfs.B200BfsError) as ex:
        srv.submit(gid, 1 << 20)
    assert ex.value.code == 1
    with pytest.raises(b200bfs.B200BfsError) as ex:
        srv.poll(12345)
    assert ex.value.code == 7
    for r in range(200):  # stop with work queued: queued requests are cancelled
        srv.submit(gid, r % 1024)
    srv.stop()
