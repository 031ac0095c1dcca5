"""SCALE 28, the headline graph, against the CPU oracle.

The oracle cannot build a SCALE 28 graph in this host's memory (its int64
CSR needs about 200 GB), so it searches the engine's plain CSR copied to host
memory (34 GB of int32 columns): orc_bfs_csr32 restates BfsBase::run_bfs_core
(bfs.hpp:3238-3609) over that CSR.  For two roots from find_roots the
plain engine's levels and auto_tuning_data slots must equal the oracle's
with the same α/β, and the headline configuration -- -A tuned α/β, CoreBFS
(-C) and group reordering, a separately built graph -- must give the same
levels again, with every parent array passing the device validator with
pf_nedge[28] (mpi/utils.hpp:3687-3733) traversed edges.  The input edges the
device validator counts come from the device generator, which is pinned bit
for bit to the reference's generator (tests/test_golden.py,
test_generator_bit_exact_scale28_sample)."""
import ctypes

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

SCALE = 28
NROOTS = 2


def oracle_search(row_ptr, col, mdeg, inv, pred_size, row, alpha=10.0, beta=14.0):
    L = O.lib()
    L.orc_bfs_csr32.argtypes = [ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
                                ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                ctypes.c_int64, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(O.BfsStats)]
    pred = np.empty(pred_size, dtype=np.int64)
    at = np.full(9, -1, dtype=np.int64)
    st = O.BfsStats()
    L.orc_bfs_csr32(row_ptr.shape[0] - 1, O._ptr(row_ptr), O._ptr(col), O._ptr(mdeg),
                    O._ptr(inv), pred_size, int(row), 16, alpha, beta, O._ptr(pred), O._ptr(at),
                    ctypes.byref(st))
    return pred, at


def test_scale28_levels_match_oracle(built):
    import b200bfs

    e = b200bfs.Engine(0)
    e.generate_graph(SCALE, 16)
    info = e.info()
    e.prepare(16)
    roots = [int(r) for r in e.find_roots(NROOTS)]
    engine_levels, engine_at = {}, {}
    for r in roots:
        engine_at[r] = e.run(r, 16)
        engine_levels[r] = e.get_levels()
        assert e.validate(r) == (0, O.PF_NEDGE[SCALE]), r
    row_ptr, col, inv, mdeg = e.get_csr()
    e.close()
    rank = np.full(1 << SCALE, -1, np.int64)
    rank[inv] = np.arange(inv.size, dtype=np.int64)
    oracle_levels = {}
    for r in roots:
        pred, at = oracle_search(row_ptr, col, mdeg, inv, info.pred_size, rank[r])
        assert np.array_equal(at, engine_at[r]), (r, at, engine_at[r])
        oracle_levels[r] = O.pred_levels(pred)
        assert np.array_equal(engine_levels[r], oracle_levels[r]), r
    del row_ptr, col, inv, mdeg, rank

    # the headline configuration on its own graph: -A, -C, group reordering
    e = b200bfs.Engine(0)
    e.generate_graph(SCALE, 16, flags=b200bfs.BUILD_COREBFS | b200bfs.BUILD_GROUP_REORDER)
    e.prepare(16)
    tune_roots = [int(x) for x in e.find_roots(8)]
    alpha, beta, _ = e.auto_tune(tune_roots, np.full(8, float(O.PF_NEDGE[SCALE])))
    for r in roots:
        e.run(r, 16, alpha, beta)
        assert np.array_equal(e.get_levels(), oracle_levels[r]), r
        assert e.validate(r) == (0, O.PF_NEDGE[SCALE]), r
    e.close()
