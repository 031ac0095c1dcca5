"""b200bfs_bfs_noalloc: the search entry point for callers that may not
allocate device memory (programs whose caching allocator owns the device,
hosts with a fixed memory budget).  Its scratch lives in a fixed device array
inside the library, so the test hands it only device inputs and outputs and
checks its results against the engine's own b200bfs_run on the same graph,
on two calls in a row.  It synchronises its stream once per level, so a
stream being captured into a CUDA graph is refused before anything is
enqueued, and the capture stays usable.  This file sorts last so that a run
stopping at the first failure has already run every other test."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _check_tree(pred, lv, row_ptr, col, root):
    """Every reached non-root row has a neighbour one level up as parent."""
    parents = (pred << 16) >> 16
    reached = np.nonzero((pred != -1) & (np.arange(pred.size) != root))[0]
    for v in reached[:: max(1, reached.size // 2000)]:
        p = parents[v]
        assert lv[p] == lv[v] - 1
        assert p in col[row_ptr[v]:row_ptr[v + 1]]


def test_noalloc_matches_engine(built):
    import torch
    import b200bfs

    eng = b200bfs.Engine(0)
    eng.generate_graph(16, 16)
    eng.prepare(16)
    row_ptr, col, inv, _ = eng.get_csr()
    nrows = row_ptr.size - 1
    d_row = torch.from_numpy(row_ptr).cuda()
    d_col = torch.from_numpy(col).cuda()
    d_pred = torch.empty(nrows, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    rank = np.full(1 << 16, -1, np.int64)
    rank[inv] = np.arange(nrows)
    roots = eng.find_roots(2)
    for call, root in enumerate(roots):  # two calls in a row
        nl = b200bfs.bfs_noalloc(d_row.data_ptr(), d_col.data_ptr(), nrows, int(rank[root]),
                                 d_pred.data_ptr())
        pred = d_pred.cpu().numpy()
        lv = O.pred_levels(pred)
        at = eng.run(int(root), 16)
        ref = eng.get_levels()
        assert np.array_equal(lv, ref[inv]), call
        assert nl == at[8]
        _check_tree(pred, lv, row_ptr, col, int(rank[root]))
    eng.close()


def test_noalloc_rejects_too_large(built):
    import torch
    import b200bfs

    dummy = torch.zeros(4, dtype=torch.int64, device="cuda")
    with pytest.raises(b200bfs.B200BfsError) as ei:
        b200bfs.bfs_noalloc(dummy.data_ptr(), dummy.data_ptr(), b200bfs.NOALLOC_MAX_ROWS + 1, 0,
                            dummy.data_ptr())
    assert ei.value.code == 1


def test_noalloc_refuses_capturing_stream(built):
    import torch
    import b200bfs

    row_ptr = torch.tensor([0, 1, 2], dtype=torch.int64, device="cuda")
    col = torch.tensor([1, 0], dtype=torch.int32, device="cuda")
    pred = torch.empty(2, dtype=torch.int64, device="cuda")
    x = torch.zeros(4, device="cuda")
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    codes = []
    with torch.cuda.graph(g, stream=s):
        x.add_(1)
        try:
            b200bfs.bfs_noalloc(row_ptr.data_ptr(), col.data_ptr(), 2, 0, pred.data_ptr(),
                                stream=s.cuda_stream)
        except b200bfs.B200BfsError as e:
            codes.append(e.code)
        x.add_(1)
    assert codes == [1]  # B200BFS_ERR_INVALID, nothing enqueued
    g.replay()
    torch.cuda.synchronize()
    assert x.tolist() == [2.0] * 4  # the capture was not broken
    # outside a capture the same call searches
    assert b200bfs.bfs_noalloc(row_ptr.data_ptr(), col.data_ptr(), 2, 0, pred.data_ptr()) == 2
    assert pred.cpu().tolist() == [0, (1 << 48) | 0]


def test_noalloc_level_overflow_is_an_error(built):
    import torch
    import b200bfs

    n = 70000  # a path searched from one end: 69,999 levels > 0xFFFE
    v = np.arange(n, dtype=np.int64)
    row_ptr = np.concatenate([[0], np.cumsum(np.where((v == 0) | (v == n - 1), 1, 2))])
    col = np.empty(row_ptr[-1], np.int32)
    for_left = v[1:]
    col[row_ptr[for_left]] = (for_left - 1).astype(np.int32)  # first neighbour: v - 1
    right = v[:-1]
    col[row_ptr[right + 1] - 1] = (right + 1).astype(np.int32)  # last neighbour: v + 1
    d_row = torch.from_numpy(row_ptr).cuda()
    d_col = torch.from_numpy(col).cuda()
    d_pred = torch.empty(n, dtype=torch.int64, device="cuda")
    with pytest.raises(b200bfs.B200BfsError) as ei:
        b200bfs.bfs_noalloc(d_row.data_ptr(), d_col.data_ptr(), n, 0, d_pred.data_ptr())
    assert ei.value.code == 6  # B200BFS_ERR_OVERFLOW
    # from the middle the same call searches the whole path
    assert b200bfs.bfs_noalloc(d_row.data_ptr(), d_col.data_ptr(), n, n // 2,
                               d_pred.data_ptr()) == n // 2 + 1
