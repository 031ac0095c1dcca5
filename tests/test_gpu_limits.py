"""Limits the engine reports as errors instead of wrong results.

A path graph of 70,000 vertices searched from one end needs 69,999 levels,
more than the 0xFFFE the pred encoding holds (level << 48 | parent, 16-bit
level field, validate.hpp:982-992): the search must fail with
B200BFS_ERR_OVERFLOW, and the engine must still serve a search from the
path's middle (35,000 levels) afterwards."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = 70000


def path_edges(n):
    v = np.arange(n - 1, dtype=np.int64)
    return np.stack([v, v + 1], axis=1)


def test_level_overflow_is_an_error(built):
    import b200bfs

    e = b200bfs.Engine(0)
    e.build_from_edges(path_edges(N))
    e.prepare(16)
    with pytest.raises(b200bfs.B200BfsError) as ei:
        e.run(0, 16)
    assert ei.value.code == 6  # B200BFS_ERR_OVERFLOW
    mid = N // 2
    at = e.run(mid, 16)
    lv = e.get_levels()[:N]
    assert np.array_equal(lv, np.abs(np.arange(N) - mid))
    assert at[8] == mid + 1  # AUTO_LEVEL: one level past the deepest vertex
    e.close()
