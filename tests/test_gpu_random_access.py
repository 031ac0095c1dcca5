"""b200bfs_random_access_rate: the random-access ceiling bench.py reports for
the top-down kernels.  It must return a positive rate for both access kinds
and refuse bad arguments before touching the device."""
import math

import pytest

import b200bfs


def test_random_access_rate_rejects_bad_arguments():
    L = b200bfs.load_library()
    import ctypes
    out = ctypes.c_double(0)
    assert L.b200bfs_random_access_rate(None, 20, 0, None, ctypes.byref(out)) == 1
    assert L.b200bfs_random_access_rate(ctypes.c_void_p(256), 9, 0, None, ctypes.byref(out)) == 1
    assert L.b200bfs_random_access_rate(ctypes.c_void_p(256), 31, 0, None, ctypes.byref(out)) == 1
    assert L.b200bfs_random_access_rate(ctypes.c_void_p(256), 20, 2, None, ctypes.byref(out)) == 1
    assert L.b200bfs_random_access_rate(ctypes.c_void_p(258), 20, 0, None, ctypes.byref(out)) == 1
    assert L.b200bfs_random_access_rate(ctypes.c_void_p(256), 20, 0, None, None) == 1


@pytest.mark.gpu
def test_random_access_rate_positive():
    import torch
    buf = torch.zeros(1 << 22, dtype=torch.int32, device="cuda")
    loads = b200bfs.random_access_rate(buf.data_ptr(), 22, 0)
    ors = b200bfs.random_access_rate(buf.data_ptr(), 22, 1)
    assert math.isfinite(loads) and loads > 1e9
    assert math.isfinite(ors) and ors > 1e9
    # the ORs set bits only inside the buffer
    assert int(torch.count_nonzero(buf)) > 0
