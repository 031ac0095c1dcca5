"""The C-ABI library loads and exports every symbol include/b200bfs.h
declares (no GPU needed; no compute calls)."""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names |= set(re.findall(r"\b(b200bfs_[a-z0-9_]+)\s*\(", src))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    for n in ("b200bfs_create", "b200bfs_run", "b200bfs_get_pred", "b200bfs_prepare",
              "b200bfs_end", "b200bfs_has_edge", "b200bfs_build_from_edges"):
        assert n in names


def test_library_exports_all_declared(built):
    import ctypes
    import b200bfs

    L = b200bfs.load_library()
    for n in declared_symbols():
        assert hasattr(L, n), n
    assert set(b200bfs.SYMBOLS) <= declared_symbols()


def test_null_handle_is_rejected(built):
    import ctypes
    import b200bfs

    L = b200bfs.load_library()
    assert L.b200bfs_run(None, 0, 16, 10.0, 14.0, None) == 1
    assert L.b200bfs_last_error(None) == b"null handle"
    assert L.b200bfs_create(None, None) == 1


def test_no_cpu_fallback_without_device(built):
    """Without a CUDA device the engine refuses to start instead of running
    a CPU path."""
    import torch
    import b200bfs

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(b200bfs.B200BfsError):
        b200bfs.Engine()


def test_server_rejects_null_and_needs_a_device(built):
    import ctypes
    import torch
    import b200bfs

    L = b200bfs.load_library()
    assert L.b200bfs_server_submit(None, 0, 0, None) == 1
    assert L.b200bfs_server_stop(None) == 1
    assert L.b200bfs_server_last_error(None) == b"null server"
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(b200bfs.B200BfsError) as ex:
        b200bfs.Server(0)
    assert ex.value.code == 2
