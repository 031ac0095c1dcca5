"""Host-side binding of the B200 BFS engine (libb200bfs.so, include/b200bfs.h).

`BfsOnB200` mirrors the member surface of the reference's `class BfsBase`
(mpi/bfs.hpp:48-172), which the benchmark driver reaches as `BfsOnCPU`
(mpi/bfs_cpu.hpp:13): construct / prepare_bfs / run_bfs / get_pred / end_bfs /
has_edge, plus a `graph_` facade with pred_size(), has_edge(v) and
log_orig_global_verts_.  Errors become `B200BfsError` (the reference throws
`const char*` / std::runtime_error).

There is no CPU fallback: importing this module on a machine without the
built library or without a CUDA device raises.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libb200bfs.so")

OK = 0
ERR_NAMES = {1: "INVALID", 2: "CUDA", 3: "OOM", 4: "STATE", 5: "TIMEOUT", 6: "OVERFLOW",
             7: "NOT_FOUND"}

BUILD_COREBFS = 1 << 0
BUILD_GROUP_REORDER = 1 << 1
BUILD_INPUT_SYMMETRIC = 1 << 2

USERSEED1, USERSEED2 = 2, 3  # mpi/parameters.h:204-205
DEFAULT_ALPHA, DEFAULT_BETA = 10.0, 14.0  # mpi/parameters.h:97-98
AUTO_NUM = 9
AUTO_NOT_DEFINED = -1

# Exported symbols (must match include/b200bfs.h).
SYMBOLS = [
    "b200bfs_create", "b200bfs_destroy", "b200bfs_last_error", "b200bfs_print_information",
    "b200bfs_build_from_edges", "b200bfs_build_from_packed", "b200bfs_generate_graph",
    "b200bfs_generate_edges", "b200bfs_graph_info_get", "b200bfs_get_csr", "b200bfs_has_edge",
    "b200bfs_has_edge_all", "b200bfs_find_roots", "b200bfs_prepare", "b200bfs_run", "b200bfs_get_pred",
    "b200bfs_get_levels", "b200bfs_get_run_stats", "b200bfs_get_stream", "b200bfs_end",
    "b200bfs_auto_tune", "b200bfs_set_option", "b200bfs_get_level_stats",
    "b200bfs_validate", "b200bfs_validate_pred", "b200bfs_bfs_noalloc", "b200bfs_run_batch", "b200bfs_batch_select", "b200bfs_batch_root_levels",
    "b200bfs_server_start", "b200bfs_server_add_graph", "b200bfs_server_graph_info",
    "b200bfs_server_find_roots", "b200bfs_tune_engine",
    "b200bfs_server_submit", "b200bfs_server_poll", "b200bfs_server_wait",
    "b200bfs_server_get_levels", "b200bfs_server_release", "b200bfs_server_get_stats",
    "b200bfs_server_reset_stats", "b200bfs_server_last_error", "b200bfs_server_stop",
    "b200bfs_random_access_rate",
]
REQ_QUEUED, REQ_RUNNING, REQ_DONE, REQ_FAILED, REQ_CANCELLED = range(5)
BATCH_MAX = 64  # B200BFS_BATCH_MAX
BATCH_ALPHA = 30.0  # batch default of the top-down -> bottom-up threshold


class B200BfsError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"b200bfs error {code} ({ERR_NAMES.get(code, '?')}): {msg}")
        self.code = code


class Config(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("reserved", ctypes.c_int),
                ("hbm_budget_bytes", ctypes.c_uint64)]


class GraphInfo(ctypes.Structure):
    _fields_ = [("scale", ctypes.c_int32), ("reorder_bits", ctypes.c_int32),
                ("pred_size", ctypes.c_int64), ("num_global_edges", ctypes.c_int64),
                ("num_global_verts", ctypes.c_int64), ("num_rows", ctypes.c_int64),
                ("num_input_edges", ctypes.c_int64), ("device_bytes", ctypes.c_int64),
                ("corebfs", ctypes.c_int32), ("prune_rounds", ctypes.c_int32),
                ("core_vertices", ctypes.c_int64), ("tree_vertices", ctypes.c_int64)]


class RunStats(ctypes.Structure):
    _fields_ = [("levels", ctypes.c_int32), ("num_td_levels", ctypes.c_int32),
                ("num_bu_levels", ctypes.c_int32), ("kernel_launches", ctypes.c_int32),
                ("bu_level_mask", ctypes.c_uint64), ("visited", ctypes.c_int64),
                ("edges_scanned_td", ctypes.c_int64), ("edges_scanned_bu", ctypes.c_int64),
                ("algorithmic_bytes", ctypes.c_int64), ("td_bytes", ctypes.c_int64),
                ("bu_bytes", ctypes.c_int64), ("device_ms", ctypes.c_double),
                ("td_ms", ctypes.c_double), ("bu_ms", ctypes.c_double),
                ("pred_bytes", ctypes.c_int64), ("pred_ms", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class LevelStats(ctypes.Structure):
    _fields_ = [("level", ctypes.c_int32), ("bottom_up", ctypes.c_int32),
                ("input", ctypes.c_int64), ("discovered", ctypes.c_int64),
                ("scanned", ctypes.c_int64), ("algorithmic_bytes", ctypes.c_int64),
                ("ms", ctypes.c_double)]


class BatchStats(ctypes.Structure):
    _fields_ = [("num_roots", ctypes.c_int32), ("levels", ctypes.c_int32),
                ("num_td_levels", ctypes.c_int32), ("num_bu_levels", ctypes.c_int32),
                ("kernel_launches", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("edges_scanned_td", ctypes.c_int64), ("edges_scanned_bu", ctypes.c_int64),
                ("algorithmic_bytes", ctypes.c_int64), ("bu_bytes", ctypes.c_int64),
                ("ms", ctypes.c_double), ("bu_ms", ctypes.c_double),
                ("td_ms", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


TUNE_FORMS, TUNE_BATCH_ALPHA, TUNE_SWITCH = 1, 2, 4


class TuneReport(ctypes.Structure):
    _fields_ = [("bu_kernel", ctypes.c_int32), ("td_kernel", ctypes.c_int32),
                ("batch_alpha", ctypes.c_double), ("single_ms", ctypes.c_double),
                ("batch_ms", ctypes.c_double), ("searches", ctypes.c_int32),
                ("batches", ctypes.c_int32), ("alpha", ctypes.c_double),
                ("beta", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServerConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("max_batch", ctypes.c_int),
                ("slots_per_graph", ctypes.c_int), ("keep_results", ctypes.c_int),
                ("hbm_budget_bytes", ctypes.c_uint64), ("alpha", ctypes.c_double),
                ("beta", ctypes.c_double)]


class RequestInfo(ctypes.Structure):
    _fields_ = [("state", ctypes.c_int32), ("graph_id", ctypes.c_int32),
                ("root", ctypes.c_int64), ("depth", ctypes.c_int32),
                ("batch_size", ctypes.c_int32), ("latency_ms", ctypes.c_double),
                ("queue_ms", ctypes.c_double)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_int64), ("completed", ctypes.c_int64),
                ("failed", ctypes.c_int64), ("batches", ctypes.c_int64),
                ("mean_batch_size", ctypes.c_double), ("p50_ms", ctypes.c_double),
                ("p99_ms", ctypes.c_double), ("max_ms", ctypes.c_double),
                ("bfs_per_s", ctypes.c_double), ("device_bytes", ctypes.c_uint64),
                ("graphs", ctypes.c_int32), ("slots", ctypes.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None


def load_library(path=LIB_PATH):
    """Loads libb200bfs.so and declares the C ABI; raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise B200BfsError(2, f"{path} is not built; run __graft_entry__.build()")
    L = ctypes.CDLL(path)
    P, i64, i32, u64, dbl, vp = (ctypes.POINTER, ctypes.c_int64, ctypes.c_int, ctypes.c_uint64,
                                 ctypes.c_double, ctypes.c_void_p)
    H = ctypes.c_void_p
    L.b200bfs_create.argtypes = [P(Config), P(H)]
    L.b200bfs_destroy.argtypes = [H]
    L.b200bfs_last_error.argtypes = [H]
    L.b200bfs_last_error.restype = ctypes.c_char_p
    L.b200bfs_print_information.argtypes = [H, ctypes.c_char_p, ctypes.c_size_t]
    L.b200bfs_build_from_edges.argtypes = [H, vp, i64, i32, i32]
    L.b200bfs_build_from_packed.argtypes = [H, vp, i64, i32, i32]
    L.b200bfs_generate_graph.argtypes = [H, i32, i32, u64, u64, i32]
    L.b200bfs_generate_edges.argtypes = [H, i32, u64, u64, i64, i64, vp]
    L.b200bfs_graph_info_get.argtypes = [H, P(GraphInfo)]
    L.b200bfs_get_csr.argtypes = [H, vp, vp, vp, vp]
    L.b200bfs_has_edge.argtypes = [H, i64, P(ctypes.c_int)]
    L.b200bfs_has_edge_all.argtypes = [H, vp]
    L.b200bfs_find_roots.argtypes = [H, i32, i32, i32, vp]
    L.b200bfs_prepare.argtypes = [H, i32, dbl, dbl]
    L.b200bfs_run.argtypes = [H, i64, i32, dbl, dbl, vp]
    L.b200bfs_auto_tune.argtypes = [H, vp, i32, vp, i32, P(dbl), P(dbl), P(dbl)]
    L.b200bfs_get_pred.argtypes = [H, vp]
    L.b200bfs_get_levels.argtypes = [H, vp]
    L.b200bfs_get_run_stats.argtypes = [H, P(RunStats)]
    L.b200bfs_get_stream.argtypes = [H, P(ctypes.c_void_p)]
    L.b200bfs_set_option.argtypes = [H, ctypes.c_char_p, i64]
    L.b200bfs_get_level_stats.argtypes = [H, vp, i32, P(ctypes.c_int)]
    L.b200bfs_end.argtypes = [H]
    L.b200bfs_validate.argtypes = [H, i64, P(ctypes.c_int64), P(ctypes.c_int64)]
    L.b200bfs_validate_pred.argtypes = [H, i64, ctypes.c_void_p, ctypes.c_int,
                                        P(ctypes.c_int64), P(ctypes.c_int64)]
    L.b200bfs_bfs_noalloc.argtypes = [vp, vp, i64, i64, vp, vp, P(ctypes.c_int32)]
    L.b200bfs_random_access_rate.argtypes = [vp, i32, i32, vp, P(dbl)]
    L.b200bfs_run_batch.argtypes = [H, vp, i32, i32, dbl, dbl, P(BatchStats)]
    L.b200bfs_tune_engine.argtypes = [H, vp, i32, i32, dbl, dbl, i32, P(TuneReport)]
    L.b200bfs_batch_select.argtypes = [H, i32]
    L.b200bfs_batch_root_levels.argtypes = [H, ctypes.c_void_p]
    S = ctypes.c_void_p
    L.b200bfs_server_start.argtypes = [P(ServerConfig), P(S)]
    L.b200bfs_server_add_graph.argtypes = [S, i32, i32, u64, u64, i32, P(ctypes.c_int)]
    L.b200bfs_server_graph_info.argtypes = [S, i32, P(GraphInfo)]
    L.b200bfs_server_find_roots.argtypes = [S, i32, i32, i32, i32, vp]
    L.b200bfs_server_submit.argtypes = [S, i32, i64, P(ctypes.c_int64)]
    L.b200bfs_server_poll.argtypes = [S, i64, P(RequestInfo)]
    L.b200bfs_server_wait.argtypes = [S, i64, dbl, P(RequestInfo)]
    L.b200bfs_server_get_levels.argtypes = [S, i64, vp]
    L.b200bfs_server_release.argtypes = [S, i64]
    L.b200bfs_server_get_stats.argtypes = [S, P(ServerStats)]
    L.b200bfs_server_reset_stats.argtypes = [S]
    L.b200bfs_server_last_error.argtypes = [S]
    L.b200bfs_server_last_error.restype = ctypes.c_char_p
    L.b200bfs_server_stop.argtypes = [S]
    _lib = L
    return L


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class Engine:
    """Thin owner of one b200bfs handle."""

    def __init__(self, device=0, hbm_budget_bytes=0):
        self.L = load_library()
        cfg = Config(device, 0, hbm_budget_bytes)
        h = ctypes.c_void_p()
        rc = self.L.b200bfs_create(ctypes.byref(cfg), ctypes.byref(h))
        if rc != OK:
            raise B200BfsError(rc, "b200bfs_create failed (no CUDA device?)")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.b200bfs_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, rc):
        if rc != OK:
            raise B200BfsError(rc, self.L.b200bfs_last_error(self.h).decode())

    def info(self):
        gi = GraphInfo()
        self.check(self.L.b200bfs_graph_info_get(self.h, ctypes.byref(gi)))
        return gi

    def print_information(self):
        buf = ctypes.create_string_buffer(512)
        self.check(self.L.b200bfs_print_information(self.h, buf, 512))
        return buf.value.decode()

    def generate_graph(self, scale, edgefactor=16, seed1=USERSEED1, seed2=USERSEED2, flags=0):
        self.check(self.L.b200bfs_generate_graph(self.h, scale, edgefactor, seed1, seed2, flags))

    def generate_edges(self, scale, start, end, seed1=USERSEED1, seed2=USERSEED2):
        out = np.empty((end - start, 2), dtype=np.int64)
        self.check(self.L.b200bfs_generate_edges(self.h, scale, seed1, seed2, start, end,
                                                 _ptr(out)))
        return out

    def build_from_edges(self, edges, scale=0, flags=0):
        edges = np.ascontiguousarray(edges, dtype=np.int64)
        self.check(self.L.b200bfs_build_from_edges(self.h, _ptr(edges), edges.shape[0], scale,
                                                   flags))

    def build_from_packed(self, packed, scale=0, flags=0):
        packed = np.ascontiguousarray(packed, dtype=np.uint32)
        self.check(self.L.b200bfs_build_from_packed(self.h, _ptr(packed), packed.shape[0],
                                                    scale, flags))

    def get_csr(self):
        """(row_ptr, col, inv, mdeg) of the searched CSR, in host memory."""
        gi = self.info()
        R, E = gi.num_rows, gi.num_global_edges
        row_ptr = np.empty(R + 1, np.int64)
        col = np.empty(E, np.int32)
        inv = np.empty(R, np.int32)
        mdeg = np.empty(R, np.int32)
        self.check(self.L.b200bfs_get_csr(self.h, _ptr(row_ptr), _ptr(col), _ptr(inv),
                                          _ptr(mdeg)))
        return row_ptr, col, inv, mdeg

    def has_edge(self, v):
        out = ctypes.c_int()
        self.check(self.L.b200bfs_has_edge(self.h, v, ctypes.byref(out)))
        return bool(out.value)

    def has_edge_all(self):
        out = np.empty(self.info().pred_size, dtype=np.uint8)
        self.check(self.L.b200bfs_has_edge_all(self.h, _ptr(out)))
        return out

    def find_roots(self, num_roots, r1=0, r2=0):
        out = np.empty(num_roots, dtype=np.int64)
        self.check(self.L.b200bfs_find_roots(self.h, num_roots, r1, r2, _ptr(out)))
        return out

    def prepare(self, edgefactor=16, alpha=DEFAULT_ALPHA, beta=DEFAULT_BETA):
        self.check(self.L.b200bfs_prepare(self.h, edgefactor, alpha, beta))

    def run(self, root, edgefactor=16, alpha=DEFAULT_ALPHA, beta=DEFAULT_BETA, at=None):
        if at is None:
            at = np.full(AUTO_NUM, AUTO_NOT_DEFINED, dtype=np.int64)
        self.check(self.L.b200bfs_run(self.h, int(root), edgefactor, alpha, beta, _ptr(at)))
        return at

    def auto_tune(self, roots, nedge, edgefactor=16, alpha=DEFAULT_ALPHA, beta=DEFAULT_BETA):
        """The -A tuner (main.cc:361-391); returns (alpha, beta, harmonic TEPS)."""
        roots = np.ascontiguousarray(roots, dtype=np.int64)
        nedge = np.ascontiguousarray(nedge, dtype=np.float64)
        a, b, t = ctypes.c_double(alpha), ctypes.c_double(beta), ctypes.c_double(0)
        self.check(self.L.b200bfs_auto_tune(self.h, _ptr(roots), roots.size, _ptr(nedge),
                                            edgefactor, ctypes.byref(a), ctypes.byref(b),
                                            ctypes.byref(t)))
        return a.value, b.value, t.value

    def get_pred(self, out=None):
        if out is None:
            out = np.empty(self.info().pred_size, dtype=np.int64)
        self.check(self.L.b200bfs_get_pred(self.h, _ptr(out)))
        return out

    def get_levels(self):
        out = np.empty(self.info().pred_size, dtype=np.int32)
        self.check(self.L.b200bfs_get_levels(self.h, _ptr(out)))
        return out

    def run_stats(self):
        rs = RunStats()
        self.check(self.L.b200bfs_get_run_stats(self.h, ctypes.byref(rs)))
        return rs

    def level_stats(self):
        """Per-level records of the last search, as dicts."""
        n = ctypes.c_int(0)
        self.check(self.L.b200bfs_get_level_stats(self.h, None, 0, ctypes.byref(n)))
        arr = (LevelStats * max(n.value, 1))()
        self.check(self.L.b200bfs_get_level_stats(self.h, ctypes.cast(arr, ctypes.c_void_p),
                                                  n.value, ctypes.byref(n)))
        return [{k: getattr(arr[i], k) for k, _ in LevelStats._fields_} for i in range(n.value)]

    def set_option(self, name, value):
        self.check(self.L.b200bfs_set_option(self.h, name.encode(), int(value)))

    def stream(self):
        """The engine's cudaStream_t as an integer handle."""
        out = ctypes.c_void_p()
        self.check(self.L.b200bfs_get_stream(self.h, ctypes.byref(out)))
        return out.value or 0

    def end(self):
        self.check(self.L.b200bfs_end(self.h))

    def run_batch(self, roots, edgefactor=16, alpha=BATCH_ALPHA, beta=DEFAULT_BETA):
        """One multi-source search from up to 64 roots; returns BatchStats."""
        r = np.ascontiguousarray(np.asarray(roots, dtype=np.int64))
        self._batch_k = len(r)
        bs = BatchStats()
        self.check(self.L.b200bfs_run_batch(self.h, _ptr(r), len(r), edgefactor, alpha, beta,
                                            ctypes.byref(bs)))
        return bs

    def tune_engine(self, roots, edgefactor=16, alpha=DEFAULT_ALPHA, beta=DEFAULT_BETA,
                    what=TUNE_FORMS | TUNE_BATCH_ALPHA):
        """Engine autotuner (b200bfs_tune_engine); returns the TuneReport."""
        r = np.ascontiguousarray(np.asarray(roots, dtype=np.int64))
        rep = TuneReport()
        self.check(self.L.b200bfs_tune_engine(self.h, _ptr(r), len(r), edgefactor, alpha, beta,
                                              what, ctypes.byref(rep)))
        return rep

    def batch_root_levels(self):
        """AUTO_LEVEL of each root of the last batch (its deepest level + 1),
        what b200bfs_run would report for that root alone."""
        out = np.zeros(BATCH_MAX, dtype=np.int64)
        self.check(self.L.b200bfs_batch_root_levels(self.h, _ptr(out)))
        return out[: getattr(self, "_batch_k", BATCH_MAX)]

    def batch_select(self, index):
        """Makes root `index` of the last batch the current result (pred,
        levels and validation then refer to it)."""
        self.check(self.L.b200bfs_batch_select(self.h, int(index)))

    def validate(self, root):
        err = ctypes.c_int64()
        cnt = ctypes.c_int64()
        self.check(self.L.b200bfs_validate(self.h, int(root), ctypes.byref(err),
                                           ctypes.byref(cnt)))
        return err.value, cnt.value

    def validate_pred(self, root, pred, corebfs=None):
        """Graph500 validation of a caller's pred (host array of pred_size
        int64 entries) on the device (validate_bfs_result, validate.hpp:1269);
        corebfs defaults to the graph's mode.  Returns (errors, edges)."""
        pred = np.ascontiguousarray(pred, dtype=np.int64)
        if pred.size != self.info().pred_size:
            raise ValueError("pred must have pred_size entries")
        if corebfs is None:
            corebfs = bool(self.info().corebfs)
        err = ctypes.c_int64()
        cnt = ctypes.c_int64()
        self.check(self.L.b200bfs_validate_pred(self.h, int(root), pred.ctypes.data,
                                                1 if corebfs else 0, ctypes.byref(err),
                                                ctypes.byref(cnt)))
        return err.value, cnt.value


NOALLOC_MAX_ROWS = 1 << 24  # B200BFS_NOALLOC_MAX_ROWS


def random_access_rate(words_dev, log2_words, kind, stream=0):
    """b200bfs_random_access_rate on a device buffer (int pointer) of
    2^log2_words uint32: random 4-byte loads (kind 0) or non-returning ORs
    (kind 1) per second on the current device."""
    L = load_library()
    out = ctypes.c_double(0)
    rc = L.b200bfs_random_access_rate(ctypes.c_void_p(words_dev), log2_words, kind,
                                      ctypes.c_void_p(stream), ctypes.byref(out))
    if rc:
        raise B200BfsError(rc, "b200bfs_random_access_rate failed")
    return out.value


def bfs_noalloc(row_ptr_dev, col_dev, nrows, root, pred_dev, stream=0):
    """b200bfs_bfs_noalloc on device pointers (ints); returns the number of
    levels.  Searches without allocating device memory (see include/b200bfs.h);
    raises B200BfsError on a non-zero status."""
    L = load_library()
    nl = ctypes.c_int32(0)
    rc = L.b200bfs_bfs_noalloc(ctypes.c_void_p(row_ptr_dev), ctypes.c_void_p(col_dev), nrows,
                               root, ctypes.c_void_p(pred_dev), ctypes.c_void_p(stream),
                               ctypes.byref(nl))
    if rc != OK:
        raise B200BfsError(rc, "b200bfs_bfs_noalloc failed")
    return nl.value


class Server:
    """BFS server with continuous batching (b200bfs_server_*): graphs stay
    resident on the device and (graph, root) queries are answered as they
    arrive, packed into batched searches by per-slot worker threads."""

    def __init__(self, device=0, max_batch=64, slots_per_graph=2, keep_results=False,
                 hbm_budget_bytes=0, alpha=0.0, beta=0.0):
        self.L = load_library()
        cfg = ServerConfig(device, max_batch, slots_per_graph, int(bool(keep_results)),
                           hbm_budget_bytes, alpha, beta)
        self.s = ctypes.c_void_p()
        rc = self.L.b200bfs_server_start(ctypes.byref(cfg), ctypes.byref(self.s))
        if rc != OK:
            raise B200BfsError(rc, "b200bfs_server_start failed")

    def check(self, rc):
        if rc != OK:
            raise B200BfsError(rc, self.L.b200bfs_server_last_error(self.s).decode())

    def add_graph(self, scale, edgefactor=16, seed1=USERSEED1, seed2=USERSEED2, flags=0):
        gid = ctypes.c_int()
        self.check(self.L.b200bfs_server_add_graph(self.s, scale, edgefactor, seed1, seed2, flags,
                                                   ctypes.byref(gid)))
        return gid.value

    def graph_info(self, gid):
        gi = GraphInfo()
        self.check(self.L.b200bfs_server_graph_info(self.s, gid, ctypes.byref(gi)))
        return gi

    def find_roots(self, gid, num_roots, r1=0, r2=0):
        out = np.zeros(num_roots, dtype=np.int64)
        self.check(self.L.b200bfs_server_find_roots(self.s, gid, num_roots, r1, r2, _ptr(out)))
        return out

    def submit(self, gid, root):
        rid = ctypes.c_int64()
        self.check(self.L.b200bfs_server_submit(self.s, gid, int(root), ctypes.byref(rid)))
        return rid.value

    def poll(self, rid):
        info = RequestInfo()
        self.check(self.L.b200bfs_server_poll(self.s, rid, ctypes.byref(info)))
        return info

    def wait(self, rid, timeout=60.0):
        info = RequestInfo()
        self.check(self.L.b200bfs_server_wait(self.s, rid, timeout, ctypes.byref(info)))
        return info

    def levels(self, rid, pred_size):
        out = np.empty(pred_size, dtype=np.int32)
        self.check(self.L.b200bfs_server_get_levels(self.s, rid, _ptr(out)))
        return out

    def release(self, rid):
        self.check(self.L.b200bfs_server_release(self.s, rid))

    def stats(self):
        st = ServerStats()
        self.check(self.L.b200bfs_server_get_stats(self.s, ctypes.byref(st)))
        return st

    def reset_stats(self):
        self.check(self.L.b200bfs_server_reset_stats(self.s))

    def stop(self):
        if self.s:
            self.L.b200bfs_server_stop(self.s)
            self.s = ctypes.c_void_p()

    def __del__(self):
        try:
            self.stop()
        except Exception:
            pass


class _GraphFacade:
    """The part of Graph2DCSR the driver reads (graph_constructor.hpp:187-333)."""

    def __init__(self, bfs):
        self._bfs = bfs

    @property
    def log_orig_global_verts_(self):
        return self._bfs.engine.info().scale

    @property
    def reorder_bits_(self):
        return self._bfs.engine.info().reorder_bits

    @property
    def num_global_edges_(self):
        return self._bfs.engine.info().num_global_edges

    @property
    def num_global_verts_(self):
        return self._bfs.engine.info().num_global_verts

    def pred_size(self):
        return self._bfs.engine.info().pred_size

    def has_edge(self, v):
        return self._bfs.engine.has_edge(v)


class BfsOnB200:
    """Drop-in for BfsBase / BfsOnCPU (mpi/bfs.hpp:48-172, mpi/bfs_cpu.hpp:13)."""

    def __init__(self, device=0, hbm_budget_bytes=0):
        self.engine = Engine(device, hbm_budget_bytes)
        self.graph_ = _GraphFacade(self)
        self._corebfs = False

    @staticmethod
    def printInformation(validation_level=2, pre_exec=False, real_benchmark=False):
        return Engine().print_information()

    def construct(self, scale, corebfs_enabled, sym_edge_list):
        """BfsBase::construct (bfs.hpp:116-139): sym_edge_list is the
        symmetric (v0, v1) list produced by make_symmetry_edge_list."""
        flags = BUILD_INPUT_SYMMETRIC | (BUILD_COREBFS if corebfs_enabled else 0)
        self._corebfs = corebfs_enabled
        self.engine.build_from_edges(sym_edge_list, scale, flags)

    def construct_generated(self, scale, edgefactor=16, corebfs_enabled=False,
                            group_reorder=False):
        """generate_graph_spec2010 + make_symmetry_edge_list + construct
        (main.cc:412-435) entirely on the device."""
        flags = (BUILD_COREBFS if corebfs_enabled else 0) | (
            BUILD_GROUP_REORDER if group_reorder else 0)
        self._corebfs = corebfs_enabled
        self.engine.generate_graph(scale, edgefactor, flags=flags)

    def prepare_bfs(self, validation_level, pre_exec, real_benchmark, edgefactor, alpha, beta,
                    pred=None):
        self.engine.prepare(edgefactor, alpha, beta)

    def run_bfs(self, root, pred, edgefactor, alpha, beta, auto_tuning_data):
        """BfsBase::run_bfs (bfs.hpp:3214); pred is filled by get_pred."""
        at = auto_tuning_data
        if at is None:
            at = np.full(AUTO_NUM, AUTO_NOT_DEFINED, dtype=np.int64)
        self.engine.run(root, edgefactor, alpha, beta, at)
        self._pred_out = pred

    def get_pred(self, pred):
        """BfsBase::get_pred (bfs.hpp:161-163): device -> host copy of pred."""
        self.engine.get_pred(pred)

    def end_bfs(self):
        self.engine.end()

    def has_edge(self, root):
        return self.engine.has_edge(root)
