"""ctypes wrapper of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, always as the checker or the timed CPU
restatement of the reference algorithm, never by the product library.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")

USERSEED1, USERSEED2 = 2, 3  # mpi/parameters.h:204-205
AUTO_NUM = 9
AUTO_NOT_DEFINED = -1

# Known traversed-edge counts for edgefactor 16, seeds (2, 3)
# (mpi/utils.hpp:3687-3733, index = SCALE).
PF_NEDGE = [
    -1, 32, 64, 128, 256, 512, 1024, 2048, 4096, 8192, 16383, 32767, 65535,
    131070, 262144, 524285, 1048570, 2097137, 4194250, 8388513, 16776976,
    33553998, 67108130, 134216177, 268432547, 536865258, 1073731075,
    2147462776, 4294927670,
]


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


_lib = None


class _Graph(ctypes.Structure):
    _fields_ = [
        ("nverts", ctypes.c_int64),
        ("scale", ctypes.c_int),
        ("row_ptr", ctypes.POINTER(ctypes.c_int64)),
        ("col", ctypes.POINTER(ctypes.c_int64)),
        ("multideg", ctypes.POINTER(ctypes.c_int64)),
        ("num_edges", ctypes.c_int64),
        ("num_verts", ctypes.c_int64),
    ]


class _Core(ctypes.Structure):
    _fields_ = [
        ("core", ctypes.POINTER(_Graph)),
        ("tree_parent", ctypes.POINTER(ctypes.c_int64)),
        ("peel_round", ctypes.POINTER(ctypes.c_int32)),
        ("rounds", ctypes.c_int),
    ]


class BfsStats(ctypes.Structure):
    _fields_ = [
        ("levels", ctypes.c_int),
        ("edges_td", ctypes.c_int64),
        ("edges_bu", ctypes.c_int64),
        ("visited", ctypes.c_int64),
        ("direction_mask", ctypes.c_uint32),
    ]


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        i64, u64, i32, dbl = ctypes.c_int64, ctypes.c_uint64, ctypes.c_int, ctypes.c_double
        vp = ctypes.c_void_p
        L.orc_generate_edges.argtypes = [i32, u64, u64, i64, i64, vp]
        L.orc_make_random_numbers.argtypes = [i64, u64, u64, i64, vp]
        L.orc_scramble_values.argtypes = [u64, u64, vp, vp]
        L.orc_scramble.argtypes = [i64, i32, u64, u64]
        L.orc_scramble.restype = i64
        L.orc_mrg_pow2_matrix.argtypes = [i32, vp]
        L.orc_graph_build.argtypes = [vp, i64, i32]
        L.orc_graph_build.restype = ctypes.POINTER(_Graph)
        L.orc_graph_free.argtypes = [ctypes.POINTER(_Graph)]
        L.orc_bfs.argtypes = [ctypes.POINTER(_Graph), i64, i64, i32, dbl, dbl, vp, vp,
                              ctypes.POINTER(BfsStats)]
        L.orc_bfs_levels_simple.argtypes = [ctypes.POINTER(_Graph), i64, vp]
        L.orc_validate.argtypes = [vp, i64, i64, i64, i32, i64, vp, vp]
        L.orc_validate.restype = i64
        L.orc_core_build.argtypes = [ctypes.POINTER(_Graph)]
        L.orc_core_build.restype = ctypes.POINTER(_Core)
        L.orc_core_reset_unreachable.argtypes = [ctypes.POINTER(_Core), i32, dbl, dbl]
        L.orc_core_has_edge.argtypes = [ctypes.POINTER(_Core), i64]
        L.orc_core_run_bfs.argtypes = [ctypes.POINTER(_Core), i64, i32, dbl, dbl, vp, vp,
                                       ctypes.POINTER(BfsStats)]
        L.orc_core_free.argtypes = [ctypes.POINTER(_Core)]
        L.orc_find_roots.argtypes = [vp, i64, i32, i32, i32, vp]
        L.orc_num_threads.restype = i32
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def num_threads():
    return lib().orc_num_threads()


def generate_edges(scale, edgefactor=16, start=0, end=None, seed1=USERSEED1, seed2=USERSEED2):
    """Kronecker edges [start, end) as an (m, 2) int64 array."""
    if end is None:
        end = (1 << scale) * edgefactor
    out = np.empty((end - start, 2), dtype=np.int64)
    lib().orc_generate_edges(scale, seed1, seed2, start, end, _ptr(out))
    return out


def make_random_numbers(n, seed1, seed2, position):
    out = np.empty(n, dtype=np.float64)
    lib().orc_make_random_numbers(n, seed1, seed2, position, _ptr(out))
    return out


def scramble_values(seed1=USERSEED1, seed2=USERSEED2):
    a = np.zeros(1, np.uint64)
    b = np.zeros(1, np.uint64)
    lib().orc_scramble_values(seed1, seed2, _ptr(a), _ptr(b))
    return int(a[0]), int(b[0])


def mrg_pow2_matrix(k):
    out = np.zeros(25, np.uint32)
    lib().orc_mrg_pow2_matrix(k, _ptr(out))
    return out.reshape(5, 5)


class Graph:
    """Symmetric, de-duplicated CSR of a generated edge list."""

    def __init__(self, edges, scale=0):
        edges = np.ascontiguousarray(edges, dtype=np.int64)
        self._edges = edges
        self._g = lib().orc_graph_build(_ptr(edges), edges.shape[0], scale)
        g = self._g.contents
        self.nverts = g.nverts
        self.scale = g.scale
        self.num_edges = g.num_edges
        self.num_verts = g.num_verts
        self.row_ptr = np.ctypeslib.as_array(g.row_ptr, shape=(self.nverts + 1,))
        self.col = np.ctypeslib.as_array(g.col, shape=(max(self.num_edges, 1),))[: self.num_edges]
        self.multideg = np.ctypeslib.as_array(g.multideg, shape=(self.nverts,))

    def __del__(self):
        if getattr(self, "_g", None):
            lib().orc_graph_free(self._g)
            self._g = None

    def has_edge(self):
        return (np.diff(self.row_ptr) > 0).astype(np.uint8)

    def bfs(self, root, edgefactor=16, alpha=10.0, beta=14.0, root_level=0):
        pred = np.empty(self.nverts, dtype=np.int64)
        at = np.full(AUTO_NUM, AUTO_NOT_DEFINED, dtype=np.int64)
        st = BfsStats()
        lib().orc_bfs(self._g, root, root_level, edgefactor, alpha, beta, _ptr(pred), _ptr(at),
                      ctypes.byref(st))
        return pred, at, st

    def levels(self, root):
        lv = np.empty(self.nverts, dtype=np.int32)
        lib().orc_bfs_levels_simple(self._g, root, _ptr(lv))
        return lv


class Core:
    """CoreBFS index: 2-core graph plus tree parents of pruned vertices."""

    def __init__(self, graph, edgefactor=16, alpha=10.0, beta=14.0):
        self._c = lib().orc_core_build(graph._g)
        if not self._c:
            raise RuntimeError("more than 32 pruning rounds")
        lib().orc_core_reset_unreachable(self._c, edgefactor, alpha, beta)
        c = self._c.contents
        self.rounds = c.rounds
        n = graph.nverts
        self.nverts = n
        self.tree_parent = np.ctypeslib.as_array(c.tree_parent, shape=(n,))
        self.peel_round = np.ctypeslib.as_array(c.peel_round, shape=(n,))
        k = c.core.contents
        self.core_num_edges = k.num_edges
        self.core_num_verts = k.num_verts
        self.core_row_ptr = np.ctypeslib.as_array(k.row_ptr, shape=(n + 1,))

    def __del__(self):
        if getattr(self, "_c", None):
            lib().orc_core_free(self._c)
            self._c = None

    def has_edge(self):
        return ((np.diff(self.core_row_ptr) > 0) | (self.tree_parent >= 0)).astype(np.uint8)

    def bfs(self, root, edgefactor=16, alpha=10.0, beta=14.0):
        pred = np.empty(self.nverts, dtype=np.int64)
        at = np.full(AUTO_NUM, AUTO_NOT_DEFINED, dtype=np.int64)
        st = BfsStats()
        rc = lib().orc_core_run_bfs(self._c, root, edgefactor, alpha, beta, _ptr(pred), _ptr(at),
                                    ctypes.byref(st))
        if rc != 0:
            raise RuntimeError("tree climb failed")
        return pred, at, st


def validate(edges, nglobalverts, pred, root, corebfs=False, nlocalverts=None):
    """Graph500 validation; returns (error_count, edge_visit_count)."""
    edges = np.ascontiguousarray(edges, dtype=np.int64)
    pred = np.ascontiguousarray(pred, dtype=np.int64).copy()
    if nlocalverts is None:
        nlocalverts = pred.shape[0]
    cnt = np.zeros(1, np.int64)
    err = lib().orc_validate(_ptr(edges), edges.shape[0], nglobalverts, nlocalverts,
                             1 if corebfs else 0, root, _ptr(pred), _ptr(cnt))
    return int(err), int(cnt[0])


def find_roots(has_edge, nglobalverts, num_roots, r1=0, r2=0):
    has_edge = np.ascontiguousarray(has_edge, dtype=np.uint8)
    roots = np.zeros(num_roots, np.int64)
    k = lib().orc_find_roots(_ptr(has_edge), nglobalverts, num_roots, r1, r2, _ptr(roots))
    return roots[:k]


def pred_levels(pred):
    """Per-vertex level from pred entries: (pred >> 48) & 0xFFFF, -1 unreached."""
    pred = np.asarray(pred, dtype=np.int64)
    lv = ((pred.view(np.uint64) >> np.uint64(48)) & np.uint64(0xFFFF)).astype(np.int32)
    lv[pred == -1] = -1
    return lv


def pred_parents(pred):
    pred = np.asarray(pred, dtype=np.int64)
    return (pred << 16) >> 16


def resolve_levels(pred):
    """Exact per-vertex levels of a pred in the reference encoding, with
    CoreBFS tree entries (level field 0xFFFF, corebfs_adaptor.hpp:290-296)
    given their parent's level + 1, resolved round by round as
    validate.hpp:1040-1141 does; -1 unreached.  Returns (levels, tree) with
    tree[v] the parent of a tree entry, -1 elsewhere."""
    pred = np.asarray(pred, dtype=np.int64)
    reached = pred != -1
    lv = np.where(reached, (pred >> 48) & 0xFFFF, -1).astype(np.int64)
    par = np.where(reached, pred & ((1 << 48) - 1), -1).astype(np.int64)
    tree = np.where(lv == 0xFFFF, par, -1)
    while True:
        todo = np.nonzero(lv == 0xFFFF)[0]
        if todo.size == 0:
            break
        pl = lv[par[todo]]
        ok = (pl != 0xFFFF) & (pl >= 0)
        if not ok.any():
            raise ValueError("tree entries whose parents never resolve")
        lv[todo[ok]] = pl[ok] + 1
    return lv, tree


def find_roots_in_large_graph(has_edge, nglobalverts, num_roots, search_levels, seed=0):
    """main.cc:334-359: roots from find_roots(seed, 0); while any root's search
    has at most REMOVE_ROOTS_LEVEL_THED = 3 levels (auto_tuning_data[8]) and
    SCALE > REMOVE_ROOTS_SCALE_THED = 6, pick again with the next seed.
    search_levels(root) returns that root's auto_tuning_data[8]."""
    r = seed
    scale = int(nglobalverts).bit_length() - 1
    while True:
        roots = find_roots(has_edge, nglobalverts, num_roots, r, 0)
        r += 1
        if scale <= 6 or all(search_levels(int(x)) > 3 for x in roots):
            return roots
