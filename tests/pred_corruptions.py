"""Single-fault corruptions of a valid pred (reference encoding
level << 48 | parent, -1 unreached), one per Graph500 rule that
validate.hpp:607-976 enforces.  Used to check that the oracle's, the
device's and the reference's own validators all reject each of them."""
import numpy as np

PMASK = (1 << 48) - 1


def _enc(level, parent):
    return np.array(((level & 0xFFFF) << 48) | (parent & PMASK), np.uint64).view(np.int64)


def _fields(pred):
    p = np.asarray(pred, np.int64)
    lv = ((p.view(np.uint64) >> np.uint64(48)) & np.uint64(0xFFFF)).astype(np.int64)
    par = (p << 16) >> 16
    return lv, par


def corruptions(pred, root, row_ptr, col, nglobal, corebfs=False, seed=7):
    """Yields (name, corrupted pred).  row_ptr/col: the symmetric CSR in
    original ids (oracle.Graph); nglobal: max used vertex + 1."""
    rng = np.random.default_rng(seed)
    pred = np.asarray(pred, np.int64)
    lv, par = _fields(pred)
    n = nglobal
    reached = np.nonzero((pred[:n] != -1) & (np.arange(n) != root))[0]
    core = reached[lv[reached] != 0xFFFF]  # entries with a real level
    deg = np.diff(row_ptr)

    def nbrs(v):
        return col[row_ptr[v]:row_ptr[v + 1]]

    def pick(cands):
        return int(cands[rng.integers(cands.size)])

    # a vertex whose parent moves to a vertex of the parent's level it has
    # no edge to: "each vertex's parent is a neighbour"
    deep = core[lv[core] >= 2]
    for _ in range(200):
        v = pick(deep)
        u = pick(core[lv[core] == lv[v] - 1])
        if u not in set(nbrs(v).tolist()):
            out = pred.copy()
            out[v] = _enc(lv[v], u)
            yield "parent_not_a_neighbour", out
            break
    # the level of one vertex off by one: "a parent is one level nearer"
    v = pick(core)
    out = pred.copy()
    out[v] = _enc(lv[v] + 1, par[v])
    yield "level_off_by_one", out
    # the root is not its own parent
    out = pred.copy()
    out[root] = _enc(0, int(nbrs(root)[0]))
    yield "root_not_self_parent", out
    # a reached vertex marked unreached: its edges to reached vertices then
    # join a reached and an unreached endpoint
    v = pick(core[deg[core] > 0])
    out = pred.copy()
    out[v] = -1
    yield "reached_left_unreached", out
    # a parent id beyond the vertex range
    v = pick(core)
    out = pred.copy()
    out[v] = _enc(lv[v], n + 3)
    yield "parent_out_of_range", out
    # a vertex that is its own parent
    v = pick(core)
    out = pred.copy()
    out[v] = _enc(lv[v], v)
    yield "self_parent", out
    # an unreachable vertex with edges given a level and the root as parent
    unreached = np.nonzero((pred[:n] == -1) & (deg[:n] > 0))[0]
    rn = set(nbrs(root).tolist())
    unreached = np.array([w for w in unreached.tolist() if w not in rn], np.int64)
    if unreached.size:
        w = pick(unreached)
        out = pred.copy()
        out[w] = _enc(1, root)
        yield "unreachable_marked_reached", out
    if corebfs:
        tree = reached[lv[reached] == 0xFFFF]
        # a pruned (tree) vertex hung on a vertex it has no edge to
        for _ in range(200):
            v = pick(tree)
            u = pick(core)
            if u not in set(nbrs(v).tolist()) and u != v:
                out = pred.copy()
                out[v] = _enc(0xFFFF, u)
                yield "tree_parent_not_a_neighbour", out
                break
        # a tree entry hanging off a core vertex given a real level that is
        # not its parent's + 1
        on_core = tree[lv[par[tree]] != 0xFFFF]
        v = pick(on_core)
        p = int(par[v])
        out = pred.copy()
        out[v] = _enc(int(lv[p]) + 3, p)
        yield "tree_entry_wrong_level", out
