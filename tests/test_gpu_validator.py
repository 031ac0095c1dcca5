"""The device validator rejects what the Graph500 rules reject.

b200bfs_validate_pred runs the device validator (validate.hpp:607-976
restated in csrc/validate.cu) on a pred the caller supplies.  For the
engine's own valid pred and for each single-fault corruption of it
(tests/pred_corruptions.py: a parent that is no neighbour, a level off by
one, a root that is not its own parent, a reached vertex marked unreached, a
parent out of range, a self-parent, an unreachable vertex marked reached,
and in CoreBFS mode a wrong tree parent and a wrong tree level), its error
count and traversed-edge count must equal the oracle validator's; the
reference's own validator rejects the same corruptions
(tests/test_validator_reference.py)."""
import numpy as np
import pytest

import oracle as O
from pred_corruptions import corruptions

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("scale,corebfs,group", [(14, False, False), (16, True, False),
                                                 (16, True, True), (18, False, True)])
def test_device_validator_matches_oracle(built, scale, corebfs, group):
    import b200bfs

    edges = O.generate_edges(scale)
    g = O.Graph(edges)
    e = b200bfs.Engine(0)
    flags = (b200bfs.BUILD_COREBFS if corebfs else 0) | (
        b200bfs.BUILD_GROUP_REORDER if group else 0)
    e.generate_graph(scale, 16, flags=flags)
    e.prepare(16)
    has = e.has_edge_all()
    nglobal = int(np.nonzero(has)[0].max()) + 1  # find_max_used_vertex + 1
    pred_size = e.info().pred_size
    root = int(e.find_roots(1)[0])
    e.run(root, 16)
    pred = e.get_pred()
    cases = [("valid", pred)] + list(corruptions(pred, root, g.row_ptr, g.col, nglobal,
                                                 corebfs=corebfs))
    # one case per rule; a vertex with edges that the search does not reach
    # (needed for "unreachable_marked_reached") exists only on some graphs
    unreached = ((pred[:nglobal] == -1) & (np.diff(g.row_ptr)[:nglobal] > 0)).any()
    assert len(cases) == 7 + int(bool(unreached)) + (2 if corebfs else 0), [c[0] for c in cases]
    for name, p in cases:
        derr, dcnt = e.validate_pred(root, p, corebfs=corebfs)
        oerr, ocnt = O.validate(edges, nglobal, p, root, corebfs=corebfs, nlocalverts=pred_size)
        assert (derr, dcnt) == (oerr, ocnt), (name, derr, dcnt, oerr, ocnt)
        if name == "valid":
            assert derr == 0 and dcnt == O.PF_NEDGE[scale]
        else:
            assert derr > 0, name
    # the caller's array is read, not modified, and the engine's own result
    # still validates afterwards
    assert np.array_equal(cases[0][1], e.get_pred())
    assert e.validate(root) == (0, O.PF_NEDGE[scale])
    e.close()


def test_validate_pred_arguments(built):
    import b200bfs

    e = b200bfs.Engine(0)
    with pytest.raises(b200bfs.B200BfsError) as ei:  # no graph yet
        e.validate_pred(0, np.zeros(1 << 16, np.int64), corebfs=False)
    assert ei.value.code == 4
    e.generate_graph(12, 16)
    with pytest.raises(ValueError):
        e.validate_pred(0, np.zeros(5, np.int64))
    with pytest.raises(b200bfs.B200BfsError) as ei:  # root out of range
        e.validate_pred(1 << 12, np.full(1 << 16, -1, np.int64))
    assert ei.value.code == 1
    e.close()
