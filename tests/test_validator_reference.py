"""The Graph500 validators against the reference's own (no GPU).

For a valid pred and for each single-fault corruption of it
(tests/pred_corruptions.py), the reference's validate_bfs_result
(oracle/_ref/ref_validate: mpi/validate.hpp over the reference's own graph)
and the oracle's restatement (oracle.validate) must agree: the valid pred is
accepted with the same traversed-edge count, every corruption is rejected.
Plain and CoreBFS modes."""
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from pred_corruptions import corruptions

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_VALIDATE = os.path.join(ROOT, "oracle", "_ref", "ref_validate")


def reference_verdicts(scale, root, corebfs, preds, tmp_path):
    if not os.path.exists(REF_VALIDATE):
        pytest.fail("oracle/_ref/ref_validate missing: build it with `make -C oracle/ref` "
                    "where the reference tree is")
    files = []
    for i, p in enumerate(preds):
        f = tmp_path / ("pred_%02d.bin" % i)
        np.ascontiguousarray(p, np.int64).tofile(f)
        files.append(str(f))
    cmd = [REF_VALIDATE, str(scale), str(root)] + (["-C"] if corebfs else []) + files
    env = dict(os.environ, OMP_NUM_THREADS=str(min(os.cpu_count() or 1, 8)))
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=300, env=env)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l.split() for l in p.stdout.splitlines() if l.strip()]
    assert len(lines) == len(preds)
    return [(int(a), int(b)) for a, b in lines]


@pytest.mark.parametrize("scale,corebfs", [(12, False), (14, True)])
def test_validators_agree_with_reference(built, tmp_path, scale, corebfs):
    edges = O.generate_edges(scale)
    g = O.Graph(edges)
    pred_size = max(1 << scale, 1 << 16)  # graph_constructor.hpp:1085-1094
    if corebfs:
        core = O.Core(g)
        has = core.has_edge()
        search = core.bfs
    else:
        has = g.has_edge()
        search = g.bfs
    nglobal = int(np.nonzero(has)[0].max()) + 1  # find_max_used_vertex + 1
    root = int(O.find_roots(has, 1 << scale, 1)[0])
    pred, _, _ = search(root)
    full = np.full(pred_size, -1, np.int64)
    full[: pred.size] = pred
    cases = [("valid", full)] + [(name, p) for name, p in corruptions(
        full, root, g.row_ptr, g.col, nglobal, corebfs=corebfs)]
    names = [c[0] for c in cases]
    # one case per rule; a vertex with edges that the search does not reach
    # (needed for "unreachable_marked_reached") exists only on some graphs
    unreached = ((full[:nglobal] == -1) & (np.diff(g.row_ptr)[:nglobal] > 0)).any()
    assert len(cases) == 7 + int(bool(unreached)) + (2 if corebfs else 0), names
    ref = reference_verdicts(scale, root, corebfs, [c[1] for c in cases], tmp_path)
    for (name, p), (ok, cnt) in zip(cases, ref):
        err, ocnt = O.validate(edges, nglobal, p, root, corebfs=corebfs, nlocalverts=pred_size)
        if name == "valid":
            assert ok == 1 and err == 0 and cnt == ocnt == O.PF_NEDGE[scale], (cnt, ocnt)
        else:
            assert ok == 0, name  # the reference rejects it
            assert err > 0, name  # and so does the oracle
