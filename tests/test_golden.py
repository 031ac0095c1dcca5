"""The oracle and the device generator against golden vectors printed by the
reference's own generator sources (generator/graph_generator.hpp,
generator/splittable_mrg.c) compiled unchanged by oracle/ref/make_golden.sh."""
import os
from collections import defaultdict

import numpy as np
import pytest

import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                      "reference_generator.txt")


def load():
    edges = defaultdict(dict)
    rnd = defaultdict(dict)
    for line in open(GOLDEN):
        f = line.split()
        if f[0] == "E":
            s, i, a, b = map(int, f[1:])
            edges[s][i] = (a, b)
        elif f[0] == "R":
            s1, s2, pos, k = map(int, f[1:5])
            rnd[(s1, s2, pos)][k] = float(f[5])
    return edges, rnd


def runs(idx):
    """Contiguous index runs of a sorted index list."""
    idx = sorted(idx)
    start = prev = idx[0]
    for i in idx[1:]:
        if i != prev + 1:
            yield start, prev + 1
            start = i
        prev = i
    yield start, prev + 1


def test_oracle_edges_match_reference(built):
    edges, _ = load()
    for scale, d in edges.items():
        for a, b in runs(d.keys()):
            ours = O.generate_edges(scale, start=a, end=b)
            ref = np.array([d[i] for i in range(a, b)], dtype=np.int64)
            assert np.array_equal(ours, ref), (scale, a, b)


def test_oracle_random_numbers_match_reference(built):
    _, rnd = load()
    for (s1, s2, pos), vals in rnd.items():
        ours = O.make_random_numbers(len(vals), s1, s2, pos)
        ref = np.array([vals[k] for k in range(len(vals))])
        assert np.array_equal(ours, ref), (s1, s2, pos)


@pytest.mark.gpu
def test_device_generator_matches_reference(built):
    import b200bfs

    edges, _ = load()
    e = b200bfs.Engine(0)
    for scale, d in edges.items():
        for a, b in runs(d.keys()):
            ours = e.generate_edges(scale, a, b)
            ref = np.array([d[i] for i in range(a, b)], dtype=np.int64)
            assert np.array_equal(ours, ref), (scale, a, b)
    e.close()
