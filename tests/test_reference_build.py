"""The reference's own programs, built unchanged on the single-rank MPI
runtime (oracle/ref/Makefile), run here without a GPU.

* the runtime's self-test (oracle/ref/shim/shim_selftest.cc);
* ref_runnable / ref_runnable_group: the reference's mpi/main.cc with its
  stock BfsBase, i.e. `mpiexec -n 1 runnable` (plain and group reordering,
  -A -C), whose built-in validation must pass with pf_nedge[SCALE] traversed
  edges for every root (main.cc:645-680, logfile.h:54-133);
* b200_runnable / b200_runnable_group: the same main.cc with
  graph500-bfs_b200/dropin/bfs_cpu.hpp as mpi/bfs_cpu.hpp, linked to
  libb200bfs.so (they need a GPU to run; here only that they were built and
  resolve the library).
"""
import os
import re
import subprocess

import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_BIN = os.path.join(ROOT, "oracle", "_ref")
PROGRAMS = ["ref_runnable", "ref_runnable_group", "ref_dump", "ref_dump_group",
            "b200_runnable", "b200_runnable_group", "gen_golden"]


def _exe(name):
    path = os.path.join(REF_BIN, name)
    if not os.path.exists(path):
        pytest.fail("%s missing: build it with `make -C oracle/ref` where the reference "
                    "tree is" % name)
    return path


def _result(out):
    fields = {}
    for k in ("SCALE", "NBFS", "min_nedge", "max_nedge", "harmonic_mean_TEPS", "alpha", "beta",
              "Reorder bits"):
        m = re.search(r"^%s:\s+(\S+)" % k, out, re.M)
        if m:
            fields[k] = float(m.group(1))
    return fields


def test_shim_selftest(built):
    p = subprocess.run([_exe("shim_selftest")], capture_output=True, text=True, timeout=60)
    assert p.returncode == 0 and p.stdout.strip() == "ok", p.stderr


def test_programs_built(built):
    for name in PROGRAMS:
        assert os.access(_exe(name), os.X_OK), name


@pytest.mark.parametrize("exe,args", [
    ("ref_runnable", ["12", "-n", "4"]),
    ("ref_runnable", ["14", "-A", "-C", "-n", "4"]),
    ("ref_runnable_group", ["14", "-A", "-C", "-n", "4"]),
])
def test_reference_driver_validates(built, exe, args):
    env = dict(os.environ, OMP_NUM_THREADS=str(min(os.cpu_count() or 1, 8)))
    p = subprocess.run([_exe(exe)] + args, capture_output=True, text=True, timeout=300, env=env)
    assert p.returncode == 0, p.stderr[-2000:]
    out = p.stdout + p.stderr
    assert "No results printed for invalid run" not in out
    res = _result(out)
    scale = int(args[0])
    assert res["SCALE"] == scale and res["NBFS"] == 4
    assert res["min_nedge"] == res["max_nedge"] == O.PF_NEDGE[scale], res
    assert res["harmonic_mean_TEPS"] > 0
    if exe.endswith("_group"):
        assert res["Reorder bits"] > 0


@pytest.mark.parametrize("exe", ["b200_runnable", "b200_runnable_group"])
def test_dropin_links_engine(built, exe):
    p = subprocess.run(["ldd", _exe(exe)], capture_output=True, text=True, timeout=60)
    line = [l for l in p.stdout.splitlines() if "libb200bfs.so" in l]
    assert line, p.stdout
    assert os.path.realpath(os.path.join(ROOT, "graph500-bfs_b200", "libb200bfs.so")) in \
        os.path.realpath(line[0].split("=>")[1].split()[0])
