"""The C++ API as a reference user would call it: tests/cxx/pcg_amg_example.cpp
is compiled against include/ with g++ and linked with liblinalg_b200.so, then
run on the GPU and checked against the oracle."""
import os
import subprocess

import numpy as np
import pytest

from linalglib_b200 import problems as P

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cxx", "pcg_amg_example.cpp")
LIBDIR = os.path.join(ROOT, "linalglib_b200")


@pytest.fixture(scope="module")
def example(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("cxx") / "pcg_amg_example")
    subprocess.run(["/usr/bin/g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                    SRC, "-o", exe, "-L", LIBDIR, "-llinalg_b200", f"-Wl,-rpath,{LIBDIR}"],
                   check=True)
    return exe


def test_cxx_example_matches_oracle(gpu, oracle, example):
    n = 96
    out = subprocess.run([example, str(n)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    levels, cycles, iters, conv, err1, err2, rel, nnz_total = out.stdout.split()
    A = P.poisson2d(n)
    h = oracle.amg_setup(A)
    assert int(levels) == h.levels
    assert int(nnz_total) == sum(h.A(l)[2].size for l in range(h.levels + 1))
    b = P.csr_matvec(*A[:3], np.ones(n * n))
    _, it_o, _ = h.pcg(b, rel_tol=1e-8, abs_tol=0.0, coarse=1)
    assert abs(int(iters) - it_o) <= 1
    _, cyc_o = h.amg_solve(b, rel_tol=1e-8, abs_tol=0.0, max_cycle=300, coarse=1)
    assert abs(int(cycles) - cyc_o) <= 1
    assert int(conv) == 1 and float(rel) <= 1e-8
