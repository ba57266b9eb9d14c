"""Generate the golden fixtures in this directory from the REFERENCE itself.

    python tests/golden/make_golden.py      (needs oracle/_ref built from the
                                             reference sources: make -C oracle ref)

Each fixture holds a small problem's SA/UA/RS hierarchy exactly as the reference
builds it (every level's A and P), the level-0 strength / aggregation integers,
and for SA/UA the reference's AMG-PCG iteration count and solution.  The tests
check the CPU oracle and the GPU library against these files, so parity stays
pinned on a machine without the reference sources.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))

GOLDEN_CASES = {
    "sa_poisson2d_32": {"problem": "poisson2d", "n": 32, "kind": 0, "eps": 0.08},
    "sa_laplacian3d_8": {"problem": "graph_laplacian3d", "n": 8, "kind": 0, "eps": 0.08},
    "ua_poisson3d_10": {"problem": "poisson3d", "n": 10, "kind": 1, "eps": 0.001},
    "rs_poisson2d_24": {"problem": "poisson2d", "n": 24, "kind": 2},
}


def build_problem(case):
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    from linalglib_b200 import problems as P
    if case["problem"] == "graph_laplacian3d":
        return P.graph_laplacian3d(case["n"], seed=7)
    return getattr(P, case["problem"])(case["n"])


def main():
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    from linalglib_b200 import problems as P
    from oracle.oracle import load_reference
    ref = load_reference()
    if ref is None:
        raise SystemExit("oracle/_ref/liblinalg_ref.so is not built")
    for name, case in GOLDEN_CASES.items():
        A = build_problem(case)
        h = ref.amg_setup(A, kind=case["kind"])
        out = {"A_rp": A[0], "A_ci": A[1], "levels": np.int64(h.levels)}
        for l in range(h.levels + 1):
            a = h.A(l)
            out[f"A{l}_rp"], out[f"A{l}_ci"], out[f"A{l}_v"] = a[0], a[1], a[2]
            if l < h.levels:
                p = h.P(l)
                out[f"P{l}_ci"], out[f"P{l}_v"] = p[1], p[2]
        if case["kind"] in (0, 1):
            conn = ref.strength(A, case["eps"])
            out["conn0"] = conn
            out["agg0"] = ref.pmis(A, conn)
            b, _ = P.rhs_from_solution(*A[:3], seed=0)
            x, it = h.pcg(b, rel_tol=1e-8, abs_tol=1e-300)
            out.update(b=b, pcg_x=x, pcg_iters=np.int64(it), rtol=np.float64(1e-8))
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(name, "levels", h.levels)


if __name__ == "__main__":
    main()
