"""Test infrastructure only: ctypes access to the two CPU oracles.

``Oracle``    -- this project's C restatement (oracle/liboracle.so, oracle.c).
``Reference`` -- the reference LinAlgLib host path compiled from its own sources
                 (oracle/_ref/liblinalg_ref.so, built by oracle/Makefile), or
                 None-returning ``load_reference()`` where it was not built.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline arm use this
module, as the checker; the CUDA library never calls it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "liblinalg_ref.so")

_i = C.c_int
_d = C.c_double
_p = C.c_void_p


def reference_root() -> str:
    """Where the reference LinAlgLib sources are: $LINALGLIB_REF, else the
    default location the Makefile uses (its REF variable)."""
    return os.environ.get("LINALGLIB_REF", "/root/reference")


def build(reference: bool = True) -> None:
    """Compile the oracle (and, where the reference sources exist, oracle/_ref)."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    if reference:
        subprocess.run(["make", "-s", "-j8", "-C", HERE, "ref", f"REF={reference_root()}"],
                       check=True)


def _ptr(a):
    return None if a is None else a.ctypes.data


class _Csr(C.Structure):
    _fields_ = [("m", _i), ("n", _i), ("nnz", _i), ("rp", C.POINTER(_i)),
                ("ci", C.POINTER(_i)), ("v", C.POINTER(_d))]


def _csr_in(rp, ci, v, n=None):
    rp = np.ascontiguousarray(rp, dtype=np.int32)
    ci = np.ascontiguousarray(ci, dtype=np.int32)
    v = np.ascontiguousarray(v, dtype=np.float64)
    m = rp.size - 1
    s = _Csr(m, m if n is None else n, int(rp[-1]),
             rp.ctypes.data_as(C.POINTER(_i)), ci.ctypes.data_as(C.POINTER(_i)),
             v.ctypes.data_as(C.POINTER(_d)))
    s._keep = (rp, ci, v)
    return s


def _csr_out(s: _Csr):
    m, nnz = s.m, s.nnz
    rp = np.ctypeslib.as_array(s.rp, shape=(m + 1,)).copy()
    ci = np.ctypeslib.as_array(s.ci, shape=(max(nnz, 1),))[:nnz].copy()
    v = np.ctypeslib.as_array(s.v, shape=(max(nnz, 1),))[:nnz].copy()
    return rp, ci, v, s.n


class _Hier(C.Structure):
    _fields_ = [("levels", _i), ("A", _Csr * 21), ("P", _Csr * 20), ("R", _Csr * 20),
                ("coarse_inv", C.POINTER(_d))]


class Oracle:
    """The C restatement (oracle.c)."""

    SA, UA, RS = 0, 1, 2
    # smoother codes of vcycle / pcg / amg_solve
    JACOBI, GS, MC_GS, MC_SSOR = 0, 1, 2, 3

    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build(reference=False)
        L = C.CDLL(path)
        self.L = L
        P = C.POINTER(_Csr)
        L.orc_csr_free.argtypes = [P]
        L.orc_spmv.argtypes = [P, _d, _p, _d, _p]
        L.orc_residual.argtypes = [P, _p, _p, _p]
        L.orc_transpose.argtypes = [P, P]
        L.orc_spgemm.argtypes = [P, P, P]
        L.orc_spgeam.argtypes = [_d, P, _d, P, P]
        L.orc_strength.argtypes = [P, _d, _p]
        L.orc_pmis.argtypes = [P, _p, _p, _p]
        L.orc_sa_prolongation.argtypes = [P, _p, _p, _d, P]
        L.orc_ua_prolongation.argtypes = [P, _p, P]
        L.orc_classical_strength.argtypes = [P, _d, _p, P]
        L.orc_cfpoints.argtypes = [P, P, _p]
        L.orc_direct_interpolation.argtypes = [P, P, _p, P]
        L.orc_amg_setup.argtypes = [_i, P, _i]
        L.orc_amg_setup.restype = C.POINTER(_Hier)
        L.orc_hier_free.argtypes = [C.POINTER(_Hier)]
        L.orc_vcycle.argtypes = [C.POINTER(_Hier), _i, _p, _p, _i, _i, _i, _d, _i]
        L.orc_amg_pcg.argtypes = [C.POINTER(_Hier), _p, _p, _i, _i, _i, _d, _i, _d, _d, _i,
                                  C.POINTER(_d)]
        L.orc_amg_solve.argtypes = [C.POINTER(_Hier), _p, _p, _i, _i, _i, _d, _i, _d, _d, _i]
        L.orc_cg.argtypes = [P, _p, _p, _i, _d, _d, _i]
        L.orc_exclusive_scan_i64.argtypes = [_p, _i]
        L.orc_mc_colouring.argtypes = [P, _p]
        L.orc_mc_colouring.restype = _i
        L.orc_csrilu0.argtypes = [P, _p, _p]
        L.orc_csric0.argtypes = [P, _p, _p]
        L.orc_trsv.argtypes = [P, _i, _i, _p, _p]
        L.orc_precond_apply.argtypes = [_i, _d, P, _p, _p]
        L.orc_precond_cg.argtypes = [_i, _d, P, _p, _p, _d, _d, _i]
        L.orc_precond_cg.restype = _i

    # -- kernels
    def spmv(self, A, x, alpha=1.0, beta=0.0, y=None):
        s = _csr_in(*A[:3], n=A[3] if len(A) > 3 else None)
        y = np.zeros(s.m) if y is None else np.array(y, dtype=np.float64)
        x = np.ascontiguousarray(x, dtype=np.float64)
        self.L.orc_spmv(C.byref(s), alpha, _ptr(x), beta, _ptr(y))
        return y

    def residual(self, A, x, b):
        s = _csr_in(*A[:3], n=A[3] if len(A) > 3 else None)
        r = np.zeros(s.m)
        x = np.ascontiguousarray(x, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64)
        self.L.orc_residual(C.byref(s), _ptr(x), _ptr(b), _ptr(r))
        return r

    def _out(self, fn, *args):
        o = _Csr()
        fn(*args, C.byref(o))
        res = _csr_out(o)
        self.L.orc_csr_free(C.byref(o))
        return res

    def transpose(self, A):
        s = _csr_in(*A[:3], n=A[3] if len(A) > 3 else None)
        return self._out(self.L.orc_transpose, C.byref(s))

    def spgemm(self, A, B):
        a = _csr_in(*A[:3], n=A[3] if len(A) > 3 else None)
        b = _csr_in(*B[:3], n=B[3] if len(B) > 3 else None)
        return self._out(self.L.orc_spgemm, C.byref(a), C.byref(b))

    def spgeam(self, alpha, A, beta, B):
        a = _csr_in(*A[:3], n=A[3] if len(A) > 3 else None)
        b = _csr_in(*B[:3], n=B[3] if len(B) > 3 else None)
        return self._out(self.L.orc_spgeam, alpha, C.byref(a), beta, C.byref(b))

    def strength(self, A, eps):
        s = _csr_in(*A[:3])
        conn = np.zeros(s.nnz, dtype=np.int32)
        self.L.orc_strength(C.byref(s), eps, _ptr(conn))
        return conn

    def pmis(self, A, conn):
        s = _csr_in(*A[:3])
        conn = np.ascontiguousarray(conn, dtype=np.int32)
        agg = np.zeros(s.m, dtype=np.int64)
        rounds = _i(0)
        self.L.orc_pmis(C.byref(s), _ptr(conn), _ptr(agg), C.byref(rounds))
        return agg, rounds.value

    def sa_prolongation(self, A, conn, agg, relax=2.0 / 3.0):
        s = _csr_in(*A[:3])
        conn = np.ascontiguousarray(conn, dtype=np.int32)
        agg = np.ascontiguousarray(agg, dtype=np.int64)
        return self._out(self.L.orc_sa_prolongation, C.byref(s), _ptr(conn), _ptr(agg), relax)

    def ua_prolongation(self, A, agg):
        s = _csr_in(*A[:3])
        agg = np.ascontiguousarray(agg, dtype=np.int64)
        return self._out(self.L.orc_ua_prolongation, C.byref(s), _ptr(agg))

    def classical_strength(self, A, theta=0.2):
        s = _csr_in(*A[:3])
        conn = np.zeros(s.nnz, dtype=np.int32)
        S = self._out(self.L.orc_classical_strength, C.byref(s), theta, _ptr(conn))
        return conn, S

    def cfpoints(self, S):
        s = _csr_in(*S[:3])
        st = _Csr()
        self.L.orc_transpose(C.byref(s), C.byref(st))
        cf = np.zeros(s.m, dtype=np.uint32)
        self.L.orc_cfpoints(C.byref(s), C.byref(st), _ptr(cf))
        self.L.orc_csr_free(C.byref(st))
        return cf

    def direct_interpolation(self, A, S, cf):
        a = _csr_in(*A[:3])
        s = _csr_in(*S[:3])
        cf = np.ascontiguousarray(cf, dtype=np.uint32)
        return self._out(self.L.orc_direct_interpolation, C.byref(a), C.byref(s), _ptr(cf))

    def exclusive_scan(self, x):
        x = np.array(x, dtype=np.int64)
        self.L.orc_exclusive_scan_i64(_ptr(x), x.size)
        return x

    def mc_colouring(self, A):
        """(colour of every row, number of colours) of the multicolour smoother."""
        s = _csr_in(*A[:3])
        col = np.zeros(s.m + 1, dtype=np.int32)
        nc = self.L.orc_mc_colouring(C.byref(s), _ptr(col))
        return col[:s.m], nc

    # -- hierarchy / solvers
    def amg_setup(self, A, kind=0, max_level=20):
        return OracleHierarchy(self, A, kind, max_level)

    # -- triangular path
    def _factor(self, fn, A):
        s = _csr_in(A[0], A[1], np.array(A[2], dtype=np.float64))  # factored in place
        sz, nz = _i(), _i()
        fn(C.byref(s), C.byref(sz), C.byref(nz))
        return s._keep[2].copy(), sz.value, nz.value

    def csrilu0(self, A):
        """(factored values, structural zero, numeric zero); INT_MAX = none."""
        return self._factor(self.L.orc_csrilu0, A)

    def csric0(self, A):
        return self._factor(self.L.orc_csric0, A)

    def trsv(self, A, b, lower=True, unit_diag=False):
        s = _csr_in(*A[:3])
        x = np.zeros(s.m)
        b = np.ascontiguousarray(b, dtype=np.float64)
        self.L.orc_trsv(C.byref(s), int(lower), int(unit_diag), _ptr(b), _ptr(x))
        return x

    def precond_apply(self, kind, A, rhs, omega=1.0):
        """kind 0 ILU(0), 1 IC(0), 2 Gauss-Seidel, 3 SOR(omega), 4 SSOR(omega)."""
        s = _csr_in(*A[:3])
        x = np.zeros(s.m)
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        self.L.orc_precond_apply(kind, omega, C.byref(s), _ptr(rhs), _ptr(x))
        return x

    def precond_cg(self, kind, A, b, omega=1.0, rel_tol=1e-8, abs_tol=1e-300, max_iter=2000):
        """CG with preconditioner kind (as precond_apply), built once; (x, iterations)."""
        s = _csr_in(*A[:3])
        x = np.zeros(s.m)
        b = np.ascontiguousarray(b, dtype=np.float64)
        it = self.L.orc_precond_cg(kind, omega, C.byref(s), _ptr(b), _ptr(x), rel_tol, abs_tol,
                                   max_iter)
        return x, it

    def cg(self, A, b, x0=None, jacobi=False, rel_tol=1e-6, abs_tol=1e-6, max_iter=1000):
        s = _csr_in(*A[:3])
        x = np.zeros(s.m) if x0 is None else np.array(x0, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64)
        it = self.L.orc_cg(C.byref(s), _ptr(b), _ptr(x), int(jacobi), rel_tol, abs_tol, max_iter)
        return x, it


class OracleHierarchy:
    def __init__(self, orc: Oracle, A, kind, max_level):
        self.orc = orc
        s = _csr_in(*A[:3])
        self.h = orc.L.orc_amg_setup(kind, C.byref(s), max_level)

    def __del__(self):
        try:
            self.orc.L.orc_hier_free(self.h)
        except Exception:
            pass

    @property
    def levels(self):
        return self.h.contents.levels

    def A(self, l):
        return _csr_out(self.h.contents.A[l])

    def P(self, l):
        return _csr_out(self.h.contents.P[l])

    def R(self, l):
        return _csr_out(self.h.contents.R[l])

    def vcycle(self, b, n1=1, n2=1, smoother=0, omega=1.0, coarse=0, x0=None):
        m = self.h.contents.A[0].m
        x = np.zeros(m) if x0 is None else np.array(x0, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64)
        self.orc.L.orc_vcycle(self.h, 0, _ptr(x), _ptr(b), n1, n2, smoother, omega, coarse)
        return x

    def pcg(self, b, x0=None, n1=1, n2=1, smoother=0, omega=1.0, coarse=0, rel_tol=1e-8,
            abs_tol=0.0, max_iter=1000):
        m = self.h.contents.A[0].m
        x = np.zeros(m) if x0 is None else np.array(x0, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64)
        rel = _d(0)
        it = self.orc.L.orc_amg_pcg(self.h, _ptr(b), _ptr(x), n1, n2, smoother, omega, coarse,
                                    rel_tol, abs_tol, max_iter, C.byref(rel))
        return x, it, rel.value

    def amg_solve(self, b, x0=None, n1=1, n2=1, smoother=0, omega=1.0, coarse=0,
                  rel_tol=1e-6, abs_tol=1e-6, max_cycle=200):
        m = self.h.contents.A[0].m
        x = np.zeros(m) if x0 is None else np.array(x0, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64)
        it = self.orc.L.orc_amg_solve(self.h, _ptr(b), _ptr(x), n1, n2, smoother, omega, coarse,
                                      rel_tol, abs_tol, max_cycle)
        return x, it


# ----------------------------------------------------------------- reference
class Reference:
    """The reference host library compiled from its sources (oracle/_ref)."""

    SA, UA, RS = 0, 1, 2

    def __init__(self, path: str = REF_SO):
        L = C.CDLL(path)
        self.L = L
        L.ref_amg_setup.restype = _p
        L.ref_amg_setup.argtypes = [_i, _i, _i, _i, _p, _p, _p, _i]
        L.ref_hier_free.argtypes = [_p]
        L.ref_hier_levels.argtypes = [_p]
        L.ref_hier_dims.argtypes = [_p, _i, _i, _p, _p, _p]
        L.ref_hier_copy.argtypes = [_p, _i, _i, _p, _p, _p]
        L.ref_amg_pcg.argtypes = [_p, _p, _p, _i, _i, _i, _d, _d, _i]
        L.ref_amg_solve.argtypes = [_p, _p, _p, _i, _i, _i, _i, _d, _d, _i]
        L.ref_amg_vcycle.argtypes = [_p, _p, _p, _i, _i, _i]
        L.ref_cg.argtypes = [_i, _i, _p, _p, _p, _p, _p, _i, _d, _d, _i]
        L.ref_gmres.argtypes = [_i, _i, _p, _p, _p, _p, _p, _i, _p, _i, _i, _d, _d, _i]
        L.ref_spmv.argtypes = [_i, _i, _i, _p, _p, _p, _d, _p, _d, _p]
        L.ref_residual.argtypes = [_i, _i, _i, _p, _p, _p, _p, _p, _p]
        L.ref_spgemm.restype = _p
        L.ref_spgemm.argtypes = [_i, _i, _i, _p, _p, _p, _i, _i, _i, _p, _p, _p]
        L.ref_spgeam.restype = _p
        L.ref_spgeam.argtypes = [_d, _i, _i, _i, _p, _p, _p, _d, _i, _p, _p, _p]
        L.ref_csrgemm.restype = _p
        L.ref_csrgemm.argtypes = [_d, _i, _i, _i, _p, _p, _p, _i, _i, _i, _p, _p, _p]
        L.ref_transpose.restype = _p
        L.ref_transpose.argtypes = [_i, _i, _i, _p, _p, _p]
        L.ref_mat_dims.argtypes = [_p, _p, _p, _p]
        L.ref_mat_copy.argtypes = [_p, _p, _p, _p]
        L.ref_mat_free.argtypes = [_p]
        L.ref_strength.argtypes = [_i, _i, _p, _p, _p, _d, _p]
        L.ref_pmis.argtypes = [_i, _i, _p, _p, _p, _p, _p]
        L.ref_classical_strength.restype = _p
        L.ref_classical_strength.argtypes = [_i, _i, _p, _p, _p, _d, _p]
        L.ref_cfpoints.argtypes = [_i, _i, _p, _p, _p, _p]
        L.ref_exclusive_scan_i64.argtypes = [_p, _i]
        L.ref_csrilu0.argtypes = [_i, _i, _p, _p, _p, _p, _p]
        L.ref_csric0.argtypes = [_i, _i, _p, _p, _p, _p, _p]
        L.ref_trsv.argtypes = [_i, _i, _p, _p, _p, _i, _i, _p, _p]
        L.ref_precond_apply.argtypes = [_i, _d, _i, _i, _p, _p, _p, _p, _p]
        L.ref_precond_cg.argtypes = [_i, _d, _i, _i, _p, _p, _p, _p, _p, _d, _d, _i]
        L.ref_triangle.restype = _p
        L.ref_triangle.argtypes = [_i, _i, _i, _p, _p, _p, _i]
        L.ref_scale.argtypes = [_i, _i, _i, _p, _p, _p, _i, _d, _p]
        L.ref_read_mtx.restype = _p
        L.ref_read_mtx.argtypes = [C.c_char_p]
        L.ref_write_mtx.argtypes = [C.c_char_p, _i, _i, _i, _p, _p, _p]

    @staticmethod
    def _arr(A):
        rp = np.ascontiguousarray(A[0], dtype=np.int32)
        ci = np.ascontiguousarray(A[1], dtype=np.int32)
        v = np.ascontiguousarray(A[2], dtype=np.float64)
        n = A[3] if len(A) > 3 else rp.size - 1
        return rp, ci, v, rp.size - 1, n, int(rp[-1])

    def _mat(self, M):
        m, n, z = _i(), _i(), _i()
        self.L.ref_mat_dims(M, C.byref(m), C.byref(n), C.byref(z))
        rp = np.zeros(m.value + 1, dtype=np.int32)
        ci = np.zeros(max(z.value, 1), dtype=np.int32)
        v = np.zeros(max(z.value, 1), dtype=np.float64)
        self.L.ref_mat_copy(M, _ptr(rp), _ptr(ci), _ptr(v))
        self.L.ref_mat_free(M)
        return rp, ci[:z.value], v[:z.value], n.value

    def spmv(self, A, x, alpha=1.0, beta=0.0, y=None):
        rp, ci, v, m, n, z = self._arr(A)
        y = np.zeros(m) if y is None else np.array(y, dtype=np.float64)
        x = np.ascontiguousarray(x, dtype=np.float64)
        self.L.ref_spmv(m, n, z, _ptr(rp), _ptr(ci), _ptr(v), alpha, _ptr(x), beta, _ptr(y))
        return y

    def residual(self, A, x, b):
        rp, ci, v, m, n, z = self._arr(A)
        r = np.zeros(m)
        x = np.ascontiguousarray(x, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64)
        self.L.ref_residual(m, n, z, _ptr(rp), _ptr(ci), _ptr(v), _ptr(x), _ptr(b), _ptr(r))
        return r

    def spgemm(self, A, B):
        a = self._arr(A)
        b = self._arr(B)
        M = self.L.ref_spgemm(a[3], a[4], a[5], _ptr(a[0]), _ptr(a[1]), _ptr(a[2]),
                              b[3], b[4], b[5], _ptr(b[0]), _ptr(b[1]), _ptr(b[2]))
        return self._mat(M)

    def csrgemm(self, alpha, A, B):
        """C = alpha * A * B through the reference's csrgemm_nnz / csrgemm_solve."""
        a = self._arr(A)
        b = self._arr(B)
        M = self.L.ref_csrgemm(alpha, a[3], a[4], a[5], _ptr(a[0]), _ptr(a[1]), _ptr(a[2]),
                               b[3], b[4], b[5], _ptr(b[0]), _ptr(b[1]), _ptr(b[2]))
        return self._mat(M)

    def spgeam(self, alpha, A, beta, B):
        a = self._arr(A)
        b = self._arr(B)
        M = self.L.ref_spgeam(alpha, a[3], a[4], a[5], _ptr(a[0]), _ptr(a[1]), _ptr(a[2]),
                              beta, b[5], _ptr(b[0]), _ptr(b[1]), _ptr(b[2]))
        return self._mat(M)

    def transpose(self, A):
        a = self._arr(A)
        return self._mat(self.L.ref_transpose(a[3], a[4], a[5], _ptr(a[0]), _ptr(a[1]),
                                              _ptr(a[2])))

    def strength(self, A, eps):
        rp, ci, v, m, n, z = self._arr(A)
        conn = np.zeros(z, dtype=np.int32)
        self.L.ref_strength(m, z, _ptr(rp), _ptr(ci), _ptr(v), eps, _ptr(conn))
        return conn

    def pmis(self, A, conn):
        rp, ci, v, m, n, z = self._arr(A)
        conn = np.ascontiguousarray(conn, dtype=np.int32)
        agg = np.zeros(m, dtype=np.int64)
        self.L.ref_pmis(m, z, _ptr(rp), _ptr(ci), _ptr(v), _ptr(conn), _ptr(agg))
        return agg

    def classical_strength(self, A, theta=0.2):
        rp, ci, v, m, n, z = self._arr(A)
        conn = np.zeros(z, dtype=np.int32)
        M = self.L.ref_classical_strength(m, z, _ptr(rp), _ptr(ci), _ptr(v), theta, _ptr(conn))
        return conn, self._mat(M)

    def cfpoints(self, S):
        rp, ci, v, m, n, z = self._arr(S)
        cf = np.zeros(m, dtype=np.uint32)
        self.L.ref_cfpoints(m, z, _ptr(rp), _ptr(ci), _ptr(v), _ptr(cf))
        return cf

    def exclusive_scan(self, x):
        x = np.array(x, dtype=np.int64)
        self.L.ref_exclusive_scan_i64(_ptr(x), x.size)
        return x

    def amg_setup(self, A, kind=0, max_level=20):
        return ReferenceHierarchy(self, A, kind, max_level)

    def cg(self, A, b, x0=None, jacobi=False, rel_tol=1e-6, abs_tol=1e-6, max_iter=1000):
        rp, ci, v, m, n, z = self._arr(A)
        x = np.zeros(m) if x0 is None else np.array(x0, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64)
        it = self.L.ref_cg(m, z, _ptr(rp), _ptr(ci), _ptr(v), _ptr(b), _ptr(x), int(jacobi),
                           rel_tol, abs_tol, max_iter)
        return x, it

    # -- triangular path
    def _factor(self, fn, A):
        rp, ci, v, m, n, z = self._arr(A)
        v = v.copy()
        sz, nz = _i(2**31 - 1), _i(2**31 - 1)
        fn(m, z, _ptr(rp), _ptr(ci), _ptr(v), C.byref(sz), C.byref(nz))
        return v, sz.value, nz.value

    def csrilu0(self, A):
        return self._factor(self.L.ref_csrilu0, A)

    def csric0(self, A):
        return self._factor(self.L.ref_csric0, A)

    def trsv(self, A, b, lower=True, unit_diag=False):
        rp, ci, v, m, n, z = self._arr(A)
        x = np.zeros(m)
        b = np.ascontiguousarray(b, dtype=np.float64)
        self.L.ref_trsv(m, z, _ptr(rp), _ptr(ci), _ptr(v), int(lower), int(unit_diag), _ptr(b),
                        _ptr(x))
        return x

    def precond_apply(self, kind, A, rhs, omega=1.0):
        rp, ci, v, m, n, z = self._arr(A)
        x = np.zeros(m)
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        self.L.ref_precond_apply(kind, omega, m, z, _ptr(rp), _ptr(ci), _ptr(v), _ptr(rhs), _ptr(x))
        return x

    def precond_cg(self, kind, A, b, omega=1.0, rel_tol=1e-8, abs_tol=1e-300, max_iter=2000):
        rp, ci, v, m, n, z = self._arr(A)
        x = np.zeros(m)
        b = np.ascontiguousarray(b, dtype=np.float64)
        it = self.L.ref_precond_cg(kind, omega, m, z, _ptr(rp), _ptr(ci), _ptr(v), _ptr(b),
                                   _ptr(x), rel_tol, abs_tol, max_iter)
        return x, it

    def triangle(self, A, upper=False):
        """copy_lower_triangular_from / copy_upper_triangular_from."""
        rp, ci, v, m, n, z = self._arr(A)
        return self._mat(self.L.ref_triangle(m, n, z, _ptr(rp), _ptr(ci), _ptr(v), int(upper)))

    def scale_diagonal(self, A, scalar):
        rp, ci, v, m, n, z = self._arr(A)
        out = np.zeros(max(z, 1))
        self.L.ref_scale(m, n, z, _ptr(rp), _ptr(ci), _ptr(v), 0, scalar, _ptr(out))
        return out[:z]

    def scale_by_inverse_diagonal(self, A):
        rp, ci, v, m, n, z = self._arr(A)
        out = np.zeros(max(z, 1))
        self.L.ref_scale(m, n, z, _ptr(rp), _ptr(ci), _ptr(v), 1, 0.0, _ptr(out))
        return out[:z]

    def read_mtx(self, path):
        """csr_matrix::read_mtx: (rp, ci, v, n), or None where it returns false."""
        M = self.L.ref_read_mtx(str(path).encode())
        return None if not M else self._mat(M)

    def write_mtx(self, path, A):
        rp, ci, v, m, n, z = self._arr(A)
        return bool(self.L.ref_write_mtx(str(path).encode(), m, n, z, _ptr(rp), _ptr(ci),
                                         _ptr(v)))

    # No gmres(): the reference's gmres_solver::build leaves its residual vectors
    # unsized (gmres.cpp:211-220) and its solve writes out of bounds (it crashed
    # the test process); gmres_restated() below is the GMRES checker.


class ReferenceHierarchy:
    def __init__(self, ref: Reference, A, kind, max_level):
        self.ref = ref
        rp, ci, v, m, n, z = ref._arr(A)
        self.h = ref.L.ref_amg_setup(kind, m, n, z, _ptr(rp), _ptr(ci), _ptr(v), max_level)

    def __del__(self):
        try:
            self.ref.L.ref_hier_free(self.h)
        except Exception:
            pass

    @property
    def levels(self):
        return self.ref.L.ref_hier_levels(self.h)

    def _get(self, l, which):
        m, n, z = _i(), _i(), _i()
        self.ref.L.ref_hier_dims(self.h, l, which, C.byref(m), C.byref(n), C.byref(z))
        rp = np.zeros(m.value + 1, dtype=np.int32)
        ci = np.zeros(max(z.value, 1), dtype=np.int32)
        v = np.zeros(max(z.value, 1), dtype=np.float64)
        self.ref.L.ref_hier_copy(self.h, l, which, _ptr(rp), _ptr(ci), _ptr(v))
        return rp, ci[:z.value], v[:z.value], n.value

    def A(self, l):
        return self._get(l, 0)

    def P(self, l):
        return self._get(l, 1)

    def R(self, l):
        return self._get(l, 2)

    def vcycle(self, b, n1=1, n2=1, smoother=0):
        m = self.A(0)[0].size - 1
        z = np.zeros(m)
        b = np.ascontiguousarray(b, dtype=np.float64)
        self.ref.L.ref_amg_vcycle(self.h, _ptr(b), _ptr(z), n1, n2, smoother)
        return z

    def pcg(self, b, x0=None, n1=1, n2=1, smoother=0, rel_tol=1e-8, abs_tol=1e-300,
            max_iter=1000):
        m = self.A(0)[0].size - 1
        x = np.zeros(m) if x0 is None else np.array(x0, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64)
        it = self.ref.L.ref_amg_pcg(self.h, _ptr(b), _ptr(x), n1, n2, smoother, rel_tol,
                                    abs_tol, max_iter)
        return x, it

    def amg_solve(self, b, x0=None, n1=1, n2=1, cycle=0, smoother=0, rel_tol=1e-6,
                  abs_tol=1e-6, max_cycle=200):
        m = self.A(0)[0].size - 1
        x = np.zeros(m) if x0 is None else np.array(x0, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64)
        it = self.ref.L.ref_amg_solve(self.h, _ptr(b), _ptr(x), n1, n2, cycle, smoother,
                                      rel_tol, abs_tol, max_cycle)
        return x, it


def gmres_restated(A, b, restart, rel_tol=1e-6, abs_tol=1e-6, max_iter=1000, x0=None,
                   precond=None):
    """Unpreconditioned restarted GMRES as the reference runs it
    (library/src/iterative_solvers/krylov/gmres.cpp:224-368): modified Gram-Schmidt
    Arnoldi (93-161), Givens rotations (163-199), 2-norm stopping test relative to
    the initial residual, back substitution, restart from the true residual.
    Returns (x, restart cycles).  The reference's own gmres_solver::build leaves
    its residual vectors unsized (gmres.cpp:211-220), so its solve writes out of
    bounds; this restatement is the checker instead.

    With ``precond`` (a callable z = M^-1 r): left preconditioning as
    gmres_solver::solve_precond states it (gmres.cpp:370-523): the stopping test
    and the Arnoldi basis use z = M^-1 (b - A x) and M^-1 A q (arnoldi,
    gmres.cpp:112-129, whose preconditioned output this restatement uses)."""
    rp, ci, v = (np.asarray(a) for a in A[:3])
    n = rp.size - 1
    rows = np.repeat(np.arange(n), np.diff(rp))

    def mv(x):
        return np.bincount(rows, weights=v * x[ci], minlength=n)

    restart = min(restart, n - 1)
    x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64)

    def conv(rn, r0):
        if np.isnan(rn) or np.isnan(r0):
            return False
        return rn <= abs_tol or rn / r0 <= rel_tol

    M = precond if precond is not None else (lambda r: r)
    op = (lambda q: M(mv(q))) if precond is not None else mv
    r = M(b - mv(x))
    rn = np.linalg.norm(r)
    r0 = rn
    if conv(rn, r0):
        return x, 0
    it = 0
    while not it > max_iter:
        Q = np.zeros((restart + 1, n))
        H = np.zeros((restart + 1, restart))
        cs = np.zeros(restart)
        sn = np.zeros(restart)
        g = np.zeros(restart + 1)
        Q[0] = r / rn
        g[0] = rn
        k = 1
        while k <= restart:
            w = op(Q[k - 1])
            for i in range(k):
                H[i, k - 1] = np.dot(Q[i], w)
                w = w - H[i, k - 1] * Q[i]
            H[k, k - 1] = np.sqrt(np.dot(w, w))
            Q[k] = w / H[k, k - 1]
            for i in range(k - 1):
                t1, t2 = H[i, k - 1], H[i + 1, k - 1]
                H[i, k - 1] = cs[i] * t1 + sn[i] * t2
                H[i + 1, k - 1] = -sn[i] * t1 + cs[i] * t2
            xi, xj = H[k - 1, k - 1], H[k, k - 1]
            if xi == 0.0:
                cs[k - 1], sn[k - 1] = 0.0, 1.0
            elif xj == 0.0:
                cs[k - 1], sn[k - 1] = 1.0, 0.0
            elif abs(xi) > abs(xj):
                t = xj / xi
                cs[k - 1] = 1.0 / np.sqrt(1.0 + t * t)
                sn[k - 1] = t * cs[k - 1]
            else:
                t = xi / xj
                sn[k - 1] = 1.0 / np.sqrt(1.0 + t * t)
                cs[k - 1] = t * sn[k - 1]
            t1, t2 = H[k - 1, k - 1], H[k, k - 1]
            H[k - 1, k - 1] = cs[k - 1] * t1 + sn[k - 1] * t2
            H[k, k - 1] = -sn[k - 1] * t1 + cs[k - 1] * t2
            g[k] = -sn[k - 1] * g[k - 1]
            g[k - 1] = cs[k - 1] * g[k - 1]
            if conv(abs(g[k]), r0) or k == restart:
                break
            k += 1
        y = g[:k].copy()
        for i in range(k - 1, -1, -1):
            for j in range(i + 1, k):
                y[i] -= H[i, j] * y[j]
            y[i] /= H[i, i]
        x = x + Q[:k].T @ y
        r = M(b - mv(x))
        rn = np.linalg.norm(r)
        if conv(rn, r0):
            break
        it += 1
    return x, it


def load_reference():
    """The compiled reference, or None where oracle/_ref was not built."""
    if os.path.exists(REF_SO):
        return Reference(REF_SO)
    return None
