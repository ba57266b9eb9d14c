"""Thin Python objects over the C ABI: device CSR matrices, hierarchies,
preconditioners and solves.  Vectors are float64 CUDA tensors (torch is used
only for device memory and the current stream).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib as L
from ._lib import AmgOptions, IterControl, SolveInfo, call, call_solve, lib

_initialised = False


def init():
    """Bind the library to torch's current CUDA device (fails loudly without one)."""
    global _initialised
    if _initialised:
        return
    if not torch.cuda.is_available():
        raise L.LabError(L.LAB_NO_DEVICE, "linalglib_b200 needs a CUDA device (sm_100a)")
    torch.cuda.init()
    call("lab_init", torch.cuda.current_device())
    _initialised = True


def stream_handle(stream=None):
    if stream is None:
        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream)


def ptr(t):
    if t is None:
        return None
    if isinstance(t, np.ndarray):
        return C.c_void_p(t.ctypes.data)
    assert t.is_cuda and t.is_contiguous(), "expected a contiguous CUDA tensor"
    return C.c_void_p(t.data_ptr())


def vec(x, dtype=torch.float64):
    """A contiguous float64 CUDA tensor from numpy / list / tensor."""
    if isinstance(x, torch.Tensor):
        return x.to(device="cuda", dtype=dtype).contiguous()
    return torch.as_tensor(np.asarray(x), dtype=dtype, device="cuda").contiguous()


class CsrMatrix:
    """Device CSR matrix owned by the library (lab_csr)."""

    def __init__(self, handle, owner=True, keep=None):
        self.h = C.c_void_p(handle) if not isinstance(handle, C.c_void_p) else handle
        self.owner = owner
        self._keep = keep  # keeps a parent (e.g. hierarchy) alive for borrowed handles

    @classmethod
    def from_arrays(cls, row_ptr, col_ind, val, n=None, stream=None):
        init()
        if any(isinstance(a, torch.Tensor) and a.is_cuda for a in (row_ptr, col_ind, val)):
            # any device operand: all three go to the device
            rp = torch.as_tensor(row_ptr, device="cuda").to(torch.int32).contiguous()
            ci = torch.as_tensor(col_ind, device="cuda").to(torch.int32).contiguous()
            v = torch.as_tensor(val, device="cuda").to(torch.float64).contiguous()
            where = L.MEM_DEVICE
            m = rp.numel() - 1
            nnz = v.numel()
        else:
            rp = np.ascontiguousarray(row_ptr, dtype=np.int32)
            ci = np.ascontiguousarray(col_ind, dtype=np.int32)
            v = np.ascontiguousarray(val, dtype=np.float64)
            where = L.MEM_HOST
            m = rp.size - 1
            nnz = v.size
        n = m if n is None else n
        h = C.c_void_p()
        call("lab_csr_create", C.byref(h), m, n, nnz, ptr(rp), ptr(ci), ptr(v), where,
             stream_handle(stream))
        return cls(h)

    def __del__(self):
        try:
            if self.owner and self.h:
                lib().lab_csr_destroy(self.h)
                self.h = C.c_void_p()
        except Exception:
            pass

    def info(self):
        m, n, z = C.c_int64(), C.c_int64(), C.c_int64()
        call("lab_csr_info", self.h, C.byref(m), C.byref(n), C.byref(z))
        return m.value, n.value, z.value

    @property
    def m(self):
        return self.info()[0]

    @property
    def n(self):
        return self.info()[1]

    @property
    def nnz(self):
        return self.info()[2]

    def to_numpy(self):
        m, n, z = self.info()
        rp = np.zeros(m + 1, dtype=np.int32)
        ci = np.zeros(max(z, 1), dtype=np.int32)
        v = np.zeros(max(z, 1), dtype=np.float64)
        call("lab_csr_copy_to", self.h, ptr(rp), ptr(ci), ptr(v), L.MEM_HOST, stream_handle())
        return rp, ci[:z], v[:z], n

    def analyse(self):
        call("lab_spmv_analysis", self.h, stream_handle())

    def set_values(self, v):
        """Overwrite the stored values in place (same pattern) through the device
        arrays, then tell the library so its cached copies are rebuilt."""
        v = vec(v)
        assert v.numel() == self.nnz
        val = C.c_void_p()
        call("lab_csr_device_arrays", self.h, None, None, C.byref(val))
        call("lab_memcpy", val, ptr(v), 8 * v.numel(), stream_handle())
        call("lab_csr_values_changed", self.h, stream_handle())

    def set_algorithm(self, alg, lanes=0):
        call("lab_spmv_set_algorithm", self.h, alg, lanes)
        self.analyse()

    def autotune(self, exact=False):
        """Time every SpMV schedule on this matrix and keep the fastest; returns
        the winner's microseconds per SpMV."""
        us = C.c_double()
        call("lab_spmv_autotune", self.h, int(bool(exact)), C.byref(us), stream_handle())
        return us.value

    def algorithm(self):
        a, w = C.c_int(), C.c_int()
        call("lab_spmv_get_algorithm", self.h, C.byref(a), C.byref(w))
        return a.value, w.value

    def halo_info(self):
        """(chunks, rows per chunk, distinct staged columns, chunks read directly)
        of the matrix's halo plan; zeros when it has none."""
        v = [C.c_int64() for _ in range(4)]
        call("lab_spmv_halo_info", self.h, *[C.byref(x) for x in v])
        return tuple(x.value for x in v)

    def spmv(self, x, y=None, alpha=1.0, beta=0.0, stream=None):
        if y is None:
            y = torch.zeros(self.m, dtype=torch.float64, device="cuda")
        call("lab_spmv", alpha, self.h, ptr(x), beta, ptr(y), stream_handle(stream))
        return y

    def residual(self, x, b, r=None, stream=None):
        if r is None:
            r = torch.empty(self.m, dtype=torch.float64, device="cuda")
        call("lab_residual", self.h, ptr(x), ptr(b), ptr(r), stream_handle(stream))
        return r

    def spmm(self, X, Y=None, alpha=1.0, beta=0.0):
        """X: (nrhs, n) row-major tensor == column-major n x nrhs."""
        k = X.shape[0]
        if Y is None:
            Y = torch.zeros((k, self.m), dtype=torch.float64, device="cuda")
        call("lab_spmm", alpha, self.h, k, ptr(X), X.shape[1], beta, ptr(Y), Y.shape[1],
             stream_handle())
        return Y

    def diagonal(self):
        d = torch.empty(self.m, dtype=torch.float64, device="cuda")
        call("lab_diagonal", self.h, ptr(d), stream_handle())
        return d

    def _new(self, fn, *args):
        h = C.c_void_p()
        call(fn, *args, C.byref(h), stream_handle())
        return CsrMatrix(h)

    def transpose(self):
        return self._new("lab_transpose", self.h)

    def trsv(self, b, lower=True, unit_diag=False, x=None):
        """x = T^-1 b on the lower or upper part (reference order, bit-identical)."""
        if x is None:
            x = torch.empty_like(b)
        call("lab_csrtrsv", self.h, int(bool(lower)), int(bool(unit_diag)), ptr(b), ptr(x),
             stream_handle())
        return x

    def factor(self, kind):
        """In-place ILU(0) ('ilu0') or IC(0) ('ic0'); returns (structural_zero,
        numeric_zero), -1 meaning none."""
        sz, nz = C.c_int(), C.c_int()
        call("lab_csrilu0" if kind == "ilu0" else "lab_csric0", self.h, C.byref(sz), C.byref(nz),
             stream_handle())
        return sz.value, nz.value

    def triangle(self, upper=False):
        """The lower (columns <= i) or upper triangle, diagonal included."""
        return self._new("lab_csr_triangle", self.h, int(bool(upper)))

    def scale_diagonal(self, scalar):
        call("lab_csr_scale_diagonal", self.h, C.c_double(scalar), stream_handle())

    def scale_by_inverse_diagonal(self):
        call("lab_csr_scale_by_inverse_diagonal", self.h, stream_handle())

    def spgemm(self, B):
        return self._new("lab_spgemm", self.h, B.h)

    def spgeam(self, alpha, beta, B):
        return self._new("lab_spgeam", alpha, self.h, beta, B.h)


# ---------------------------------------------------------------- BLAS-1
def dot(x, y):
    r = C.c_double()
    call("lab_dot", x.numel(), ptr(x), ptr(y), C.byref(r), stream_handle())
    return r.value


def norm_inf(x):
    r = C.c_double()
    call("lab_norm_inf", x.numel(), ptr(x), C.byref(r), stream_handle())
    return r.value


def norm_euclid(x):
    r = C.c_double()
    call("lab_norm_euclid", x.numel(), ptr(x), C.byref(r), stream_handle())
    return r.value


def axpy(alpha, x, y):
    call("lab_axpy", x.numel(), alpha, ptr(x), ptr(y), stream_handle())


def axpby(alpha, x, beta, y):
    call("lab_axpby", x.numel(), alpha, ptr(x), beta, ptr(y), stream_handle())


def axpbypgz(alpha, x, beta, y, gamma, z):
    call("lab_axpbypgz", x.numel(), alpha, ptr(x), beta, ptr(y), gamma, ptr(z), stream_handle())


def exclusive_scan(x):
    """In-place exclusive scan of an int32/int64 CUDA tensor."""
    fn = "lab_exclusive_scan_i64" if x.dtype == torch.int64 else "lab_exclusive_scan_i32"
    call(fn, x.numel(), ptr(x), stream_handle())
    return x


def launch_count():
    return lib().lab_launch_count()


# ---------------------------------------------------------------- options
def amg_options(n1=1, n2=1, cycle=L.CYCLE_V, smoother=L.SMOOTH_JACOBI, omega=1.0,
                omega_sor=0.5, coarse=L.COARSE_DIRECT, precision=L.PREC_FP64):
    o = AmgOptions()
    lib().lab_amg_options_default(C.byref(o))
    o.n1, o.n2, o.cycle, o.smoother = n1, n2, cycle, smoother
    o.omega, o.omega_sor, o.coarse, o.precision = omega, omega_sor, coarse, precision
    return o


def iter_control(rel_tol=1e-6, abs_tol=1e-6, max_iter=1000, max_cycle=200):
    c = IterControl()
    c.rel_tol, c.abs_tol, c.max_iter, c.max_cycle = rel_tol, abs_tol, max_iter, max_cycle
    return c


# ---------------------------------------------------------------- AMG
class Hierarchy:
    def __init__(self, A: CsrMatrix | None, kind=L.AMG_SA, max_level=20, stream=None):
        init()
        self.h = C.c_void_p()
        if A is not None:
            call("lab_amg_setup", kind, A.h, max_level, C.byref(self.h), stream_handle(stream))

    @classmethod
    def load(cls, path, stream=None):
        """A hierarchy written by save(), back on the device."""
        H = cls(None)
        call("lab_hierarchy_load", str(path).encode(), C.byref(H.h), stream_handle(stream))
        return H

    def autotune(self, exact=False):
        call("lab_hierarchy_autotune", self.h, int(bool(exact)), stream_handle())

    def save(self, path, stream=None):
        call("lab_hierarchy_save", self.h, str(path).encode(), stream_handle(stream))

    def __del__(self):
        try:
            if self.h:
                lib().lab_hierarchy_destroy(self.h)
                self.h = C.c_void_p()
        except Exception:
            pass

    @property
    def levels(self):
        n = C.c_int()
        call("lab_hierarchy_levels", self.h, C.byref(n))
        return n.value

    def setup_ms(self):
        d = C.c_double()
        call("lab_hierarchy_setup_ms", self.h, C.byref(d))
        return d.value

    def _level(self, l, which):
        hs = [C.c_void_p(), C.c_void_p(), C.c_void_p()]
        args = [C.byref(hs[k]) if k == which else None for k in range(3)]
        call("lab_hierarchy_level", self.h, l, *args)
        return CsrMatrix(hs[which], owner=False, keep=self)

    def A(self, l):
        return self._level(l, 0)

    def P(self, l):
        return self._level(l, 1)

    def R(self, l):
        return self._level(l, 2)

    def cycle(self, b, x=None, options=None):
        options = options or amg_options()
        if x is None:
            x = torch.zeros_like(b)
        call("lab_amg_cycle", self.h, C.byref(options), ptr(b), ptr(x), stream_handle())
        return x

    def solve(self, b, x=None, options=None, control=None):
        options = options or amg_options()
        control = control or iter_control()
        if x is None:
            x = torch.zeros_like(b)
        info = SolveInfo()
        call_solve("lab_amg_solve", self.h, C.byref(options), ptr(b), ptr(x), C.byref(control),
                   C.byref(info), stream_handle())
        return x, info


class Preconditioner:
    def __init__(self, h, keep=None):
        self.h = h
        self._keep = keep

    @classmethod
    def amg(cls, hier: Hierarchy, options=None):
        options = options or amg_options()
        h = C.c_void_p()
        call("lab_precond_create_amg", hier.h, C.byref(options), C.byref(h), stream_handle())
        return cls(h, keep=hier)

    @classmethod
    def jacobi(cls, A: CsrMatrix):
        h = C.c_void_p()
        call("lab_precond_create_jacobi", A.h, C.byref(h), stream_handle())
        return cls(h, keep=A)

    @classmethod
    def _tri(cls, fn, A, *extra):
        h = C.c_void_p()
        call(fn, A.h, *extra, C.byref(h), stream_handle())
        return cls(h, keep=A)

    @classmethod
    def ilu0(cls, A: CsrMatrix):
        return cls._tri("lab_precond_create_ilu0", A)

    @classmethod
    def ic0(cls, A: CsrMatrix):
        return cls._tri("lab_precond_create_ic0", A)

    @classmethod
    def gauss_seidel(cls, A: CsrMatrix):
        return cls._tri("lab_precond_create_gauss_seidel", A)

    @classmethod
    def sor(cls, A: CsrMatrix, omega: float):
        return cls._tri("lab_precond_create_sor", A, C.c_double(omega))

    @classmethod
    def ssor(cls, A: CsrMatrix, omega: float):
        return cls._tri("lab_precond_create_ssor", A, C.c_double(omega))

    def apply(self, r, z=None):
        if z is None:
            z = torch.empty_like(r)
        call("lab_precond_apply", self.h, ptr(r), ptr(z), stream_handle())
        return z

    def __del__(self):
        try:
            if self.h:
                lib().lab_precond_destroy(self.h)
                self.h = C.c_void_p()
        except Exception:
            pass


def pcg(A: CsrMatrix, b, x=None, M: Preconditioner | None = None, control=None):
    control = control or iter_control()
    if x is None:
        x = torch.zeros_like(b)
    info = SolveInfo()
    call_solve("lab_pcg_solve", A.h, M.h if M is not None else None, ptr(b), ptr(x),
               C.byref(control), C.byref(info), stream_handle())
    return x, info


def pcg_host(A: CsrMatrix, b: np.ndarray, x: np.ndarray, M=None, control=None):
    """PCG with host (numpy) b and x: the copies happen inside the call."""
    control = control or iter_control()
    info = SolveInfo()
    call_solve("lab_pcg_solve_host", A.h, M.h if M is not None else None, ptr(b), ptr(x),
               C.byref(control), C.byref(info), stream_handle())
    return x, info


def gmres(A: CsrMatrix, b, x=None, M: Preconditioner | None = None, restart=30, control=None):
    control = control or iter_control()
    if x is None:
        x = torch.zeros_like(b)
    info = SolveInfo()
    call_solve("lab_gmres_solve", A.h, M.h if M is not None else None, restart, ptr(b), ptr(x),
               C.byref(control), C.byref(info), stream_handle())
    return x, info


def adjoint_solve(A: CsrMatrix, g, M: Preconditioner | None = None, symmetric=True,
                  control=None, lam=None):
    """lambda = A^{-T} g (= dL/db for g = dL/dx)."""
    control = control or iter_control()
    if lam is None:
        lam = torch.zeros_like(g)
    info = SolveInfo()
    call_solve("lab_adjoint_solve", A.h, M.h if M is not None else None, int(bool(symmetric)),
               ptr(g), ptr(lam), C.byref(control), C.byref(info), stream_handle())
    return lam, info


def adjoint_grad_A(A: CsrMatrix, lam, x):
    """dL/dA on A's pattern: grad[j] = -lam[i] * x[col[j]]."""
    grad = torch.empty(A.nnz, dtype=torch.float64, device="cuda")
    call("lab_adjoint_grad_A", A.h, ptr(lam), ptr(x), ptr(grad), stream_handle())
    return grad


# ---------------------------------------------------------------- batching
def block_diag(blocks):
    """Stack CsrMatrix blocks block-diagonally; returns (matrix, offsets)."""
    arr = (C.c_void_p * len(blocks))(*[b.h.value for b in blocks])
    offs = (C.c_int64 * (len(blocks) + 1))()
    h = C.c_void_p()
    call("lab_csr_block_diag", arr, len(blocks), C.byref(h), offs, stream_handle())
    return CsrMatrix(h), np.array(offs[:], dtype=np.int64)


def batched_pcg(A: CsrMatrix, offsets, b, M: Preconditioner, x=None, control=None):
    """Independent systems stacked in A (rows offsets[k]:offsets[k+1])."""
    control = control or iter_control()
    if x is None:
        x = torch.zeros_like(b)
    nsys = len(offsets) - 1
    offs = (C.c_int64 * (nsys + 1))(*[int(o) for o in offsets])
    iters = (C.c_int * nsys)()
    conv = (C.c_int * nsys)()
    info = SolveInfo()
    call_solve("lab_batched_pcg_solve", A.h, M.h, nsys, offs, ptr(b), ptr(x), C.byref(control),
               iters, conv, C.byref(info), stream_handle())
    return x, np.array(iters[:]), np.array(conv[:]), info


def multi_rhs_pcg(A: CsrMatrix, B, M: Preconditioner, X=None, control=None):
    """B: (nrhs, n) tensor (row k = right-hand side k, i.e. column-major n x nrhs)."""
    control = control or iter_control()
    if X is None:
        X = torch.zeros_like(B)
    k = B.shape[0]
    iters = (C.c_int * k)()
    conv = (C.c_int * k)()
    info = SolveInfo()
    call_solve("lab_multi_rhs_pcg_solve", A.h, M.h, k, ptr(B), ptr(X), C.byref(control), iters,
               conv, C.byref(info), stream_handle())
    return X, np.array(iters[:]), np.array(conv[:]), info
