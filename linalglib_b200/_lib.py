"""ctypes binding of the liblinalg_b200 C ABI (include/lab.h).

The shared library is built in-tree (``python -m linalglib_b200.build``); there is
no CPU implementation behind these entry points: without the library or a
usable device every call raises ``LabError``.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblinalg_b200.so")

LAB_OK, LAB_NOT_CONVERGED, LAB_BREAKDOWN, LAB_NAN, LAB_BAD_ARG, LAB_OOM, LAB_TIMEOUT, \
    LAB_CUDA_ERROR, LAB_NOT_SUPPORTED, LAB_NO_DEVICE = range(10)
MEM_HOST, MEM_DEVICE = 0, 1
AMG_SA, AMG_UA, AMG_RS = 0, 1, 2
CYCLE_V, CYCLE_W, CYCLE_F = 0, 1, 2
SMOOTH_JACOBI, SMOOTH_GS, SMOOTH_SGS, SMOOTH_SOR, SMOOTH_SSOR = range(5)
COARSE_DIRECT, COARSE_GS = 0, 1
PREC_FP64, PREC_FP32, PREC_FP32_BF16 = 0, 1, 2
SPMV_AUTO, SPMV_ROWSEQ, SPMV_VECTOR, SPMV_MERGE, SPMV_VECTOR_STREAM, SPMV_VECTOR_HALO = (
    0, 1, 2, 3, 4, 5)


class LabError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{msg} (status {status})")
        self.status = status


class AmgOptions(C.Structure):
    _fields_ = [("n1", C.c_int), ("n2", C.c_int), ("cycle", C.c_int), ("smoother", C.c_int),
                ("omega", C.c_double), ("omega_sor", C.c_double), ("coarse", C.c_int),
                ("precision", C.c_int)]


class IterControl(C.Structure):
    _fields_ = [("rel_tol", C.c_double), ("abs_tol", C.c_double), ("max_iter", C.c_int),
                ("max_cycle", C.c_int)]


class SolveInfo(C.Structure):
    _fields_ = [("iterations", C.c_int), ("converged", C.c_int),
                ("initial_residual", C.c_double), ("final_residual", C.c_double),
                ("solve_ms", C.c_double), ("status", C.c_int)]


_p = C.c_void_p
_i64 = C.c_int64
_d = C.c_double
_i = C.c_int

# name: (restype is lab_status unless given, argtypes)
_SIGS = {
    "lab_init": [_i],
    "lab_synchronize": [_p],
    "lab_malloc": [C.POINTER(_p), C.c_size_t, _p],
    "lab_free": [_p, _p],
    "lab_memcpy": [_p, _p, C.c_size_t, _p],
    "lab_wait_timeouts": [C.POINTER(_i64), _p],
    "lab_csr_create": [C.POINTER(_p), _i64, _i64, _i64, _p, _p, _p, _i, _p],
    "lab_csr_create_empty": [C.POINTER(_p), _i64, _i64, _i64, _p],
    "lab_csr_destroy": [_p],
    "lab_csr_info": [_p, C.POINTER(_i64), C.POINTER(_i64), C.POINTER(_i64)],
    "lab_csr_device_arrays": [_p, C.POINTER(_p), C.POINTER(_p), C.POINTER(_p)],
    "lab_csr_copy_to": [_p, _p, _p, _p, _i, _p],
    "lab_csr_clone": [_p, C.POINTER(_p), _p],
    "lab_csr_values_changed": [_p, _p],
    "lab_csr_structure_changed": [_p, _p],
    "lab_spmv_analysis": [_p, _p],
    "lab_spmv_set_algorithm": [_p, _i, _i],
    "lab_spmv_get_algorithm": [_p, C.POINTER(_i), C.POINTER(_i)],
    "lab_spmv_halo_info": [_p, C.POINTER(_i64), C.POINTER(_i64), C.POINTER(_i64),
                           C.POINTER(_i64)],
    "lab_spmv": [_d, _p, _p, _d, _p, _p],
    "lab_residual": [_p, _p, _p, _p, _p],
    "lab_spmm": [_d, _p, _i, _p, _i64, _d, _p, _i64, _p],
    "lab_axpy": [_i64, _d, _p, _p, _p],
    "lab_axpby": [_i64, _d, _p, _d, _p, _p],
    "lab_axpbypgz": [_i64, _d, _p, _d, _p, _d, _p, _p],
    "lab_dot": [_i64, _p, _p, C.POINTER(_d), _p],
    "lab_norm_inf": [_i64, _p, C.POINTER(_d), _p],
    "lab_norm_euclid": [_i64, _p, C.POINTER(_d), _p],
    "lab_fill": [_i64, _d, _p, _p],
    "lab_diagonal": [_p, _p, _p],
    "lab_jacobi_solve": [_i64, _p, _p, _p, _p],
    "lab_exclusive_scan_i64": [_i64, _p, _p],
    "lab_exclusive_scan_i32": [_i64, _p, _p],
    "lab_exclusive_scan_i64_noalloc": [_i64, _p, _p],
    "lab_spgemm": [_p, _p, C.POINTER(_p), _p],
    "lab_spgeam": [_d, _p, _d, _p, C.POINTER(_p), _p],
    "lab_transpose": [_p, C.POINTER(_p), _p],
    "lab_strength": [_p, _d, _p, _p],
    "lab_classical_strength": [_p, _d, _p, C.POINTER(_p), _p],
    "lab_pmis_aggregate": [_p, _p, _p, C.POINTER(_i), _p],
    "lab_sa_prolongation": [_p, _p, _p, _d, C.POINTER(_p), _p],
    "lab_ua_prolongation": [_p, _p, C.POINTER(_p), _p],
    "lab_cfpoints": [_p, _p, _p],
    "lab_direct_interpolation": [_p, _p, _p, C.POINTER(_p), _p],
    "lab_amg_setup": [_i, _p, _i, C.POINTER(_p), _p],
    "lab_hierarchy_destroy": [_p],
    "lab_hierarchy_levels": [_p, C.POINTER(_i)],
    "lab_hierarchy_level": [_p, _i, C.POINTER(_p), C.POINTER(_p), C.POINTER(_p)],
    "lab_hierarchy_setup_ms": [_p, C.POINTER(_d)],
    "lab_csrtrsv": [_p, _i, _i, _p, _p, _p],
    "lab_csrtrsv_analysis": [_p, _p],
    "lab_mtx_read": [_p, C.POINTER(_i64), C.POINTER(_i64), C.POINTER(_i64), C.POINTER(_p),
                     C.POINTER(_p), C.POINTER(_p)],
    "lab_mtx_write": [_p, _i64, _i64, _i64, _p, _p, _p],
    "lab_batch_partition": [_i, _p, _i, _p],
    "lab_csrtrsv_wait_control": [_p, _i64, _i64, _p],
    "lab_csr_triangle": [_p, _i, C.POINTER(_p), _p],
    "lab_csr_scale_diagonal": [_p, _d, _p],
    "lab_csr_scale_by_inverse_diagonal": [_p, _p],
    "lab_csrilu0": [_p, C.POINTER(_i), C.POINTER(_i), _p],
    "lab_csric0": [_p, C.POINTER(_i), C.POINTER(_i), _p],
    "lab_precond_create_ilu0": [_p, C.POINTER(_p), _p],
    "lab_precond_create_ic0": [_p, C.POINTER(_p), _p],
    "lab_precond_create_gauss_seidel": [_p, C.POINTER(_p), _p],
    "lab_precond_create_sor": [_p, _d, C.POINTER(_p), _p],
    "lab_precond_create_ssor": [_p, _d, C.POINTER(_p), _p],
    "lab_spmv_autotune": [_p, _i, C.POINTER(_d), _p],
    "lab_hierarchy_autotune": [_p, _i, _p],
    "lab_spgemm_autotune": [_p, _p, C.POINTER(_d), _p],
    "lab_hierarchy_tune_products": [_p, _p],
    "lab_tune_cache_save": [C.c_char_p],
    "lab_tune_cache_load": [C.c_char_p],
    "lab_tune_cache_clear": [],
    "lab_hierarchy_save": [_p, C.c_char_p, _p],
    "lab_hierarchy_load": [C.c_char_p, C.POINTER(_p), _p],
    "lab_amg_cycle": [_p, C.POINTER(AmgOptions), _p, _p, _p],
    "lab_amg_solve": [_p, C.POINTER(AmgOptions), _p, _p, C.POINTER(IterControl),
                      C.POINTER(SolveInfo), _p],
    "lab_precond_create_amg": [_p, C.POINTER(AmgOptions), C.POINTER(_p), _p],
    "lab_precond_create_jacobi": [_p, C.POINTER(_p), _p],
    "lab_precond_apply": [_p, _p, _p, _p],
    "lab_precond_destroy": [_p],
    "lab_pcg_solve": [_p, _p, _p, _p, C.POINTER(IterControl), C.POINTER(SolveInfo), _p],
    "lab_pcg_solve_host": [_p, _p, _p, _p, C.POINTER(IterControl), C.POINTER(SolveInfo), _p],
    "lab_gmres_solve": [_p, _p, _i, _p, _p, C.POINTER(IterControl), C.POINTER(SolveInfo), _p],
    "lab_adjoint_solve": [_p, _p, _i, _p, _p, C.POINTER(IterControl), C.POINTER(SolveInfo), _p],
    "lab_adjoint_grad_A": [_p, _p, _p, _p, _p],
    "lab_pmis_aggregate_roots": [_p, _p, _p, _p, C.POINTER(_i), _p],
    "lab_cfpoints_passes": [_p, _p, _i, _i, _p],
    "lab_csr_block_diag": [_p, _i, C.POINTER(_p), _p, _p],
    "lab_batched_pcg_solve": [_p, _p, _i, _p, _p, _p, C.POINTER(IterControl), _p, _p,
                              C.POINTER(SolveInfo), _p],
    "lab_multi_rhs_pcg_solve": [_p, _p, _i, _p, _p, C.POINTER(IterControl), _p, _p,
                                C.POINTER(SolveInfo), _p],
}

_lib = None


def lib():
    """Load liblinalg_b200.so (raises LabError if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise LabError(LAB_NO_DEVICE, f"{LIB_PATH} is not built; run python -m linalglib_b200.build")
    L = C.CDLL(LIB_PATH)
    for name, args in _SIGS.items():
        fn = getattr(L, name, None)
        if fn is None:
            continue
        fn.argtypes = args
        fn.restype = C.c_int
    L.lab_status_string.restype = C.c_char_p
    L.lab_status_string.argtypes = [_i]
    L.lab_last_error.restype = C.c_char_p
    L.lab_last_error.argtypes = []
    L.lab_launch_count.restype = C.c_int64
    L.lab_launch_count.argtypes = []
    L.lab_amg_options_default.restype = None
    L.lab_amg_options_default.argtypes = [C.POINTER(AmgOptions)]
    L.lab_iter_control_default.restype = None
    L.lab_iter_control_default.argtypes = [C.POINTER(IterControl)]
    L.lab_mtx_free.restype = None
    L.lab_mtx_free.argtypes = [_p]
    _lib = L
    return L


def check(status, what="call"):
    """Raise LabError for any status other than LAB_OK / LAB_NOT_CONVERGED."""
    if status in (LAB_OK, LAB_NOT_CONVERGED):
        return status
    L = lib()
    raise LabError(status, f"{what}: {L.lab_status_string(status).decode()}: "
                           f"{L.lab_last_error().decode()}")


def call(name, *args):
    return check(getattr(lib(), name)(*args), name)


def call_solve(name, *args):
    """Like call(), for solvers: a NaN/Inf residual or a breakdown is an outcome
    reported in the solve info, not an exception."""
    st = getattr(lib(), name)(*args)
    if st in (LAB_NAN, LAB_BREAKDOWN):
        return st
    return check(st, name)


def mtx_read(path):
    """lab_mtx_read on the host: (row_ptr, col_ind, val, n) numpy arrays."""
    L = lib()
    m, n, z = C.c_int64(), C.c_int64(), C.c_int64()
    rp, ci, v = C.c_void_p(), C.c_void_p(), C.c_void_p()
    call("lab_mtx_read", str(path).encode(), C.byref(m), C.byref(n), C.byref(z), C.byref(rp),
         C.byref(ci), C.byref(v))
    try:
        import numpy as np
        a = np.ctypeslib.as_array(C.cast(rp, C.POINTER(C.c_int32)), shape=(m.value + 1,)).copy()
        b = np.ctypeslib.as_array(C.cast(ci, C.POINTER(C.c_int32)), shape=(max(z.value, 1),))
        c = np.ctypeslib.as_array(C.cast(v, C.POINTER(C.c_double)), shape=(max(z.value, 1),))
        return a, b[:z.value].copy(), c[:z.value].copy(), n.value
    finally:
        for p in (rp, ci, v):
            L.lab_mtx_free(p)


def mtx_write(path, rp, ci, v, n=None):
    """lab_mtx_write of host CSR arrays."""
    import numpy as np
    rp = np.ascontiguousarray(rp, dtype=np.int32)
    ci = np.ascontiguousarray(ci, dtype=np.int32)
    v = np.ascontiguousarray(v, dtype=np.float64)
    m = rp.size - 1
    call("lab_mtx_write", str(path).encode(), m, m if n is None else n, int(rp[-1]),
         rp.ctypes.data, ci.ctypes.data, v.ctypes.data)


def declared_symbols(header_path=None):
    """Names of the functions include/lab.h declares (for export checks)."""
    import re
    header_path = header_path or os.path.join(os.path.dirname(HERE), "include", "lab.h")
    text = open(header_path).read()
    return sorted(set(re.findall(r"LAB_API\s+[\w\s\*]+?\b(lab_\w+)\s*\(", text)))
