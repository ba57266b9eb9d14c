"""CPU tests of the drop-in boundary: the C-ABI library loads and exports every
symbol include/lab.h declares, the C++ API library exports the reference's
linalg:: entry points, and host-side argument handling needs no GPU."""
import ctypes
import os
import subprocess

import pytest

from linalglib_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_declared_symbol():
    lib = L.lib()
    declared = L.declared_symbols()
    assert len(declared) > 50
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing


def test_status_strings_and_defaults_without_device():
    lib = L.lib()
    assert lib.lab_status_string(L.LAB_NAN).decode() == "NaN in residual"
    o = L.AmgOptions()
    lib.lab_amg_options_default(ctypes.byref(o))
    assert (o.n1, o.n2, o.cycle, o.smoother, o.omega, o.omega_sor) == (1, 1, 0, 0, 1.0, 0.5)
    c = L.IterControl()
    lib.lab_iter_control_default(ctypes.byref(c))
    # iter_control.h:52-78
    assert (c.rel_tol, c.abs_tol, c.max_iter, c.max_cycle) == (1e-6, 1e-6, 1000, 200)


def test_null_arguments_rejected_without_device():
    lib = L.lib()
    assert lib.lab_spmv(1.0, None, None, 0.0, None, None) == L.LAB_BAD_ARG
    assert lib.lab_amg_setup(0, None, 20, None, None) == L.LAB_BAD_ARG
    assert lib.lab_pcg_solve(None, None, None, None, None, None, None) == L.LAB_BAD_ARG


def test_no_device_is_an_error_not_a_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("device present")
    lib = L.lib()
    h = ctypes.c_void_p()
    rp = (ctypes.c_int32 * 2)(0, 1)
    ci = (ctypes.c_int32 * 1)(0)
    v = (ctypes.c_double * 1)(2.0)
    st = lib.lab_csr_create(ctypes.byref(h), 1, 1, 1, rp, ci, v, L.MEM_HOST, None)
    assert st == L.LAB_NO_DEVICE


def test_cxx_api_symbols():
    """The C++ layer exports the reference's public functions (namespace linalg)."""
    so = os.path.join(ROOT, "linalglib_b200", "liblinalg_b200.so")
    out = subprocess.run(["nm", "-D", "--defined-only", "-C", so], capture_output=True,
                         text=True).stdout
    for sym in ["linalg::saamg_setup(", "linalg::uaamg_setup(", "linalg::rsamg_setup(",
                "linalg::amg_solve(", "linalg::cg_solver::solve(", "linalg::gmres_solver::solve(",
                "linalg::csr_matrix<double>::multiply_by_vector(",
                "linalg::csr_matrix<double>::multiply_by_matrix(",
                "linalg::csr_matrix<double>::transpose(", "linalg::compute_residual(",
                "linalg::dot_product(", "linalg::norm_inf(", "linalg::amg_precond::solve("]:
        assert sym in out, sym
