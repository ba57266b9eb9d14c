// The reference's triangular-solve preconditioners and free functions
// (preconditioner.h: ilu_precond, ic_precond, gauss_seidel_precond, SOR_precond,
// SSOR_precond;
// linalg_math.h: csrilu0, csrtrsv_*) through this library's C++ API.
// Usage: tri_precond_example <grid n>.  Prints one line
//   "<ilu cg iters> <converged> <gs gmres cycles> <sor gmres cycles> <gmres rel res>
//    <structural zero> <numeric zero> <ssor cg iters>"
// then the ILU(0) factor values and the unit-lower solve of ones, one hex float
// per line, for a bit-for-bit comparison.
#include "linalg.h"

#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

using namespace linalg;

static void poisson2d(int n, std::vector<int>& rp, std::vector<int>& ci, std::vector<double>& v)
{
    rp.assign(1, 0);
    for(int i = 0; i < n * n; i++)
    {
        int x = i % n, y = i / n;
        if(y > 0)
            ci.push_back(i - n), v.push_back(-1.0);
        if(x > 0)
            ci.push_back(i - 1), v.push_back(-1.0);
        ci.push_back(i), v.push_back(4.0);
        if(x < n - 1)
            ci.push_back(i + 1), v.push_back(-1.0);
        if(y < n - 1)
            ci.push_back(i + n), v.push_back(-1.0);
        rp.push_back((int)ci.size());
    }
}

int main(int argc, char** argv)
{
    int                 n = argc > 1 ? std::atoi(argv[1]) : 24;
    std::vector<int>    rp, ci;
    std::vector<double> v;
    poisson2d(n, rp, ci, v);
    int                m = n * n;
    csr_matrix<double> A(rp, ci, v, m, m, (int)v.size());

    vector<double> e(m), b(m), x(m);
    e.ones();
    A.multiply_by_vector(b, e);

    // ILU(0)-preconditioned CG (the reference's pcg_example with ilu_precond)
    iter_control control;
    control.rel_tol  = 1e-8;
    control.abs_tol  = 1e-300;
    control.max_iter = 1000;
    ilu_precond ilu;
    ilu.build(A);
    cg_solver cg;
    cg.build(A);
    x.zeros();
    int iters = cg.solve(A, x, b, &ilu, control);
    int conv  = cg.last_info().converged;

    // SSOR(1.3)-preconditioned CG
    SSOR_precond ssor(1.3);
    ssor.build(A);
    x.zeros();
    int ssor_iters = cg.solve(A, x, b, &ssor, control);
    conv           = conv && cg.last_info().converged;

    // Gauss-Seidel and SOR under restarted GMRES
    gmres_solver gm;
    gm.build(A, 20);
    gauss_seidel_precond gs;
    gs.build(A);
    x.zeros();
    control.rel_tol = 1e-10;
    int gs_cycles   = gm.solve(A, x, b, &gs, control);
    SOR_precond sor(1.3);
    sor.build(A);
    x.zeros();
    int            sor_cycles = gm.solve(A, x, b, &sor, control);
    vector<double> r(m);
    compute_residual(A, x, b, r);
    double rel = norm_inf(r) / norm_inf(b);

    // the free functions: in-place ILU(0) of a copy, then a unit-lower solve
    csr_matrix<double> LU;
    LU.copy_from(A);
    int sz = INT_MAX, nz = INT_MAX;
    csrilu0(LU, &sz, &nz);
    csrtrsv_descr* d = nullptr;
    create_csrtrsv_descr(&d);
    csrtrsv_analysis(LU, triangular_type::lower, diagonal_type::unit, d);
    vector<double> y(m);
    csrtrsv_solve(LU, e, y, 1.0, triangular_type::lower, diagonal_type::unit, d);
    destroy_csrtrsv_descr(d);

    std::printf("%d %d %d %d %.3e %d %d %d\n", iters, conv, gs_cycles, sor_cycles, rel,
                sz == INT_MAX ? -1 : sz, nz == INT_MAX ? -1 : nz, ssor_iters);
    const double* lv = LU.get_val();
    for(int j = 0; j < LU.get_nnz(); j++)
        std::printf("%a\n", lv[j]);
    for(int i = 0; i < m; i++)
        std::printf("%a\n", y[i]);
    return conv ? 0 : 1;
}
