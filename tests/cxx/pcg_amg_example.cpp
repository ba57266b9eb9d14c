// The reference's client pattern (clients/examples/saamg_example.cpp:33-67,
// clients/examples/pcg_example.cpp:33-74, clients/testing/test_functions_amg.cpp:35-139)
// written against this library's C++ API: unchanged user code, GPU underneath.
// Usage: pcg_amg_example <grid n> ; prints "levels iters converged max_err rel_res".
#include "linalg.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

using namespace linalg;

static void poisson2d(int n, std::vector<int>& rp, std::vector<int>& ci, std::vector<double>& v)
{
    int m = n * n;
    rp.assign(1, 0);
    for(int i = 0; i < m; i++)
    {
        int x = i % n, y = i / n;
        if(y > 0)
        {
            ci.push_back(i - n);
            v.push_back(-1.0);
        }
        if(x > 0)
        {
            ci.push_back(i - 1);
            v.push_back(-1.0);
        }
        ci.push_back(i);
        v.push_back(4.0);
        if(x < n - 1)
        {
            ci.push_back(i + 1);
            v.push_back(-1.0);
        }
        if(y < n - 1)
        {
            ci.push_back(i + n);
            v.push_back(-1.0);
        }
        rp.push_back((int)ci.size());
    }
}

int main(int argc, char** argv)
{
    int                 n = argc > 1 ? std::atoi(argv[1]) : 64;
    std::vector<int>    rp, ci;
    std::vector<double> v;
    poisson2d(n, rp, ci, v);
    int m = n * n;

    csr_matrix<double> A(rp, ci, v, m, m, (int)v.size());

    // b = A * e with e = 1 (test_functions_amg.cpp:63)
    vector<double> e(m);
    e.ones();
    vector<double> b(m);
    A.multiply_by_vector(b, e);
    vector<double> x(m);
    x.zeros();

    // 1) stationary SA-AMG (amg_solve), as the reference's AMG tests run it
    hierarchy h;
    saamg_setup(A, 100, h);
    iter_control control;
    control.rel_tol   = 1e-8;
    control.abs_tol   = 1e-300;
    control.max_cycle = 300;
    int cycles = amg_solve(h, x, b, 1, 1, cycle::vcycle, smoother::jacobi, control);
    double err1 = 0.0;
    for(int i = 0; i < m; i++)
        err1 = std::fmax(err1, std::fabs(x[i] - 1.0));

    // 2) SA-AMG preconditioned CG through the preconditioner plug-in point
    amg_precond M;
    M.attach(h);
    M.build(A);
    cg_solver cg;
    cg.build(A);
    vector<double> x2(m);
    x2.zeros();
    control.max_iter = 500;
    int iters = cg.solve(A, x2, b, &M, control);

    vector<double> r(m);
    compute_residual(A, x2, b, r);
    double rel = norm_inf(r) / norm_inf(b);
    double err2 = 0.0;
    for(int i = 0; i < m; i++)
        err2 = std::fmax(err2, std::fabs(x2[i] - 1.0));

    // 3) level structure is readable through the hierarchy arrays
    long nnz_total = 0;
    for(int l = 0; l <= h.total_levels; l++)
        nnz_total += h.A_cs[l].get_nnz();

    std::printf("%d %d %d %d %.3e %.3e %.3e %ld\n", h.total_levels, cycles, iters,
                cg.last_info().converged, err1, err2, rel, nnz_total);
    return (cg.last_info().converged && rel <= 1e-8) ? 0 : 1;
}
