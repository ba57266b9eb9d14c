// csr_matrix members and descriptor calls a reference client uses, through this
// library's C++ API: read_mtx / write_mtx, copy_lower_triangular_from /
// copy_upper_triangular_from, scale_diagonal_by, scale_by_inverse_diagonal,
// triangular_solve_lower / triangular_solve_upper, the in-place IC(0) / ILU(0)
// members and the csric0 / csrilu0 descriptor form.
// Usage: matrix_members_example <in.mtx> <out dir>.  Writes lower.mtx, upper.mtx,
// diag.mtx, invdiag.mtx, ic0.mtx, ilu0.mtx, ic0_descr.mtx and ilu0_descr.mtx into
// <out dir>, then prints the lower and upper solves of a vector of ones on A,
// one hex float per line (lower first).
#include "linalg.h"

#include <cstdio>
#include <string>

using namespace linalg;

static bool save(csr_matrix<double>& M, const std::string& dir, const char* name)
{
    return M.write_mtx(dir + "/" + name);
}

int main(int argc, char** argv)
{
    if(argc < 3)
        return 2;
    const std::string  dir = argv[2];
    csr_matrix<double> A;
    if(!A.read_mtx(argv[1]))
        return 3;

    csr_matrix<double> L, U;
    L.copy_lower_triangular_from(A, false);
    U.copy_upper_triangular_from(A, false);
    if(!save(L, dir, "lower.mtx") || !save(U, dir, "upper.mtx"))
        return 4;

    csr_matrix<double> D;
    D.copy_from(A);
    D.scale_diagonal_by(2.5);
    csr_matrix<double> I;
    I.copy_from(A);
    I.scale_by_inverse_diagonal();
    if(!save(D, dir, "diag.mtx") || !save(I, dir, "invdiag.mtx"))
        return 5;

    csr_matrix<double> C, F;
    C.copy_from(A);
    C.compute_incomplete_cholesky_factorization();
    F.copy_from(A);
    F.compute_incomplete_LU_factorization();
    if(!save(C, dir, "ic0.mtx") || !save(F, dir, "ilu0.mtx"))
        return 6;

    csr_matrix<double> C2, F2;
    C2.copy_from(A);
    F2.copy_from(A);
    csric0_descr*  dc = nullptr;
    csrilu0_descr* df = nullptr;
    create_csric0_descr(&dc);
    create_csrilu0_descr(&df);
    csric0_analysis(C2, dc);
    csric0_compute(C2, dc);
    csrilu0_analysis(F2, df);
    csrilu0_compute(F2, df);
    destroy_csric0_descr(dc);
    destroy_csrilu0_descr(df);
    if(!save(C2, dir, "ic0_descr.mtx") || !save(F2, dir, "ilu0_descr.mtx"))
        return 7;

    const int      m = A.get_m();
    vector<double> y(m), xl(m), xu(m);
    y.ones();
    A.triangular_solve_lower(xl, y, false);
    A.triangular_solve_upper(xu, y, false);
    for(int i = 0; i < m; i++)
        std::printf("%a\n", xl[i]);
    for(int i = 0; i < m; i++)
        std::printf("%a\n", xu[i]);
    return 0;
}
