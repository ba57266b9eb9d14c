// csrgemm through this library's C++ API, as a reference client calls it:
// create_csrgemm_descr, csrgemm_nnz, csrgemm_solve(alpha, A, B, beta, D, C),
// destroy_csrgemm_descr.
// Usage: csrgemm_example <A.mtx> <B.mtx> <D.mtx> <alpha> <beta>.
// Prints "m n nnz", then C's row pointers, columns and values (hex floats), one per
// line.
#include "linalg.h"

#include <cstdio>
#include <cstdlib>

using namespace linalg;

int main(int argc, char** argv)
{
    if(argc < 6)
        return 2;
    csr_matrix<double> A, B, D;
    if(!A.read_mtx(argv[1]) || !B.read_mtx(argv[2]) || !D.read_mtx(argv[3]))
        return 3;
    const double alpha = std::strtod(argv[4], nullptr);
    const double beta  = std::strtod(argv[5], nullptr);

    csr_matrix<double> C;
    csrgemm_descr*     d = nullptr;
    create_csrgemm_descr(&d);
    csrgemm_nnz(A, B, D, C, csrgemm_algorithm::default_algorithm, d);
    csrgemm_solve(alpha, A, B, beta, D, C, csrgemm_algorithm::default_algorithm, d);
    destroy_csrgemm_descr(d);

    const csr_matrix<double>& R   = C;
    const int                 m   = R.get_m();
    const int                 nnz = R.get_nnz();
    std::printf("%d %d %d\n", m, R.get_n(), nnz);
    const int*    rp = R.get_row_ptr();
    const int*    ci = R.get_col_ind();
    const double* v  = R.get_val();
    for(int i = 0; i <= m; i++)
        std::printf("%d\n", rp[i]);
    for(int j = 0; j < nnz; j++)
        std::printf("%d\n", ci[j]);
    for(int j = 0; j < nnz; j++)
        std::printf("%a\n", v[j]);
    return 0;
}
