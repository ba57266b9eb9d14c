// Free functions of the reference's op front-end (library/include/linalg_math.h:52-520)
// on the AMG-PCG path.  Each runs on the GPU through the C ABI (lab.h).
#ifndef LINALG_B200_MATH_H
#define LINALG_B200_MATH_H

#include "csr_matrix.h"
#include "vector.h"

namespace linalg
{
    // linalg_math.h:52, 63, 76
    void axpy(double alpha, const vector<double>& x, vector<double>& y);
    void axpby(double alpha, const vector<double>& x, double beta, vector<double>& y);
    void axpbypgz(double alpha, const vector<double>& x, double beta, const vector<double>& y,
                  double gamma, vector<double>& z);
    // linalg_math.h:119
    void transpose_matrix(const csr_matrix<double>& A, csr_matrix<double>& transposeA);
    // linalg_math.h:132-175
    double dot_product(const vector<double>& x, const vector<double>& y);
    void   compute_residual(const csr_matrix<double>& A, const vector<double>& x,
                            const vector<double>& b, vector<double>& res);
    void   diagonal(const csr_matrix<double>& A, vector<double>& d);
    double norm_euclid(const vector<double>& array);
    double norm_inf(const vector<double>& array);

    // In-place incomplete factorizations (linalg_math.h:95, 109; host_csric0.cpp,
    // host_csrilu0.cpp), computed on the GPU bit-identically to the reference's
    // host loops.  As there, the column of a missing (structural) or zero
    // (numeric) pivot is folded into *structural_zero / *numeric_zero with
    // std::min, so callers initialise them (e.g. to INT_MAX); null is allowed.
    void csric0(csr_matrix<double>& LL, int* structural_zero, int* numeric_zero);
    void csrilu0(csr_matrix<double>& LU, int* structural_zero, int* numeric_zero);

    // Descriptor form of the same factorizations (linalg_math.h:447-520): the
    // analysis builds the dependency levels of A's pattern (kept with the matrix),
    // the compute step factors A in place.
    struct csric0_descr;
    struct csrilu0_descr;
    void create_csric0_descr(csric0_descr** descr);
    void destroy_csric0_descr(csric0_descr* descr);
    void csric0_analysis(const csr_matrix<double>& A, csric0_descr* descr);
    void csric0_compute(csr_matrix<double>& A, const csric0_descr* descr);
    void create_csrilu0_descr(csrilu0_descr** descr);
    void destroy_csrilu0_descr(csrilu0_descr* descr);
    void csrilu0_analysis(const csr_matrix<double>& A, csrilu0_descr* descr);
    void csrilu0_compute(csr_matrix<double>& A, const csrilu0_descr* descr);

    // Sparse triangular solve on the lower or upper part of A (linalg_math.h:
    // 198-254, linalg_enums.h:37-48).  The analysis builds the level schedule of
    // A's pattern (cached on the matrix); x = T^-1 (alpha b).
    enum class triangular_type
    {
        lower,
        upper
    };
    enum class diagonal_type
    {
        non_unit,
        unit
    };
    struct csrtrsv_descr;
    void create_csrtrsv_descr(csrtrsv_descr** descr);
    void destroy_csrtrsv_descr(csrtrsv_descr* descr);
    void csrtrsv_analysis(const csr_matrix<double>& A, triangular_type tri_type,
                          diagonal_type diag_type, csrtrsv_descr* descr);
    void csrtrsv_solve(const csr_matrix<double>& A, const vector<double>& b, vector<double>& x,
                       double alpha, triangular_type tri_type, diagonal_type diag_type,
                       const csrtrsv_descr* descr);

    // csrmv descriptor: a cached SpMV plan (linalg_math.h:263-310)
    enum class csrmv_algorithm
    {
        default_algorithm,
        merge_path,
        rowsplit,
        nnzsplit
    };
    struct csrmv_descr;
    void create_csrmv_descr(csrmv_descr** descr);
    void destroy_csrmv_descr(csrmv_descr* descr);
    void csrmv_analysis(const csr_matrix<double>& A, csrmv_algorithm alg, csrmv_descr* descr);
    void csrmv_solve(double alpha, const csr_matrix<double>& A, const vector<double>& x,
                     double beta, vector<double>& y, csrmv_algorithm alg,
                     const csrmv_descr* descr);

    // csrgeam / csrgemm (linalg_math.h:319-440)
    enum class csrgeam_algorithm
    {
        default_algorithm
    };
    enum class csrgemm_algorithm
    {
        default_algorithm
    };
    struct csrgeam_descr;
    struct csrgemm_descr;
    void create_csrgeam_descr(csrgeam_descr** descr);
    void destroy_csrgeam_descr(csrgeam_descr* descr);
    void csrgeam_nnz(const csr_matrix<double>& A, const csr_matrix<double>& B,
                     csr_matrix<double>& C, csrgeam_algorithm alg, csrgeam_descr* descr);
    void csrgeam_solve(double alpha, const csr_matrix<double>& A, double beta,
                       const csr_matrix<double>& B, csr_matrix<double>& C, csrgeam_algorithm alg,
                       const csrgeam_descr* descr);
    void create_csrgemm_descr(csrgemm_descr** descr);
    void destroy_csrgemm_descr(csrgemm_descr* descr);
    void csrgemm_nnz(const csr_matrix<double>& A, const csr_matrix<double>& B,
                     const csr_matrix<double>& D, csr_matrix<double>& C, csrgemm_algorithm alg,
                     csrgemm_descr* descr);
    void csrgemm_solve(double alpha, const csr_matrix<double>& A, const csr_matrix<double>& B,
                       double beta, const csr_matrix<double>& D, csr_matrix<double>& C,
                       csrgemm_algorithm alg, const csrgemm_descr* descr);

    // linalg_primitives.h:98
    template <typename T>
    void exclusive_scan(vector<T>& x);

    // linalg_memory.h
    bool is_device_available();
    void synchronize();
}

#endif
