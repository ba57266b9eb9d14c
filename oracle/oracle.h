/* Test infrastructure only: a CPU restatement, in plain C, of the reference
 * LinAlgLib algorithms on the AMG-PCG path.  It is the checker for the CUDA
 * library (tests, smoke test and the CPU-baseline arm of bench.py load it);
 * nothing in the product links or calls it.
 *
 * Pinning: every function here is compared in tests/test_oracle_vs_reference.py
 * against the reference itself, compiled from its own sources into
 * oracle/_ref/liblinalg_ref.so, and against the committed golden fixtures in
 * tests/golden/ that the reference produced (tests/golden/make_golden.py).
 *
 * Arithmetic follows the reference operation by operation (same evaluation
 * order, same association, fma only where the reference calls std::fma), and the
 * file is compiled with -ffp-contract=off, so integer outputs and the setup's
 * floating-point values are bit-identical to the reference's single-threaded
 * results.  Reductions (dot, norm) are sequential; the reference's OpenMP
 * reductions may round differently, which only moves PCG iterates by ulps.
 */
#ifndef LAB_ORACLE_H
#define LAB_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct
{
    int     m, n, nnz;
    int*    rp;
    int*    ci;
    double* v;
} orc_csr;

typedef struct
{
    int     levels; /* number of coarse levels built (reference hierarchy::total_levels) */
    orc_csr A[21];
    orc_csr P[20];
    orc_csr R[20];
    /* dense inverse of the coarsest operator (built on demand for ORC_COARSE_DIRECT) */
    double* coarse_inv;
    /* multicolour orderings of the levels (built on demand for ORC_SMOOTH_MC_*):
     * rows of colour c are mc_order[l][mc_ptr[l][c] .. mc_ptr[l][c+1]) */
    int* mc_order[21];
    int* mc_ptr[21];
    int  mc_ncol[21];
} orc_hier;

enum
{
    ORC_SA = 0,
    ORC_UA = 1,
    ORC_RS = 2
};
enum
{
    ORC_SMOOTH_JACOBI  = 0,
    ORC_SMOOTH_GS      = 1, /* the reference's lexicographic sweep */
    ORC_SMOOTH_MC_GS   = 2, /* the device's multicolour sweep, weight omega (GS, SGS: 1) */
    ORC_SMOOTH_MC_SSOR = 3  /* multicolour sweep forward then backward, weight omega */
};
enum
{
    ORC_COARSE_GS     = 0, /* 1000 lexicographic GS sweeps, as the reference */
    ORC_COARSE_DIRECT = 1  /* exact solve through a dense inverse */
};

void orc_csr_free(orc_csr* A);
int  orc_csr_alloc(orc_csr* A, int m, int n, int nnz);

/* kernels */
void orc_diag(const orc_csr* A, double* d);
void orc_spmv(const orc_csr* A, double alpha, const double* x, double beta, double* y);
void orc_residual(const orc_csr* A, const double* x, const double* b, double* r);
int  orc_transpose(const orc_csr* A, orc_csr* T);
int  orc_spgemm(const orc_csr* A, const orc_csr* B, orc_csr* C);
int  orc_spgeam(double alpha, const orc_csr* A, double beta, const orc_csr* B, orc_csr* C);
void orc_exclusive_scan_i64(int64_t* x, int n);
double orc_dot(const double* x, const double* y, int n);
double orc_norm_inf(const double* x, int n);

/* AMG setup pieces */
void orc_strength(const orc_csr* A, double eps, int* conn);
void orc_pmis(const orc_csr* A, const int* conn, int64_t* aggregates, int* rounds);
int  orc_sa_prolongation(const orc_csr* A, const int* conn, const int64_t* aggregates,
                         double relax, orc_csr* P);
int  orc_ua_prolongation(const orc_csr* A, const int64_t* aggregates, orc_csr* P);
int  orc_classical_strength(const orc_csr* A, double theta, int* conn, orc_csr* S);
void orc_cfpoints(const orc_csr* S, const orc_csr* ST, uint32_t* cf);
int  orc_direct_interpolation(const orc_csr* A, const orc_csr* S, const uint32_t* cf,
                              orc_csr* P);

orc_hier* orc_amg_setup(int kind, const orc_csr* A, int max_level);
/* Jones-Plassmann-Luby colouring of the pattern of A + A^T as the device smoother
 * builds it: colour[i] for every row; returns the number of colours. */
int orc_mc_colouring(const orc_csr* A, int* colour);
void      orc_hier_free(orc_hier* h);

/* solve phase.  omega: Jacobi weight (1.0 reproduces the reference's unweighted
 * Jacobi, jacobi.cpp:58-74, bit for bit). */
void orc_vcycle(orc_hier* h, int level, double* x, const double* b, int n1, int n2,
                int smoother, double omega, int coarse);
int  orc_amg_pcg(orc_hier* h, const double* b, double* x, int n1, int n2, int smoother,
                 double omega, int coarse, double rel_tol, double abs_tol, int max_iter,
                 double* final_rel);
int  orc_cg(const orc_csr* A, const double* b, double* x, int jacobi, double rel_tol,
            double abs_tol, int max_iter);
int  orc_amg_solve(orc_hier* h, const double* b, double* x, int n1, int n2, int smoother,
                   double omega, int coarse, double rel_tol, double abs_tol, int max_cycle);

/* triangular path: in-place ILU(0) / IC(0) (the factors overwrite A's values;
 * *structural_zero / *numeric_zero get the smallest column of a missing / zero
 * pivot, INT_MAX when none), triangular solves on the lower or upper part of A,
 * and one application x = M^-1 rhs of the ILU(0), IC(0), Gauss-Seidel and SOR
 * preconditioners (kind 0..3). */
void orc_csrilu0(orc_csr* A, int* structural_zero, int* numeric_zero);
void orc_csric0(orc_csr* A, int* structural_zero, int* numeric_zero);
void orc_trsv(const orc_csr* A, int lower, int unit_diag, const double* b, double* x);
void orc_precond_apply(int kind, double omega, const orc_csr* A, const double* rhs, double* x);
int  orc_precond_cg(int kind, double omega, const orc_csr* A, const double* b, double* x,
                    double rel_tol, double abs_tol, int max_iter);

#ifdef __cplusplus
}
#endif
#endif
