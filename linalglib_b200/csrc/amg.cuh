// AMG hierarchy shared by the setup (amg_setup.cu) and solve (solve.cu) units.
#pragma once

#include "internal.cuh"

namespace lab
{
    constexpr int kMaxLevels = 20; // hierarchy arrays of the reference, amg.h:76-99

    struct level_ws
    {
        // per-level cycle vectors (device, m_l entries each)
        double* x   = nullptr; // level correction / iterate
        double* b   = nullptr; // level right-hand side
        double* r   = nullptr; // residual
        double* t   = nullptr; // scratch (Jacobi old iterate, W/F second pass)
        float*  xf  = nullptr; // fp32 cycle vectors (mixed precision)
        float*  bf  = nullptr;
        float*  rf  = nullptr;
        float*  tf  = nullptr;
        double* xk  = nullptr; // block cycle vectors: m_l x 8 columns, interleaved per row
        double* bk  = nullptr;
        double* rk  = nullptr;
        double* tk  = nullptr;
        int32_t* colour = nullptr; // multicolour GS: row order by colour
        int32_t* colour_ptr_h = nullptr; // host copy of colour offsets
        int      ncolours = 0;
    };

    struct hierarchy_impl
    {
        int           kind   = 0;
        int           levels = 0;
        lab_csr_impl* A[kMaxLevels + 1] = {};
        lab_csr_impl* P[kMaxLevels]     = {};
        lab_csr_impl* R[kMaxLevels]     = {};
        double        setup_ms          = 0.0;
        level_ws      ws[kMaxLevels + 1];
        int           ws_ready = 0;
        // dense inverse of the coarsest operator (LAB_COARSE_DIRECT), row major
        double* coarse_inv   = nullptr;
        float*  coarse_inv32 = nullptr;
        int     coarse_n     = 0;
        int     coarse_singular = 0;
    };

    lab_status hierarchy_release(hierarchy_impl* h);
    // SpMV schedules of the coarse levels (after a setup or a load).
    lab_status hierarchy_plans(hierarchy_impl* h, cudaStream_t s);

    // pieces (amg_setup.cu)
    lab_status amg_strength(const lab_csr_impl* A, double eps, int32_t* conn, cudaStream_t s);
    lab_status amg_pmis(const lab_csr_impl* A, const int32_t* conn, int64_t* agg, int* rounds,
                        cudaStream_t s, int64_t* roots);
    lab_status amg_sa_prolongation(const lab_csr_impl* A, const int32_t* conn, const int64_t* agg,
                                   double relax, lab_csr_impl** P, cudaStream_t s);
    lab_status amg_ua_prolongation(const lab_csr_impl* A, const int64_t* agg, lab_csr_impl** P,
                                   cudaStream_t s);
    lab_status amg_classical_strength(const lab_csr_impl* A, double theta, int32_t* conn,
                                      lab_csr_impl** S, cudaStream_t s);
    lab_status amg_cfpoints(const lab_csr_impl* S, uint32_t* cf, cudaStream_t s, int first,
                            int second);
    lab_status amg_direct_interpolation(const lab_csr_impl* A, const lab_csr_impl* S,
                                        const uint32_t* cf, lab_csr_impl** P, cudaStream_t s);

    // sparse products (spgemm.cu)
    lab_status transpose(const lab_csr_impl* A, lab_csr_impl** T, cudaStream_t s);
    // Table sizing of the hash SpGEMM row classes (spgemm.cu gemm_class): symbolic
    // tables hold >= sym / 2 x the row's product bound, numeric tables are filled to
    // at most fill_num / fill_den.  Results do not depend on it (only table sizes).
    struct gemm_tune
    {
        int sym      = 2;
        int fill_num = 3;
        int fill_den = 4;
    };
    // The tuned sizing for products of matrices of A's and B's shapes (tune.cu
    // cache; the defaults when none was tuned) and its store.
    gemm_tune gemm_tune_lookup(const lab_csr_impl* A, const lab_csr_impl* B);
    void      gemm_tune_store(const lab_csr_impl* A, const lab_csr_impl* B, gemm_tune t);
    lab_status spgemm(const lab_csr_impl* A, const lab_csr_impl* B, lab_csr_impl** C,
                      cudaStream_t s);
    lab_status spgemm_tuned(const lab_csr_impl* A, const lab_csr_impl* B, lab_csr_impl** C,
                            cudaStream_t s, gemm_tune tune);
    lab_status row_lengths(const int32_t* rp, int64_t m, int32_t* len, cudaStream_t s);
    lab_status spgeam(double alpha, const lab_csr_impl* A, double beta, const lab_csr_impl* B,
                      lab_csr_impl** C, cudaStream_t s);
}

struct lab_hier_s : lab::hierarchy_impl
{
};
