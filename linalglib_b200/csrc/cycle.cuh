// Multigrid cycles (cycle.cu) as used by the solvers (solve.cu).
#pragma once

#include "amg.cuh"
#include "spmv_engine.cuh"

namespace lab
{
    struct cyc_ctx
    {
        const lab_amg_options* o;
        cudaStream_t           s;
        const int*             skip; // early-exit flag (PCG graph), may be null
    };

    // Allocate every per-level vector, analyse every operator, build the
    // reduced-precision copies / colourings / coarse inverse the options need.
    // Synchronises; never called inside a graph capture.
    lab_status cycle_prepare(hierarchy_impl* h, const lab_amg_options* o, cudaStream_t s);

    // z = cycle(0; r) on level 0 (FP64 interface whatever the cycle precision).
    // With dot.out set, also (z, r) -> dot.out.  Enqueue only (capturable).
    lab_status cycle_precond(hierarchy_impl* h, const cyc_ctx& c, const double* r, double* z,
                             red_buf dot);
    // Reduced-precision preconditioner step of flexible PCG: the FP32 cycle on r,
    // (z, r) into zr.out and (z, q) into zq.out with z = fp64 of the cycle's result,
    // which stays in FP32 in the level-0 workspace (*z32; valid until the next cycle).
    lab_status cycle_precond_flex(hierarchy_impl* h, const cyc_ctx& c, const double* r,
                                  const double* q, red_buf zr, red_buf zq, const float** z32);

    // x <- cycle(x; b) on level 0 (stationary iteration step).  FP64 cycles run in
    // place; reduced-precision cycles run in correction form x += cycle(0; b - A x).
    lab_status cycle_iterate(hierarchy_impl* h, const cyc_ctx& c, const double* b, double* x);

    // Block V-cycle over many right-hand sides (cycle_blk.cu): whether the options
    // are covered (V-cycle, Jacobi, FP64, 1x1 or dense coarsest solve; call after
    // cycle_prepare), the block workspace (outside graph capture), and
    // z[:, k] = cycle(0; r[:, k]) for ncols column-major columns, 8 per pass.
    bool       cycle_block_supported(const hierarchy_impl* h, const lab_amg_options* o);
    lab_status cycle_prepare_block(hierarchy_impl* h, cudaStream_t s);
    lab_status cycle_precond_block(hierarchy_impl* h, const cyc_ctx& c, int ncols, const double* r,
                                   int64_t ldr, double* z, int64_t ldz);

    // deterministic device reductions into r.out (grid <= kRedBlocks)
    lab_status dot_device(int64_t n, const double* x, const double* y, red_buf r, cudaStream_t s);
    lab_status norm_inf_device(int64_t n, const double* x, red_buf r, cudaStream_t s);
    unsigned   red_grid(int64_t n);
    unsigned   grid_for(int64_t n);

    __global__ void k_copy_d(double* __restrict__ y, const double* __restrict__ x, int64_t n,
                             const int* skip);
}
