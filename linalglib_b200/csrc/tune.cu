// SpMV schedule autotuner.  The default plan comes from row-length statistics
// (spmv_analyse); the tuner instead times every candidate schedule on the
// matrix itself (CUDA events, back-to-back launches of y = A x) and keeps the
// fastest.  Candidates: the one-thread-per-row pipeline (CSR-order accumulation,
// bit-identical to the reference host SpMV) and, unless the caller asks for
// bit-exact results, W = 2, 4, 8, 16, 32 lanes per row (reordered sums), each
// with the matrix read directly and, on operators large enough, streamed
// through shared memory.  The
// fused V-cycle passes (smoother, restriction, prolongation) run on the same
// schedule as the plain SpMV of their matrix, so tuning a hierarchy tunes them.
#include "amg.cuh"
#include "spmv_engine.cuh"

#include <vector>

namespace lab
{
    namespace
    {
        constexpr int kTuneWarm = 2;
        constexpr int kTuneReps = 10;

        lab_status tune_one(lab_csr_impl* A, int exact, double* best_us, cudaStream_t s)
        {
            A->plan.forced   = 0;
            A->plan.stream   = 0;
            A->plan.analysed = 0;
            LAB_TRY(spmv_analyse(A, s)); // row statistics (and the default plan)
            if(A->m == 0 || A->nnz == 0)
            {
                if(best_us)
                    *best_us = 0.0;
                return LAB_OK;
            }
            struct cand
            {
                int alg, lanes, stream;
            };
            std::vector<cand> cands = {{LAB_SPMV_ROWSEQ, 1, 0}};
            if(!exact)
                for(int w : {2, 4, 8, 16, 32})
                {
                    cands.push_back({LAB_SPMV_VECTOR, w, 0});
                    if(A->plan.st_rows > 0) // the streamed form where the matrix has one
                        cands.push_back({LAB_SPMV_VECTOR, w, 1});
                }
            dbuf<double> x, y;
            LAB_TRY(x.alloc((size_t)A->n + 1, s));
            LAB_TRY(y.alloc((size_t)A->m + 1, s));
            LAB_TRY(lab_fill(A->n, 1.0, x.get(), s));
            cudaEvent_t e0, e1;
            LAB_CUDA(cudaEventCreate(&e0));
            LAB_CUDA(cudaEventCreate(&e1));
            lab_status st   = LAB_OK;
            float      best = -1.f;
            cand       win  = cands[0];
            for(const cand& c : cands)
            {
                A->plan.alg    = c.alg;
                A->plan.lanes  = c.lanes;
                A->plan.stream = c.stream;
                op_spmv op{x.get(), y.get(), 1.0, 0.0};
                for(int k = 0; k < kTuneWarm && st == LAB_OK; k++)
                    st = launch_rowop(A, A->val, op, s);
                cudaEventRecord(e0, s);
                for(int k = 0; k < kTuneReps && st == LAB_OK; k++)
                    st = launch_rowop(A, A->val, op, s);
                cudaEventRecord(e1, s);
                if(st != LAB_OK)
                    break;
                cudaError_t e = cudaEventSynchronize(e1);
                if(e != cudaSuccess)
                {
                    st = cuda_status(e, "spmv autotune", __FILE__, __LINE__);
                    break;
                }
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                if(best < 0.f || ms < best)
                {
                    best = ms;
                    win  = c;
                }
            }
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            A->plan.alg    = win.alg;
            A->plan.lanes  = win.lanes;
            A->plan.stream = win.stream;
            A->plan.forced = 1;
            if(st != LAB_OK)
                return st;
            if(best_us)
                *best_us = 1e3 * best / kTuneReps;
            return LAB_OK;
        }
    }
}

using namespace lab;

extern "C" {

LAB_API lab_status lab_spmv_autotune(lab_csr A, int exact, double* best_us, lab_stream ls)
{
    LAB_ARG(A, "null matrix");
    LAB_TRY(ensure_init());
    cudaStream_t s = to_stream(ls);
    // a solver iteration graph captured on this matrix keeps the old schedule
    solver_cache_forget(A);
    return tune_one(A, exact, best_us, s);
}

LAB_API lab_status lab_hierarchy_autotune(lab_hierarchy h, int exact, lab_stream ls)
{
    LAB_ARG(h, "null hierarchy");
    LAB_TRY(ensure_init());
    cudaStream_t s = to_stream(ls);
    solver_cache_forget(h);
    for(int l = 0; l <= h->levels; l++)
    {
        LAB_TRY(tune_one(h->A[l], exact, nullptr, s));
        if(l < h->levels)
        {
            LAB_TRY(tune_one(h->P[l], exact, nullptr, s));
            LAB_TRY(tune_one(h->R[l], exact, nullptr, s));
        }
    }
    return LAB_OK;
}

} // extern "C"
