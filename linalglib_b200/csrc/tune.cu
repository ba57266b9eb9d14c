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

#include <algorithm>
#include <array>
#include <cstdio>
#include <map>
#include <mutex>
#include <string>
#include <vector>

namespace lab
{
    // ------------------------------------------------------------ plan cache
    // Tuned choices keyed by the operands' shapes (rows, columns, nonzeros): SpMV
    // schedules per matrix and exactness, SpGEMM table sizing per pair of
    // matrices.  A rerun on the same problem (a new setup of the same operator, a
    // hierarchy loaded from a file) finds its plans here instead of timing again;
    // lab_tune_cache_save / load keep them across processes.
    namespace
    {
        using spmv_key = std::array<int64_t, 4>; // m, n, nnz, exact
        using gemm_key = std::array<int64_t, 6>; // A m, n, nnz, B m, n, nnz
        struct spmv_entry
        {
            int    alg = LAB_SPMV_ROWSEQ, lanes = 1;
            int    form = 0; // VECTOR: 0 direct loads, 1 streamed, 2 halo
            double us  = 0.0;
        };
        struct gemm_entry
        {
            gemm_tune t;
            double    us = 0.0;
        };
        std::mutex                        g_cache_mu;
        std::map<spmv_key, spmv_entry>    g_spmv_cache;
        std::map<gemm_key, gemm_entry>    g_gemm_cache;

        gemm_key key_of(const lab_csr_impl* A, const lab_csr_impl* B)
        {
            return {A->m, A->n, A->nnz, B->m, B->n, B->nnz};
        }
    }

    gemm_tune gemm_tune_lookup(const lab_csr_impl* A, const lab_csr_impl* B)
    {
        std::lock_guard<std::mutex> g(g_cache_mu);
        auto                        it = g_gemm_cache.find(key_of(A, B));
        return it == g_gemm_cache.end() ? gemm_tune() : it->second.t;
    }

    void gemm_tune_store(const lab_csr_impl* A, const lab_csr_impl* B, gemm_tune t)
    {
        std::lock_guard<std::mutex> g(g_cache_mu);
        g_gemm_cache[key_of(A, B)].t = t;
    }

    namespace
    {
        constexpr int kTuneWarm = 2;
        constexpr int kTuneReps = 10;

        lab_status tune_one(lab_csr_impl* A, int exact, double* best_us, cudaStream_t s)
        {
            A->plan.forced   = 0;
            A->plan.stream   = 0;
            A->plan.halo_use = 0;
            A->plan.analysed = 0;
            LAB_TRY(spmv_analyse(A, s)); // row statistics (and the default plan)
            if(A->m == 0 || A->nnz == 0)
            {
                if(best_us)
                    *best_us = 0.0;
                return LAB_OK;
            }
            const spmv_key key{A->m, A->n, A->nnz, exact ? 1 : 0};
            {
                std::lock_guard<std::mutex> g(g_cache_mu);
                auto                        hit = g_spmv_cache.find(key);
                if(hit != g_spmv_cache.end())
                {
                    A->plan.alg      = hit->second.alg;
                    A->plan.lanes    = hit->second.lanes;
                    A->plan.stream   = hit->second.form == 1;
                    A->plan.halo_use = hit->second.form == 2;
                    A->plan.forced   = 1;
                    if(best_us)
                        *best_us = hit->second.us;
                    return LAB_OK;
                }
            }
            if(!exact && A->plan.max_row > 32)
                LAB_TRY(halo_build(A, s)); // the halo form's plan, a candidate below
            // form: 0 direct loads, 1 streamed, 2 halo (each where the matrix has one)
            struct cand
            {
                int alg, lanes, form;
            };
            std::vector<cand> cands = {{LAB_SPMV_ROWSEQ, 1, 0}};
            if(!exact)
                for(int w : {2, 4, 8, 16, 32})
                {
                    cands.push_back({LAB_SPMV_VECTOR, w, 0});
                    if(A->plan.st_rows > 0)
                        cands.push_back({LAB_SPMV_VECTOR, w, 1});
                    if(A->plan.halo_state == 1)
                        cands.push_back({LAB_SPMV_VECTOR, w, 2});
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
                A->plan.alg      = c.alg;
                A->plan.lanes    = c.lanes;
                A->plan.stream   = c.form == 1;
                A->plan.halo_use = c.form == 2;
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
            A->plan.alg      = win.alg;
            A->plan.lanes    = win.lanes;
            A->plan.stream   = win.form == 1;
            A->plan.halo_use = win.form == 2;
            A->plan.forced   = 1;
            if(st != LAB_OK)
                return st;
            if(best_us)
                *best_us = 1e3 * best / kTuneReps;
            std::lock_guard<std::mutex> g(g_cache_mu);
            g_spmv_cache[key] = {win.alg, win.lanes, win.form, 1e3 * best / kTuneReps};
            return LAB_OK;
        }

        // Time every table sizing on C = A B (results are the same for all) and keep
        // the fastest for A's and B's shapes.
        lab_status tune_gemm(const lab_csr_impl* A, const lab_csr_impl* B, double* best_us,
                             cudaStream_t s)
        {
            const gemm_tune cands[] = {{2, 3, 4}, {1, 3, 4}, {4, 3, 4}, {2, 1, 2}, {1, 1, 2},
                                       {4, 1, 2}};
            cudaEvent_t e0, e1;
            LAB_CUDA(cudaEventCreate(&e0));
            LAB_CUDA(cudaEventCreate(&e1));
            lab_status st   = LAB_OK;
            float      best = -1.f;
            gemm_tune  win  = cands[0];
            for(const gemm_tune& t : cands)
            {
                std::vector<float> ms;
                for(int r = 0; r < 4 && st == LAB_OK; r++) // one warm-up, three timed
                {
                    lab_csr_impl* C = nullptr;
                    cudaEventRecord(e0, s);
                    st = spgemm_tuned(A, B, &C, s, t);
                    cudaEventRecord(e1, s);
                    if(st == LAB_OK)
                    {
                        cudaError_t e = cudaEventSynchronize(e1);
                        if(e != cudaSuccess)
                            st = cuda_status(e, "spgemm autotune", __FILE__, __LINE__);
                        float x = 0.f;
                        cudaEventElapsedTime(&x, e0, e1);
                        if(r > 0)
                            ms.push_back(x);
                    }
                    if(C)
                        csr_release(C);
                }
                if(st != LAB_OK)
                    break;
                std::sort(ms.begin(), ms.end());
                const float med = ms[ms.size() / 2];
                if(best < 0.f || med < best)
                {
                    best = med;
                    win  = t;
                }
            }
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            LAB_TRY(st);
            std::lock_guard<std::mutex> g(g_cache_mu);
            g_gemm_cache[key_of(A, B)] = {win, 1e3 * best};
            if(best_us)
                *best_us = 1e3 * best;
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

LAB_API lab_status lab_spgemm_autotune(lab_csr A, lab_csr B, double* best_us, lab_stream ls)
{
    LAB_ARG(A && B, "null matrix");
    LAB_ARG(A->n == B->m, "inner dimensions differ");
    LAB_TRY(ensure_init());
    return tune_gemm(A, B, best_us, to_stream(ls));
}

LAB_API lab_status lab_hierarchy_tune_products(lab_hierarchy h, lab_stream ls)
{
    LAB_ARG(h, "null hierarchy");
    LAB_TRY(ensure_init());
    cudaStream_t s = to_stream(ls);
    for(int l = 0; l < h->levels; l++)
    {
        LAB_TRY(tune_gemm(h->A[l], h->P[l], nullptr, s));
        lab_csr_impl* AP = nullptr;
        LAB_TRY(spgemm(h->A[l], h->P[l], &AP, s));
        lab_status st = tune_gemm(h->R[l], AP, nullptr, s);
        csr_release(AP);
        LAB_TRY(st);
    }
    return LAB_OK;
}

LAB_API lab_status lab_tune_cache_save(const char* path)
{
    LAB_ARG(path, "null path");
    FILE* f = std::fopen(path, "w");
    if(!f)
    {
        set_error("lab_tune_cache_save: cannot open %s", path);
        return LAB_BAD_ARG;
    }
    std::lock_guard<std::mutex> g(g_cache_mu);
    std::fprintf(f, "linalglib_b200 tune cache 1\n");
    for(const auto& kv : g_spmv_cache)
        std::fprintf(f, "spmv %lld %lld %lld %lld %d %d %d %.6f\n", (long long)kv.first[0],
                     (long long)kv.first[1], (long long)kv.first[2], (long long)kv.first[3],
                     kv.second.alg, kv.second.lanes, kv.second.form, kv.second.us);
    for(const auto& kv : g_gemm_cache)
        std::fprintf(f, "gemm %lld %lld %lld %lld %lld %lld %d %d %d %.6f\n",
                     (long long)kv.first[0], (long long)kv.first[1], (long long)kv.first[2],
                     (long long)kv.first[3], (long long)kv.first[4], (long long)kv.first[5],
                     kv.second.t.sym, kv.second.t.fill_num, kv.second.t.fill_den, kv.second.us);
    const bool ok = std::ferror(f) == 0;
    if(std::fclose(f) != 0 || !ok)
    {
        set_error("lab_tune_cache_save: write to %s failed", path);
        return LAB_BAD_ARG;
    }
    return LAB_OK;
}

LAB_API lab_status lab_tune_cache_load(const char* path)
{
    LAB_ARG(path, "null path");
    FILE* f = std::fopen(path, "r");
    if(!f)
    {
        set_error("lab_tune_cache_load: cannot open %s", path);
        return LAB_BAD_ARG;
    }
    char line[512];
    bool ok = std::fgets(line, sizeof(line), f) &&
              std::string(line).rfind("linalglib_b200 tune cache 1", 0) == 0;
    std::map<spmv_key, spmv_entry> sp;
    std::map<gemm_key, gemm_entry> gm;
    while(ok && std::fgets(line, sizeof(line), f))
    {
        long long a[6];
        int       p[3];
        double    us = 0.0;
        if(std::sscanf(line, "spmv %lld %lld %lld %lld %d %d %d %lf", &a[0], &a[1], &a[2], &a[3],
                       &p[0], &p[1], &p[2], &us) == 8)
        {
            const bool lanes_ok = p[1] == 1 || p[1] == 2 || p[1] == 4 || p[1] == 8 ||
                                  p[1] == 16 || p[1] == 32;
            ok = (p[0] == LAB_SPMV_ROWSEQ || p[0] == LAB_SPMV_VECTOR) && lanes_ok &&
                 (p[2] == 0 || p[2] == 1 || p[2] == 2) && (a[3] == 0 || a[3] == 1);
            if(ok)
                sp[{a[0], a[1], a[2], a[3]}] = {p[0], p[1], p[2], us};
        }
        else if(std::sscanf(line, "gemm %lld %lld %lld %lld %lld %lld %d %d %d %lf", &a[0], &a[1],
                            &a[2], &a[3], &a[4], &a[5], &p[0], &p[1], &p[2], &us) == 10)
        {
            ok = (p[0] == 1 || p[0] == 2 || p[0] == 4) &&
                 ((p[1] == 3 && p[2] == 4) || (p[1] == 1 && p[2] == 2));
            if(ok)
                gm[{a[0], a[1], a[2], a[3], a[4], a[5]}] = {gemm_tune{p[0], p[1], p[2]}, us};
        }
        else
            ok = false;
    }
    std::fclose(f);
    if(!ok)
    {
        set_error("lab_tune_cache_load: %s is not a tune cache or holds a bad entry", path);
        return LAB_BAD_ARG;
    }
    std::lock_guard<std::mutex> g(g_cache_mu);
    for(const auto& kv : sp)
        g_spmv_cache[kv.first] = kv.second;
    for(const auto& kv : gm)
        g_gemm_cache[kv.first] = kv.second;
    return LAB_OK;
}

LAB_API lab_status lab_tune_cache_clear(void)
{
    std::lock_guard<std::mutex> g(g_cache_mu);
    g_spmv_cache.clear();
    g_gemm_cache.clear();
    return LAB_OK;
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
