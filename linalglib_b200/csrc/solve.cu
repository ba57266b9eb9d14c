// Solve phase: fused multigrid cycles, preconditioners, PCG (device-resident
// scalars, one CUDA graph per iteration), stationary AMG and GMRES.
#include "cycle.cuh"
#include "tri.cuh"

#include <cmath>
#include <cstdlib>
#include <map>
#include <mutex>
#include <tuple>

namespace lab
{
    // ================================================================ preconditioners
    struct precond_impl
    {
        uint64_t         uid  = next_uid();
        // 0 AMG, 1 Jacobi, 2 ILU(0), 3 IC(0), 4 Gauss-Seidel, 5 SOR, 6 SSOR
        int              kind = 0;
        hierarchy_impl*  h    = nullptr;
        lab_amg_options  o;
        lab_csr_impl*    A    = nullptr; // the operator
        double*          diag = nullptr; // Jacobi: own copy of the diagonal taken at build
                                         // (jacobi_precond::build keeps its own, preconditioner.cpp:41-78)
        lab_csr_impl*    F    = nullptr; // kinds 2-5: factored / copied operator; SSOR: L
        lab_csr_impl*    G    = nullptr; // SSOR: U
        double*          y    = nullptr; // intermediate of the two solves (kinds 2, 3, 6)
        double           dscale = 0.0;   // SOR: diagonal scale 1 / omega
        ~precond_impl()
        {
            if(F)
                csr_release(F);
            if(G)
                csr_release(G);
            if(y)
                cudaFree(y);
            if(diag)
                cudaFree(diag);
        }
    };

    __global__ void k_jacobi_dot(int64_t n, const double* __restrict__ r,
                                 const double* __restrict__ d, double* __restrict__ z,
                                 double* partial, unsigned int* counter, double* out,
                                 const int* skip)
    {
        if(skip && *skip)
            return;
        double acc = 0.0;
        for(int64_t i = blockIdx.x * 256ll + threadIdx.x; i < n; i += (int64_t)gridDim.x * 256)
        {
            double zi = __ddiv_rn(r[i], d[i]);
            z[i]      = zi;
            acc += zi * r[i];
        }
        if(out)
            reduce_finish_sum<256>(acc, partial, counter, out);
    }

    // z = M^-1 r; with dot.out set, also dot(z, r) -> dot.out.
    static lab_status precond_apply(precond_impl* M, const double* r, double* z, cudaStream_t s,
                                    const int* skip, red_buf dot)
    {
        if(M->kind >= 2)
        {
            // preconditioner.cpp: ILU(0) 452-467, IC(0) 527-542 (lower then upper
            // solve of the factored copy), Gauss-Seidel 98-105 and SOR 149-156
            // (one lower solve on A, SOR's diagonal scaled by 1 / omega), SSOR
            // (lower solve with L, upper solve with U)
            if(M->kind == 2 || M->kind == 3)
            {
                LAB_TRY(tri_solve(M->F, true, M->kind == 2, 0.0, r, M->y, s, skip));
                LAB_TRY(tri_solve(M->F, false, false, 0.0, M->y, z, s, skip));
            }
            else if(M->kind == 6) // SSOR_precond::solve 355-395 (host trsv: alpha unused)
            {
                LAB_TRY(tri_solve(M->F, true, false, 0.0, r, M->y, s, skip));
                LAB_TRY(tri_solve(M->G, false, false, 0.0, M->y, z, s, skip));
            }
            else
                LAB_TRY(tri_solve(M->F, true, false, M->dscale, r, z, s, skip));
            if(dot.out)
                LAB_TRY(dot_device(M->F->m, z, r, dot, s));
            return LAB_OK;
        }
        if(M->kind == 1)
        {
            int64_t n = M->A->m;
            LAB_LAUNCH(k_jacobi_dot, red_grid(n), 256, 0, s, n, r, (const double*)M->diag, z,
                       dot.partial, dot.counter, dot.out, skip);
            return LAB_OK;
        }
        cyc_ctx c{&M->o, s, skip};
        return cycle_precond(M->h, c, r, z, dot);
    }

    // dL/dA_ij = -lambda_i x_j on the pattern of A (thread per row; the row's
    // entries are contiguous, so the writes and the col_ind reads coalesce).
    __global__ void k_adjoint_grad(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                   int64_t m, const double* __restrict__ lambda,
                                   const double* __restrict__ x, double* __restrict__ grad)
    {
        int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
        if(i >= m)
            return;
        const double li = -lambda[i];
        for(int j = rp[i]; j < rp[i + 1]; j++)
            grad[j] = li * __ldg(x + ci[j]);
    }

    // ================================================================ device-side loops
    // A solver's iterations as ONE graph launch: a conditional WHILE node runs the
    // captured iteration body again and again on the device.  A small kernel
    // before the node and one at the end of each body pass set the node's
    // condition: continue while *done == 0 and fewer than `limit` passes ran (the
    // pass counter lives in device memory and is reset by the first kernel).  The
    // host neither launches nor waits per iteration.
    __global__ void k_loop_cond(cudaGraphConditionalHandle h, const int* done, int* counter,
                                int limit, int reset)
    {
        if(threadIdx.x == 0)
        {
            const int c = reset ? 0 : *counter + 1;
            *counter    = c;
            cudaGraphSetConditional(h, (*(volatile const int*)done == 0 && c < limit) ? 1u : 0u);
        }
    }

    // LAB_SOLVE_HOST_LOOP=1 in the environment makes the host drive the iterations
    // (one graph launch per iteration, the same kernels): kernel profilers cannot
    // attribute kernels inside graphs that hold conditional nodes.
    static bool host_loop_forced()
    {
        static const bool forced = [] {
            const char* e = std::getenv("LAB_SOLVE_HOST_LOOP");
            return e && e[0] == '1';
        }();
        return forced;
    }

    // Builds and instantiates the loop graph; `body(stream)` enqueues one iteration
    // on the capturing stream.  *nodes receives the body's node count (kernel
    // launches per pass, for the launch counter).  Returns LAB_NOT_SUPPORTED,
    // with nothing built, where the driver has no conditional nodes.
    template <class Body>
    static lab_status build_loop_graph(cudaStream_t cap, const int* done, int* counter, int limit,
                                       Body&& body, cudaGraphExec_t* out, int64_t* nodes)
    {
        *out             = nullptr;
        if(host_loop_forced())
            return LAB_NOT_SUPPORTED;
        cudaGraph_t    g = nullptr;
        LAB_CUDA(cudaGraphCreate(&g, 0));
        cudaGraphConditionalHandle h;
        if(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault) != cudaSuccess)
        {
            cudaGetLastError();
            cudaGraphDestroy(g);
            return LAB_NOT_SUPPORTED;
        }
        lab_status  st = LAB_OK;
        cudaError_t e  = cudaStreamBeginCaptureToGraph(cap, g, nullptr, nullptr, 0,
                                                       cudaStreamCaptureModeThreadLocal);
        if(e == cudaSuccess)
        {
            k_loop_cond<<<1, 32, 0, cap>>>(h, done, counter, limit, 1);
            cudaGraph_t gg = nullptr;
            e              = cudaStreamEndCapture(cap, &gg);
        }
        cudaGraphNode_t pro = nullptr;
        size_t          np  = 1;
        if(e == cudaSuccess)
            e = cudaGraphGetNodes(g, &pro, &np);
        cudaGraphNodeParams cp = {};
        cp.type                = cudaGraphNodeTypeConditional;
        cp.conditional.handle  = h;
        cp.conditional.type    = cudaGraphCondTypeWhile;
        cp.conditional.size    = 1;
        cudaGraphNode_t cn     = nullptr;
        if(e == cudaSuccess)
            e = cudaGraphAddNode(&cn, g, &pro, 1, &cp);
        if(e == cudaSuccess)
        {
            cudaGraph_t bodyg = cp.conditional.phGraph_out[0];
            e = cudaStreamBeginCaptureToGraph(cap, bodyg, nullptr, nullptr, 0,
                                              cudaStreamCaptureModeThreadLocal);
            if(e == cudaSuccess)
            {
                st = body(cap);
                k_loop_cond<<<1, 32, 0, cap>>>(h, done, counter, limit, 0);
                cudaGraph_t bg = nullptr;
                e              = cudaStreamEndCapture(cap, &bg);
                size_t n       = 0;
                if(e == cudaSuccess && st == LAB_OK)
                    e = cudaGraphGetNodes(bodyg, nullptr, &n);
                *nodes = (int64_t)n;
            }
        }
        if(e == cudaSuccess && st == LAB_OK)
            e = cudaGraphInstantiate(out, g, 0);
        cudaGraphDestroy(g);
        if(st != LAB_OK)
            return st;
        if(e != cudaSuccess)
        {
            *out = nullptr;
            return cuda_status(e, "loop graph", __FILE__, __LINE__);
        }
        return LAB_OK;
    }

    // ================================================================ PCG
    enum
    {
        S_GAMMA = 0,
        S_PQ    = 1,
        S_RN    = 2,
        S_R0    = 3,
        S_GNEW  = 4,
        S_RTOL  = 5,
        S_ATOL  = 6,
        S_ZQ    = 7, // (z_{k+1}, q_k), flexible variant only
        S_COUNT = 8
    };
    enum
    {
        F_DONE   = 0,
        F_ITER   = 1,
        F_STATUS = 2,
        F_CONV   = 3,
        F_MAXIT  = 4,
        F_LOOP   = 5, // passes of the device-side iteration loop
        F_COUNT  = 8
    };

    // Host-side resources of a PCG workspace (pinned flag slots, two events, the
    // capture stream), kept per device for reuse when a workspace goes away: a
    // caller that builds a new matrix for every solve then pays no page-locking,
    // event or stream creation per solve, and no cudaFreeHost (which synchronises
    // the device).  At most kResPool sets per device are kept; the lists are never
    // destroyed (workspaces can be released during static destruction).
    struct pcg_host_res
    {
        int*         hflags = nullptr;
        cudaEvent_t  ev[2]  = {nullptr, nullptr};
        cudaStream_t cap    = nullptr;
    };
    constexpr size_t kResPool = 16;
    static std::mutex& res_mu()
    {
        static std::mutex* mu = new std::mutex;
        return *mu;
    }
    static std::map<int, std::vector<pcg_host_res>>& res_pool()
    {
        static auto* pool = new std::map<int, std::vector<pcg_host_res>>;
        return *pool;
    }
    static lab_status res_take(int dev, pcg_host_res* out)
    {
        {
            std::lock_guard<std::mutex> g(res_mu());
            auto&                       v = res_pool()[dev];
            if(!v.empty())
            {
                *out = v.back();
                v.pop_back();
                return LAB_OK;
            }
        }
        pcg_host_res r;
        LAB_CUDA(cudaMallocHost(&r.hflags, sizeof(int) * F_COUNT * 2));
        LAB_CUDA(cudaEventCreateWithFlags(&r.ev[0], cudaEventDisableTiming));
        LAB_CUDA(cudaEventCreateWithFlags(&r.ev[1], cudaEventDisableTiming));
        LAB_CUDA(cudaStreamCreateWithFlags(&r.cap, cudaStreamNonBlocking));
        *out = r;
        return LAB_OK;
    }
    static void res_give(int dev, const pcg_host_res& r)
    {
        {
            std::lock_guard<std::mutex> g(res_mu());
            auto&                       v = res_pool()[dev];
            if(v.size() < kResPool && r.hflags && r.ev[0] && r.ev[1] && r.cap)
            {
                v.push_back(r);
                return;
            }
        }
        if(r.hflags)
            cudaFreeHost(r.hflags);
        for(auto e : r.ev)
            if(e)
                cudaEventDestroy(e);
        if(r.cap)
            cudaStreamDestroy(r.cap);
    }

    struct pcg_ws
    {
        int           dev   = 0; // device the host-side resources belong to
        int64_t       m     = 0;
        double*       r     = nullptr;
        double*       z     = nullptr;
        double*       p     = nullptr;
        double*       q     = nullptr;
        double*       sc    = nullptr; // device scalars
        int*          flags = nullptr; // device flags
        double*       partial = nullptr;
        unsigned int* counters = nullptr; // 8 independent tickets
        int64_t       partial_n = 0;
        int*          hflags  = nullptr; // pinned: two slots of F_COUNT
        cudaEvent_t   ev[2]   = {nullptr, nullptr};
        // private stream the iteration graph is captured on (the caller's stream
        // may be the legacy default stream, which cannot be captured)
        cudaStream_t  cap     = nullptr;
        int64_t       graph_nodes = 0; // kernel nodes per iteration graph
        cudaGraphExec_t graph = nullptr;
        uint64_t      key_M   = 0;
        const double* key_x   = nullptr;
        uint64_t      key_A   = 0;
        cudaStream_t  key_s   = nullptr;
        int           key_lim = 0; // max_iter + 1 the loop graph was built for
        int           host_loop = 0; // 1: conditional nodes unavailable, host drives
        // iterative-refinement vectors (mixed precision): kept with the matrix so the
        // inner solve's iteration graph (keyed by its x = ir_e) is captured once
        double*       ir_r   = nullptr;
        double*       ir_e   = nullptr;
        double*       ir_sc  = nullptr;
        unsigned int* ir_cnt = nullptr;
        ~pcg_ws()
        {
            if(graph)
                cudaGraphExecDestroy(graph);
            void* dp[] = {r, z, p, q, sc, flags, partial, counters, ir_r, ir_e, ir_sc, ir_cnt};
            for(void* x : dp)
                if(x)
                    cudaFree(x);
            pcg_host_res res;
            res.hflags = hflags;
            res.ev[0]  = ev[0];
            res.ev[1]  = ev[1];
            res.cap    = cap;
            res_give(dev, res);
        }
    };

    // x += alpha p; r -= alpha q (host_axpy.cpp:35-45 semantics); ||r||_inf;
    // the last block applies iter_control::residual_converges (iter_control.cpp:38-78).
    __global__ void __launch_bounds__(256)
        k_pcg_update(int64_t n, double* __restrict__ x, double* __restrict__ r,
                     const double* __restrict__ p, const double* __restrict__ q, double* sc,
                     int* flags, double* partial, unsigned int* counter)
    {
        if(flags[F_DONE])
            return;
        const double alpha = sc[S_GAMMA] / sc[S_PQ];
        const double na    = -1.0 * alpha;
        double       acc   = 0.0;
        for(int64_t i = blockIdx.x * 256ll + threadIdx.x; i < n; i += (int64_t)gridDim.x * 256)
        {
            double xi = alpha == 1.0 ? __dadd_rn(p[i], x[i]) : __dadd_rn(__dmul_rn(alpha, p[i]), x[i]);
            double ri = na == 1.0 ? __dadd_rn(q[i], r[i]) : __dadd_rn(__dmul_rn(na, q[i]), r[i]);
            x[i]      = xi;
            r[i]      = ri;
            acc       = nanmax(acc, fabs(ri));
        }
        double b = block_max<256>(acc);
        if(threadIdx.x == 0)
            partial[blockIdx.x] = b;
        if(grid_ticket(counter))
        {
            double s = 0.0;
            for(unsigned i = threadIdx.x; i < gridDim.x; i += 256)
                s = nanmax(s, __ldcg(partial + i));
            s = block_max<256>(s);
            if(threadIdx.x == 0)
            {
                *counter      = 0;
                sc[S_RN]      = s;
                double r0     = sc[S_R0];
                bool   nan    = isnan(s) || isnan(r0);
                bool   conv   = !nan && (s <= sc[S_ATOL] || s / r0 <= sc[S_RTOL]);
                if(conv)
                {
                    flags[F_CONV]   = 1;
                    flags[F_DONE]   = 1;
                    flags[F_STATUS] = LAB_OK;
                }
                else if(nan)
                {
                    flags[F_DONE]   = 1;
                    flags[F_STATUS] = LAB_NAN;
                }
            }
        }
    }

    // p = 1*z + beta*p (host_axpy.cpp:47-69), gamma <- (z, r), iter++.
    // FLEX: beta = -(z_{k+1}, q_k) / (p_k, q_k), the flexible (Polak-Ribiere)
    // choice: it equals (z_{k+1}, r_{k+1} - r_k) / (z_k, r_k), which keeps the
    // search directions A-conjugate to the previous one when the preconditioner
    // is not exactly the same symmetric operator at every application (a V-cycle
    // rounded to FP32 / BF16).  With a fixed SPD preconditioner both choices agree
    // in exact arithmetic.
    // ZT = float: z is the reduced-precision cycle's FP32 result, widened exactly.
    template <bool FLEX, class ZT = double>
    __global__ void __launch_bounds__(256)
        k_pcg_pupdate(int64_t n, double* __restrict__ p, const ZT* __restrict__ z, double* sc,
                      int* flags, unsigned int* counter)
    {
        if(flags[F_DONE])
            return;
        const double beta = FLEX ? -(sc[S_ZQ] / sc[S_PQ]) : sc[S_GNEW] / sc[S_GAMMA];
        for(int64_t i = blockIdx.x * 256ll + threadIdx.x; i < n; i += (int64_t)gridDim.x * 256)
        {
            const double zi = (double)z[i];
            p[i]            = beta == 0.0 ? zi : __dadd_rn(zi, __dmul_rn(beta, p[i]));
        }
        if(grid_ticket(counter))
        {
            if(threadIdx.x == 0)
            {
                *counter      = 0;
                sc[S_GAMMA]   = sc[S_GNEW];
                int it        = flags[F_ITER] + 1;
                flags[F_ITER] = it;
                if(it > flags[F_MAXIT])
                {
                    flags[F_DONE]   = 1;
                    flags[F_STATUS] = LAB_NOT_CONVERGED;
                }
            }
        }
    }

    // q = A p and (p, q) fused.
    struct op_spmv_dot
    {
        using val_t                   = double;
        using acc_t                   = double;
        static constexpr bool kFma    = true;
        static constexpr bool kReduce = true;
        const double* __restrict__ p;
        double* __restrict__ q;
        __device__ __forceinline__ double gather(int c) const
        {
            return __ldg(p + c);
        }
        __device__ __forceinline__ double finish(int i, double s) const
        {
            q[i] = s;
            return p[i] * s;
        }
        using pre_t = double; // p_i
        __device__ __forceinline__ double pre(int i) const
        {
            return __ldg(p + i);
        }
        __device__ __forceinline__ double finish(int i, double s, double pi) const
        {
            q[i] = s;
            return pi * s;
        }
    };

    // Initial state: gamma = gnew, flags, r0 == 0 short cut.
    __global__ void k_pcg_init(double* sc, int* flags, double rtol, double atol, int max_iter)
    {
        sc[S_GAMMA]     = sc[S_GNEW];
        sc[S_RTOL]      = rtol;
        sc[S_ATOL]      = atol;
        sc[S_RN]        = sc[S_R0];
        flags[F_ITER]   = 0;
        flags[F_CONV]   = 0;
        flags[F_STATUS] = LAB_NOT_CONVERGED;
        flags[F_MAXIT]  = max_iter;
        flags[F_DONE]   = 0;
        if(sc[S_R0] == 0.0)
        {
            // b == A x0 already: the reference would divide 0/0 in alpha; stop here.
            flags[F_DONE]   = 1;
            flags[F_CONV]   = 1;
            flags[F_STATUS] = LAB_OK;
        }
    }

    __global__ void k_pcg_setflags_for_plain(double* sc, int* flags)
    {
        sc[S_GAMMA] = sc[S_GNEW];
    }

    static std::mutex                     g_pcg_mu;
    static std::map<const void*, pcg_ws*> g_pcg_cache; // keyed by A (or hierarchy)

    void solver_cache_forget(const void* key)
    {
        pcg_ws* w = nullptr;
        {
            std::lock_guard<std::mutex> g(g_pcg_mu);
            auto                        it = g_pcg_cache.find(key);
            if(it == g_pcg_cache.end())
                return;
            w = it->second;
            g_pcg_cache.erase(it);
        }
        delete w;
    }
    static lab_status ensure_pcg_ws(pcg_ws* w, const lab_csr_impl* A, cudaStream_t s)
    {
        const int64_t m = A->m;
        if(w->m == m && w->r)
            return LAB_OK;
        w->m = m;
        LAB_TRY(dalloc(&w->r, (size_t)m + 1, s));
        LAB_TRY(dalloc(&w->z, (size_t)m + 1, s));
        LAB_TRY(dalloc(&w->p, (size_t)m + 1, s));
        LAB_TRY(dalloc(&w->q, (size_t)m + 1, s));
        LAB_TRY(dalloc(&w->sc, S_COUNT, s));
        LAB_TRY(dalloc(&w->flags, F_COUNT, s));
        w->partial_n = std::max<int64_t>(kRedBlocks, ceil_div<int64_t>(m * 32, 256)) + 1;
        LAB_TRY(dalloc(&w->partial, (size_t)w->partial_n * 6, s));
        LAB_TRY(dalloc(&w->counters, 16, s));
        LAB_CUDA(cudaMemsetAsync(w->counters, 0, sizeof(unsigned int) * 16, s));
        LAB_CUDA(cudaMemsetAsync(w->flags, 0, sizeof(int) * F_COUNT, s));
        LAB_CUDA(cudaGetDevice(&w->dev));
        pcg_host_res res;
        LAB_TRY(res_take(w->dev, &res));
        w->hflags = res.hflags;
        w->ev[0]  = res.ev[0];
        w->ev[1]  = res.ev[1];
        w->cap    = res.cap;
        return LAB_OK;
    }

    static red_buf rbuf(pcg_ws* w, int slot, double* out, const int* skip)
    {
        red_buf r;
        r.partial = w->partial + (size_t)slot * w->partial_n;
        r.counter = w->counters + slot;
        r.out     = out;
        r.skip    = skip;
        return r;
    }

    // Reduced-precision cycles take the flexible beta (k_pcg_pupdate<true>).
    static bool pcg_flexible(const precond_impl* M)
    {
        return M && M->kind == 0 && M->o.precision != LAB_PREC_FP64;
    }

    // One PCG iteration (cg.cpp:185-213): enqueue only, captured into a graph.
    static lab_status pcg_iteration(lab_csr_impl* A, precond_impl* M, double* x, pcg_ws* w,
                                    cudaStream_t s)
    {
        const int* skip = w->flags + F_DONE;
        op_spmv_dot op{w->p, w->q};
        LAB_TRY(launch_rowop(A, A->val, op, s, rbuf(w, 0, w->sc + S_PQ, skip)));
        LAB_LAUNCH(k_pcg_update, red_grid(A->m), 256, 0, s, A->m, x, w->r, (const double*)w->p,
                   (const double*)w->q, w->sc, w->flags, w->partial + w->partial_n,
                   w->counters + 1);
        if(pcg_flexible(M))
        {
            // FP32 cycle, then (z, r) and (z, q) in one pass over its FP32 result,
            // which p = z + beta p reads directly (no FP64 copy of z)
            cyc_ctx      c{&M->o, s, skip};
            const float* z32 = nullptr;
            LAB_TRY(cycle_precond_flex(M->h, c, w->r, w->q, rbuf(w, 2, w->sc + S_GNEW, skip),
                                       rbuf(w, 5, w->sc + S_ZQ, skip), &z32));
            LAB_LAUNCH((k_pcg_pupdate<true, float>), red_grid(A->m), 256, 0, s, A->m, w->p, z32,
                       w->sc, w->flags, w->counters + 3);
            return LAB_OK;
        }
        LAB_TRY(precond_apply(M, w->r, w->z, s, skip, rbuf(w, 2, w->sc + S_GNEW, skip)));
        LAB_LAUNCH(k_pcg_pupdate<false>, red_grid(A->m), 256, 0, s, A->m, w->p,
                   (const double*)w->z, w->sc, w->flags, w->counters + 3);
        return LAB_OK;
    }

    static lab_status pcg_solve(lab_csr_impl* A, precond_impl* M, const double* b, double* x,
                                const lab_iter_control* ctl, lab_solve_info* info, cudaStream_t s)
    {
        LAB_TRY(spmv_analyse(A, s));
        if(M && M->kind == 0)
            LAB_TRY(cycle_prepare(M->h, &M->o, s));
        pcg_ws* w = nullptr;
        {
            std::lock_guard<std::mutex> g(g_pcg_mu);
            auto                        it = g_pcg_cache.find(A);
            if(it == g_pcg_cache.end())
                it = g_pcg_cache.emplace(A, new pcg_ws()).first;
            w = it->second;
        }
        LAB_TRY(ensure_pcg_ws(w, A, s));
        cudaEvent_t t0, t1;
        cudaEventCreate(&t0);
        cudaEventCreate(&t1);
        cudaEventRecord(t0, s);
        const int* noskip = nullptr;
        // r = b - A x; r0 = ||r||_inf; z = M r; gamma = (z, r); p = z
        op_residual opr{x, b, w->r};
        LAB_TRY(launch_rowop(A, A->val, opr, s));
        LAB_TRY(norm_inf_device(A->m, w->r, rbuf(w, 4, w->sc + S_R0, noskip), s));
        LAB_TRY(precond_apply(M, w->r, w->z, s, noskip, rbuf(w, 2, w->sc + S_GNEW, noskip)));
        LAB_CUDA(cudaMemcpyAsync(w->p, w->z, sizeof(double) * A->m, cudaMemcpyDeviceToDevice, s));
        LAB_LAUNCH(k_pcg_init, 1, 1, 0, s, w->sc, w->flags, ctl->rel_tol, ctl->abs_tol,
                   ctl->max_iter);

        // iteration graph (rebuilt when the operands change): the whole iteration
        // loop as one graph launch (conditional WHILE node, bounded by max_iter + 1
        // passes), or, where conditional nodes are unavailable, one iteration per
        // launch driven by the host
        const int max_launch = ctl->max_iter + 1;
        if(!w->graph || w->key_M != M->uid || w->key_x != x || w->key_A != A->uid ||
           w->key_lim != max_launch)
        {
            if(w->graph)
                cudaGraphExecDestroy(w->graph);
            w->graph         = nullptr;
            const int64_t l0 = g_launches.load();
            lab_status    st = w->host_loop
                                   ? LAB_NOT_SUPPORTED
                                   : build_loop_graph(
                                         w->cap, w->flags + F_DONE, w->flags + F_LOOP, max_launch,
                                         [&](cudaStream_t c) { return pcg_iteration(A, M, x, w, c); },
                                         &w->graph, &w->graph_nodes);
            if(st == LAB_NOT_SUPPORTED)
            {
                w->host_loop = 1;
                cudaGraph_t g = nullptr;
                LAB_CUDA(cudaStreamBeginCapture(w->cap, cudaStreamCaptureModeThreadLocal));
                st             = pcg_iteration(A, M, x, w, w->cap);
                cudaError_t ce = cudaStreamEndCapture(w->cap, &g);
                if(st != LAB_OK && g)
                    cudaGraphDestroy(g);
                LAB_TRY(st);
                LAB_CUDA(ce);
                size_t nodes = 0;
                cudaGraphGetNodes(g, nullptr, &nodes);
                w->graph_nodes = (int64_t)nodes;
                ce             = cudaGraphInstantiate(&w->graph, g, 0);
                cudaGraphDestroy(g);
                LAB_CUDA(ce);
            }
            LAB_TRY(st);
            // launches counted while capturing are counted again as they run
            g_launches.fetch_sub(g_launches.load() - l0);
            w->key_M   = M->uid;
            w->key_x   = x;
            w->key_A   = A->uid;
            w->key_s   = s;
            w->key_lim = max_launch;
        }
        if(!w->host_loop)
        {
            LAB_CUDA(cudaGraphLaunch(w->graph, s));
        }
        else
        {
            // Pipelined host loop: iteration k+1 is queued before the flags of
            // iteration k are inspected; a queued iteration after convergence is a
            // no-op because every kernel checks flags[F_DONE] first.
            for(int launched = 0; launched < max_launch; launched++)
            {
                LAB_CUDA(cudaGraphLaunch(w->graph, s));
                g_launches.fetch_add(w->graph_nodes, std::memory_order_relaxed);
                int slot = launched & 1;
                LAB_CUDA(cudaMemcpyAsync(w->hflags + slot * F_COUNT, w->flags,
                                         sizeof(int) * F_COUNT, cudaMemcpyDeviceToHost, s));
                LAB_CUDA(cudaEventRecord(w->ev[slot], s));
                if(launched >= 1)
                {
                    int prev = (launched - 1) & 1;
                    LAB_CUDA(cudaEventSynchronize(w->ev[prev]));
                    if(w->hflags[prev * F_COUNT + F_DONE])
                        break;
                }
            }
        }
        cudaEventRecord(t1, s);
        int    hf[F_COUNT];
        double hs[S_COUNT];
        LAB_TRY(copy_d2h_sync(hf, w->flags, sizeof(hf), s));
        LAB_TRY(copy_d2h_sync(hs, w->sc, sizeof(hs), s));
        if(!w->host_loop) // the loop's passes ran on the device: prologue + passes x body
            g_launches.fetch_add(1 + (int64_t)hf[F_LOOP] * w->graph_nodes,
                                 std::memory_order_relaxed);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, t0, t1);
        cudaEventDestroy(t0);
        cudaEventDestroy(t1);
        lab_status status = hf[F_DONE] ? (lab_status)hf[F_STATUS] : LAB_NOT_CONVERGED;
        if(info)
        {
            info->iterations       = hf[F_ITER];
            info->converged        = hf[F_CONV];
            info->initial_residual = hs[S_R0];
            info->final_residual   = hs[S_RN];
            info->solve_ms         = ms;
            info->status           = status;
        }
        return status;
    }

    // Unpreconditioned CG as the reference runs it (cg.cpp:60-134): with
    // restart_iter = -1, `iter % restart_iter == 0` holds for every iter > 0, so
    // each iteration restarts from the true residual (steepest descent).
    // Mixed precision: FP64 iterative refinement around flexible PCG with the
    // reduced-precision cycle.  Each outer step recomputes the true residual
    // r = b - A x in FP64, applies the reference's stopping test to it, solves
    // A e = r by PCG (FP64 vectors, scalars and dots; FP32 / BF16 cycle; flexible
    // beta) to what is still needed, and corrects x += e.  Usually one pass
    // suffices; the outer FP64 check catches a recurrence residual that drifted
    // from the true one.
    static lab_status pcg_refine(lab_csr_impl* A, precond_impl* M, const double* b, double* x,
                                 const lab_iter_control* ctl, lab_solve_info* info,
                                 cudaStream_t s)
    {
        const int64_t m = A->m;
        pcg_ws*       w = nullptr;
        {
            std::lock_guard<std::mutex> g(g_pcg_mu);
            auto                        it = g_pcg_cache.find(A);
            if(it == g_pcg_cache.end())
                it = g_pcg_cache.emplace(A, new pcg_ws()).first;
            w = it->second;
        }
        if(!w->ir_r)
        {
            LAB_TRY(dalloc(&w->ir_r, (size_t)m + 1, s));
            LAB_TRY(dalloc(&w->ir_e, (size_t)m + 1, s));
            LAB_TRY(dalloc(&w->ir_sc, (size_t)kRedBlocks + 4, s));
            LAB_TRY(dalloc(&w->ir_cnt, 2, s));
            LAB_CUDA(cudaMemsetAsync(w->ir_cnt, 0, sizeof(unsigned int) * 2, s));
        }
        double* r  = w->ir_r;
        double* e  = w->ir_e;
        double* sc = w->ir_sc;
        red_buf rb{w->ir_sc + 4, w->ir_cnt, w->ir_sc, nullptr};
        cudaEvent_t t0, t1;
        cudaEventCreate(&t0);
        cudaEventCreate(&t1);
        cudaEventRecord(t0, s);
        double r0 = 0.0, rn = 0.0, rprev = 0.0;
        int    total = 0, conv = 0;
        bool   nan   = false;
        lab_status st = LAB_OK;
        for(int outer = 0; outer < 50; outer++)
        {
            op_residual opr{x, b, r};
            if((st = launch_rowop(A, A->val, opr, s)) != LAB_OK)
                break;
            if((st = norm_inf_device(m, r, rb, s)) != LAB_OK)
                break;
            if((st = copy_d2h_sync(&rn, sc, sizeof(double), s)) != LAB_OK)
                break;
            if(outer == 0)
                r0 = rn;
            nan = std::isnan(rn) || std::isnan(r0);
            if(nan)
                break;
            if(rn <= ctl->abs_tol || rn / r0 <= ctl->rel_tol || rn == 0.0)
            {
                conv = 1;
                break;
            }
            if(total > ctl->max_iter)
                break;
            if(outer > 0 && !(rn < 0.5 * rprev))
                break; // the last correction did not help: stop, not converged
            rprev                  = rn;
            lab_iter_control inner = *ctl;
            inner.abs_tol          = ctl->abs_tol;
            inner.rel_tol          = ctl->rel_tol * r0 / rn;
            inner.max_iter         = ctl->max_iter - total;
            lab_solve_info ii{};
            cudaMemsetAsync(e, 0, sizeof(double) * m, s);
            st = pcg_solve(A, M, r, e, &inner, &ii, s);
            if(st != LAB_OK && st != LAB_NOT_CONVERGED)
                break;
            st = LAB_OK;
            total += ii.iterations + (ii.converged ? 0 : 1);
            if((st = lab_axpy(m, 1.0, e, x, s)) != LAB_OK)
                break;
        }
        cudaEventRecord(t1, s);
        cudaEventSynchronize(t1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, t0, t1);
        cudaEventDestroy(t0);
        cudaEventDestroy(t1);
        if(st != LAB_OK)
            return st;
        lab_status status = conv ? LAB_OK : (nan ? LAB_NAN : LAB_NOT_CONVERGED);
        if(status == LAB_NAN)
            set_error("pcg: NaN/Inf residual after %d iterations", total);
        if(info)
        {
            info->iterations       = total;
            info->converged        = conv;
            info->initial_residual = r0;
            info->final_residual   = rn;
            info->solve_ms         = ms;
            info->status           = status;
        }
        return status;
    }

    static lab_status cg_plain(lab_csr_impl* A, const double* b, double* x,
                               const lab_iter_control* ctl, lab_solve_info* info, cudaStream_t s)
    {
        LAB_TRY(spmv_analyse(A, s));
        pcg_ws* w = nullptr;
        {
            std::lock_guard<std::mutex> g(g_pcg_mu);
            auto                        it = g_pcg_cache.find(A);
            if(it == g_pcg_cache.end())
                it = g_pcg_cache.emplace(A, new pcg_ws()).first;
            w = it->second;
        }
        LAB_TRY(ensure_pcg_ws(w, A, s));
        cudaEvent_t t0, t1;
        cudaEventCreate(&t0);
        cudaEventCreate(&t1);
        cudaEventRecord(t0, s);
        const int* skip = w->flags + F_DONE;
        op_residual opr{x, b, w->r};
        LAB_TRY(launch_rowop(A, A->val, opr, s));
        LAB_TRY(norm_inf_device(A->m, w->r, rbuf(w, 4, w->sc + S_R0, nullptr), s));
        LAB_TRY(dot_device(A->m, w->r, w->r, rbuf(w, 2, w->sc + S_GNEW, nullptr), s));
        LAB_CUDA(cudaMemcpyAsync(w->p, w->r, sizeof(double) * A->m, cudaMemcpyDeviceToDevice, s));
        LAB_LAUNCH(k_pcg_init, 1, 1, 0, s, w->sc, w->flags, ctl->rel_tol, ctl->abs_tol,
                   ctl->max_iter);
        for(int it = 0; it <= ctl->max_iter; it++)
        {
            if(it > 0)
            {
                op_residual opr2{x, b, w->r};
                red_buf     rb;
                rb.skip = skip;
                LAB_TRY(launch_rowop(A, A->val, opr2, s, rb));
                LAB_LAUNCH(k_copy_d, grid_for(A->m), 256, 0, s, w->p, (const double*)w->r, A->m,
                           skip);
                LAB_TRY(dot_device(A->m, w->r, w->r, rbuf(w, 2, w->sc + S_GNEW, skip), s));
                LAB_LAUNCH(k_pcg_setflags_for_plain, 1, 1, 0, s, w->sc, w->flags);
            }
            op_spmv_dot op{w->p, w->q};
            LAB_TRY(launch_rowop(A, A->val, op, s, rbuf(w, 0, w->sc + S_PQ, skip)));
            LAB_LAUNCH(k_pcg_update, red_grid(A->m), 256, 0, s, A->m, x, w->r, (const double*)w->p,
                       (const double*)w->q, w->sc, w->flags, w->partial + w->partial_n,
                       w->counters + 1);
            // gamma = (r, r), beta, p update as the reference (overwritten by the restart)
            LAB_TRY(dot_device(A->m, w->r, w->r, rbuf(w, 2, w->sc + S_GNEW, skip), s));
            LAB_LAUNCH(k_pcg_pupdate<false>, red_grid(A->m), 256, 0, s, A->m, w->p, (const double*)w->r,
                       w->sc, w->flags, w->counters + 3);
            if((it & 7) == 7)
            {
                int hf[F_COUNT];
                LAB_TRY(copy_d2h_sync(hf, w->flags, sizeof(hf), s));
                if(hf[F_DONE])
                    break;
            }
        }
        cudaEventRecord(t1, s);
        int    hf[F_COUNT];
        double hs[S_COUNT];
        LAB_TRY(copy_d2h_sync(hf, w->flags, sizeof(hf), s));
        LAB_TRY(copy_d2h_sync(hs, w->sc, sizeof(hs), s));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, t0, t1);
        cudaEventDestroy(t0);
        cudaEventDestroy(t1);
        lab_status status = hf[F_DONE] ? (lab_status)hf[F_STATUS] : LAB_NOT_CONVERGED;
        if(info)
        {
            info->iterations       = hf[F_ITER];
            info->converged        = hf[F_CONV];
            info->initial_residual = hs[S_R0];
            info->final_residual   = hs[S_RN];
            info->solve_ms         = ms;
            info->status           = status;
        }
        return status;
    }

    // ================================================================ stationary AMG
    static lab_status amg_solve(hierarchy_impl* h, const lab_amg_options* o, const double* b,
                                double* x, const lab_iter_control* ctl, lab_solve_info* info,
                                cudaStream_t s)
    {
        LAB_TRY(cycle_prepare(h, o, s));
        lab_csr_impl* A = h->A[0];
        pcg_ws*       w = nullptr;
        {
            std::lock_guard<std::mutex> g(g_pcg_mu);
            auto                        it = g_pcg_cache.find(h);
            if(it == g_pcg_cache.end())
                it = g_pcg_cache.emplace(h, new pcg_ws()).first;
            w = it->second;
        }
        LAB_TRY(ensure_pcg_ws(w, A, s));
        cudaEvent_t t0, t1;
        cudaEventCreate(&t0);
        cudaEventCreate(&t1);
        cudaEventRecord(t0, s);
        cyc_ctx c{o, s, nullptr};
        op_residual opr{x, b, w->r};
        LAB_TRY(launch_rowop(A, A->val, opr, s));
        LAB_TRY(norm_inf_device(A->m, w->r, rbuf(w, 4, w->sc + S_R0, nullptr), s));
        double r0 = 0.0, rn = 0.0;
        LAB_TRY(copy_d2h_sync(&r0, w->sc + S_R0, sizeof(double), s));
        int  cyc  = 0;
        bool conv = false, nan = false;
        // amg.cpp:539-563
        while(!(cyc > ctl->max_cycle))
        {
            LAB_TRY(cycle_iterate(h, c, b, x));
            op_residual opr2{x, b, w->r};
            LAB_TRY(launch_rowop(A, A->val, opr2, s));
            LAB_TRY(norm_inf_device(A->m, w->r, rbuf(w, 4, w->sc + S_RN, nullptr), s));
            LAB_TRY(copy_d2h_sync(&rn, w->sc + S_RN, sizeof(double), s));
            nan = std::isnan(rn) || std::isnan(r0);
            if(!nan && (rn <= ctl->abs_tol || rn / r0 <= ctl->rel_tol))
            {
                conv = true;
                break;
            }
            if(nan)
                break;
            cyc++;
        }
        cudaEventRecord(t1, s);
        cudaEventSynchronize(t1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, t0, t1);
        cudaEventDestroy(t0);
        cudaEventDestroy(t1);
        lab_status status = conv ? LAB_OK : (nan ? LAB_NAN : LAB_NOT_CONVERGED);
        if(status == LAB_NAN)
            set_error("amg_solve: NaN/Inf residual after %d cycles", cyc);
        if(info)
        {
            info->iterations       = cyc;
            info->converged        = conv;
            info->initial_residual = r0;
            info->final_residual   = rn;
            info->solve_ms         = ms;
            info->status           = status;
        }
        return status;
    }

    // ================================================================ GMRES
    __global__ void __launch_bounds__(256)
        k_multidot(int64_t n, int k, const double* __restrict__ Q, const double* __restrict__ w,
                   double* __restrict__ partial, int nblk)
    {
        // partial[j * nblk + block] = sum over the block's slice of Q_j . w
        for(int j = 0; j < k; j++)
        {
            double acc = 0.0;
            for(int64_t i = blockIdx.x * 256ll + threadIdx.x; i < n; i += (int64_t)gridDim.x * 256)
                acc += Q[(size_t)j * n + i] * w[i];
            double b = block_sum<256>(acc);
            if(threadIdx.x == 0)
                partial[(size_t)j * nblk + blockIdx.x] = b;
        }
    }

    __global__ void k_multidot_finish(const double* partial, int nblk, int k, double* h)
    {
        int j = blockIdx.x;
        if(j >= k)
            return;
        double s = 0.0;
        for(int b = threadIdx.x; b < nblk; b += 256)
            s += partial[(size_t)j * nblk + b];
        s = block_sum<256>(s);
        if(threadIdx.x == 0)
            h[j] = s;
    }

    // w -= Q h (k vectors)
    __global__ void k_qh_sub(int64_t n, int k, const double* __restrict__ Q,
                             const double* __restrict__ h, double* __restrict__ w)
    {
        for(int64_t i = blockIdx.x * 256ll + threadIdx.x; i < n; i += (int64_t)gridDim.x * 256)
        {
            double s = w[i];
            for(int j = 0; j < k; j++)
                s -= h[j] * Q[(size_t)j * n + i];
            w[i] = s;
        }
    }

    __global__ void k_scale(int64_t n, const double* __restrict__ x, double a, double* __restrict__ y)
    {
        for(int64_t i = blockIdx.x * 256ll + threadIdx.x; i < n; i += (int64_t)gridDim.x * 256)
            y[i] = x[i] * a;
    }

    // x += Q y (k vectors)
    __global__ void k_qy_add(int64_t n, int k, const double* __restrict__ Q,
                             const double* __restrict__ y, double* __restrict__ x)
    {
        for(int64_t i = blockIdx.x * 256ll + threadIdx.x; i < n; i += (int64_t)gridDim.x * 256)
        {
            double s = x[i];
            for(int j = 0; j < k; j++)
                s += Q[(size_t)j * n + i] * y[j];
            x[i] = s;
        }
    }

    // Restarted GMRES(m) (gmres.cpp): Arnoldi with classical Gram-Schmidt applied
    // twice (two fused multi-dot / update passes, numerically on par with the
    // reference's modified Gram-Schmidt), Givens rotations and the back
    // substitution on the host, the 2-norm stopping test of the reference.
    // Left preconditioning z = M^-1 r as the reference intends (its Arnoldi step
    // discards the preconditioner output, gmres.cpp:121-134; here it is used).
    static lab_status gmres_solve(lab_csr_impl* A, precond_impl* M, int restart, const double* b,
                                  double* x, const lab_iter_control* ctl, lab_solve_info* info,
                                  cudaStream_t s)
    {
        const int64_t n = A->m;
        LAB_TRY(spmv_analyse(A, s));
        if(M && M->kind == 0)
            LAB_TRY(cycle_prepare(M->h, &M->o, s));
        restart = (int)std::min<int64_t>(restart, n - 1);
        if(restart < 1)
            restart = 1;
        const int    nblk = (int)red_grid(n);
        dbuf<double> Q, w, r, z, hdev, part, ydev, sc;
        LAB_TRY(Q.alloc((size_t)(restart + 1) * n, s));
        LAB_TRY(w.alloc((size_t)n, s));
        LAB_TRY(r.alloc((size_t)n, s));
        LAB_TRY(z.alloc((size_t)n, s));
        LAB_TRY(hdev.alloc((size_t)restart + 2, s));
        LAB_TRY(ydev.alloc((size_t)restart + 2, s));
        LAB_TRY(part.alloc((size_t)(restart + 2) * nblk, s));
        LAB_TRY(sc.alloc(4, s));
        dbuf<unsigned int> cnt;
        LAB_TRY(cnt.alloc(4, s));
        LAB_CUDA(cudaMemsetAsync(cnt.get(), 0, sizeof(unsigned int) * 4, s));
        red_buf rb{part.get(), cnt.get(), sc.get(), nullptr};
        cudaEvent_t t0, t1;
        cudaEventCreate(&t0);
        cudaEventCreate(&t1);
        cudaEventRecord(t0, s);

        std::vector<double> H((size_t)(restart + 1) * restart, 0.0), cs(restart), sn(restart),
            g(restart + 1), hcol(restart + 2);
        auto residual_vec = [&](double* out, double& nrm) -> lab_status {
            op_residual opr{x, b, r.get()};
            LAB_TRY(launch_rowop(A, A->val, opr, s));
            const double* v = r.get();
            if(M)
            {
                LAB_TRY(precond_apply(M, r.get(), out, s, nullptr, red_buf()));
                v = out;
            }
            else
                LAB_CUDA(cudaMemcpyAsync(out, r.get(), sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
            LAB_TRY(dot_device(n, v, v, rb, s));
            double d2 = 0;
            LAB_TRY(copy_d2h_sync(&d2, sc.get(), sizeof(double), s));
            nrm = std::sqrt(d2);
            return LAB_OK;
        };
        auto converges = [&](double rn, double r0) {
            if(std::isnan(rn) || std::isnan(r0))
                return false;
            return rn <= ctl->abs_tol || rn / r0 <= ctl->rel_tol;
        };
        double rn = 0;
        LAB_TRY(residual_vec(z.get(), rn));
        const double r0   = rn;
        int          iter = 0;
        bool         conv = converges(rn, r0);
        bool         bad  = std::isnan(rn);
        while(!conv && !bad && !(iter > ctl->max_iter))
        {
            LAB_LAUNCH(k_scale, red_grid(n), 256, 0, s, n, (const double*)z.get(), 1.0 / rn, Q.get());
            std::fill(g.begin(), g.end(), 0.0);
            g[0]  = rn;
            int k = 1;
            for(k = 1; k <= restart; k++)
            {
                double* qk   = Q.get() + (size_t)k * n;
                double* qkm1 = Q.get() + (size_t)(k - 1) * n;
                if(M)
                {
                    op_spmv ops{qkm1, w.get(), 1.0, 0.0};
                    LAB_TRY(launch_rowop(A, A->val, ops, s));
                    LAB_TRY(precond_apply(M, w.get(), qk, s, nullptr, red_buf()));
                }
                else
                {
                    op_spmv ops{qkm1, qk, 1.0, 0.0};
                    LAB_TRY(launch_rowop(A, A->val, ops, s));
                }
                std::fill(hcol.begin(), hcol.end(), 0.0);
                for(int pass = 0; pass < 2; pass++)
                {
                    LAB_LAUNCH(k_multidot, nblk, 256, 0, s, n, k, (const double*)Q.get(),
                               (const double*)qk, part.get(), nblk);
                    LAB_LAUNCH(k_multidot_finish, k, 256, 0, s, (const double*)part.get(), nblk, k,
                               hdev.get());
                    LAB_LAUNCH(k_qh_sub, red_grid(n), 256, 0, s, n, k, (const double*)Q.get(),
                               (const double*)hdev.get(), qk);
                    std::vector<double> hh(k);
                    LAB_TRY(copy_d2h_sync(hh.data(), hdev.get(), sizeof(double) * k, s));
                    for(int i = 0; i < k; i++)
                        hcol[i] += hh[i];
                }
                LAB_TRY(dot_device(n, qk, qk, rb, s));
                double vv = 0;
                LAB_TRY(copy_d2h_sync(&vv, sc.get(), sizeof(double), s));
                hcol[k] = std::sqrt(vv);
                if(hcol[k] != 0.0)
                    LAB_LAUNCH(k_scale, red_grid(n), 256, 0, s, n, (const double*)qk, 1.0 / hcol[k], qk);
                for(int i = 0; i <= k; i++)
                    H[(size_t)i + (size_t)(k - 1) * (restart + 1)] = hcol[i];
                // gmres.cpp:163-199: Givens rotations
                auto Hc = [&](int i) -> double& { return H[(size_t)i + (size_t)(k - 1) * (restart + 1)]; };
                for(int i = 0; i < k - 1; i++)
                {
                    double t1v = Hc(i), t2v = Hc(i + 1);
                    Hc(i)      = cs[i] * t1v + sn[i] * t2v;
                    Hc(i + 1)  = -sn[i] * t1v + cs[i] * t2v;
                }
                double xi = Hc(k - 1), xj = Hc(k);
                if(xi == 0.0)
                {
                    cs[k - 1] = 0.0;
                    sn[k - 1] = 1.0;
                }
                else if(xj == 0.0)
                {
                    cs[k - 1] = 1.0;
                    sn[k - 1] = 0.0;
                }
                else if(std::abs(xi) > std::abs(xj))
                {
                    double t  = xj / xi;
                    cs[k - 1] = 1.0 / std::sqrt(1.0 + t * t);
                    sn[k - 1] = t * cs[k - 1];
                }
                else
                {
                    double t  = xi / xj;
                    sn[k - 1] = 1.0 / std::sqrt(1.0 + t * t);
                    cs[k - 1] = t * sn[k - 1];
                }
                double t1v = Hc(k - 1), t2v = Hc(k);
                Hc(k - 1)  = cs[k - 1] * t1v + sn[k - 1] * t2v;
                Hc(k)      = -sn[k - 1] * t1v + cs[k - 1] * t2v;
                g[k]       = -sn[k - 1] * g[k - 1];
                g[k - 1]   = cs[k - 1] * g[k - 1];
                if(converges(std::abs(g[k]), r0) || k == restart)
                    break;
            }
            if(k > restart)
                k = restart;
            // back substitution (gmres.cpp:290-298)
            std::vector<double> y(g.begin(), g.begin() + k);
            for(int i = k - 1; i >= 0; i--)
            {
                for(int j = i + 1; j < k; j++)
                    y[i] -= H[(size_t)i + (size_t)(restart + 1) * j] * y[j];
                y[i] /= H[(size_t)i + (size_t)(restart + 1) * i];
            }
            LAB_CUDA(cudaMemcpyAsync(ydev.get(), y.data(), sizeof(double) * k, cudaMemcpyHostToDevice, s));
            LAB_LAUNCH(k_qy_add, red_grid(n), 256, 0, s, n, k, (const double*)Q.get(),
                       (const double*)ydev.get(), x);
            LAB_TRY(residual_vec(z.get(), rn));
            bad = std::isnan(rn);
            if(converges(rn, r0))
            {
                conv = true;
                break;
            }
            iter++;
        }
        cudaEventRecord(t1, s);
        cudaEventSynchronize(t1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, t0, t1);
        cudaEventDestroy(t0);
        cudaEventDestroy(t1);
        lab_status status = conv ? LAB_OK : (bad ? LAB_NAN : LAB_NOT_CONVERGED);
        if(status == LAB_NAN)
            set_error("gmres: NaN/Inf residual after %d iterations", iter);
        if(info)
        {
            info->iterations       = iter;
            info->converged        = conv;
            info->initial_residual = r0;
            info->final_residual   = rn;
            info->solve_ms         = ms;
            info->status           = status;
        }
        return status;
    }
}

namespace lab
{
    // ================================================================ segmented PCG
    // Batched systems and multi-RHS solves share one machinery: the vectors are
    // split into `nseg` segments (a system's rows, or one right-hand side), each
    // with its own scalars and stopping test.  Every segmented kernel runs on a
    // (K, nseg) grid: K CTAs per segment, each over a fixed contiguous chunk, the
    // last CTA of a segment (per-segment ticket) reducing the K partials in order
    // -- deterministic, and a converged segment is skipped (convergence mask).
    constexpr int kSegK = 8;
    enum
    {
        G_GAMMA = 0,
        G_PQ    = 1,
        G_RN    = 2,
        G_R0    = 3,
        G_GNEW  = 4,
        G_N     = 8
    };
    enum
    {
        GF_DONE   = 0,
        GF_ITER   = 1,
        GF_CONV   = 2,
        GF_STATUS = 3,
        GF_N      = 4
    };
    // global flags: [0] = all done, [1] = active segments, [2] = max_iter,
    // [3] = passes of the device-side iteration loop
    struct seg_ws
    {
        int           nseg   = 0;
        int64_t       total  = 0;
        int64_t*      off    = nullptr; // device [nseg + 1]
        double *      r = nullptr, *z = nullptr, *p = nullptr, *q = nullptr;
        double*       sc      = nullptr; // [nseg][G_N]
        int*          sf      = nullptr; // [nseg][GF_N]
        int*          gflags  = nullptr; // [4]
        double*       partial = nullptr; // [4 slots][nseg][kSegK]
        unsigned int* tickets = nullptr; // [4 slots][nseg]
        double        rtol = 0, atol = 0;
        void release()
        {
            void* ps[] = {off, r, z, p, q, sc, sf, gflags, partial, tickets};
            for(void* x : ps)
                if(x)
                    cudaFree(x);
        }
    };

    __device__ __forceinline__ void seg_range(const int64_t* off, int s, int k, int64_t& a,
                                              int64_t& b)
    {
        const int64_t s0 = off[s], s1 = off[s + 1];
        const int64_t ch = (s1 - s0 + kSegK - 1) / kSegK;
        a                = s0 + k * ch;
        b                = min(s1, a + ch);
    }

    // Per-segment ticket: true in every thread of the segment's last CTA.
    __device__ __forceinline__ bool seg_ticket(unsigned int* t)
    {
        __shared__ bool last;
        __syncthreads();
        if(threadIdx.x == 0)
        {
            __threadfence();
            last = atomicAdd(t, 1u) == kSegK - 1;
        }
        __syncthreads();
        return last;
    }

    // (x, y) per segment -> sc[s][slot]; OP 1: max |x|
    template <int OP>
    __global__ void __launch_bounds__(256)
        k_seg_reduce(const int64_t* off, const double* __restrict__ x, const double* __restrict__ y,
                     double* sc, int slot, const int* sf, const int* gflags, double* partial,
                     unsigned int* tickets, int skip_done)
    {
        const int s = blockIdx.y, k = blockIdx.x, nseg = gridDim.y;
        if(gflags[0] || (skip_done && sf[s * GF_N + GF_DONE]))
            return;
        int64_t a, b;
        seg_range(off, s, k, a, b);
        double acc = 0.0;
        for(int64_t i = a + threadIdx.x; i < b; i += 256)
            acc = OP == 0 ? acc + x[i] * y[i] : nanmax(acc, fabs(x[i]));
        double bs = OP == 0 ? block_sum<256>(acc) : block_max<256>(acc);
        if(threadIdx.x == 0)
            partial[(size_t)s * kSegK + k] = bs;
        (void)nseg;
        if(seg_ticket(&tickets[s]))
        {
            if(threadIdx.x == 0)
            {
                double t = 0.0;
                for(int j = 0; j < kSegK; j++)
                {
                    double v = __ldcg(partial + (size_t)s * kSegK + j);
                    t        = OP == 0 ? t + v : nanmax(t, v);
                }
                sc[s * G_N + slot] = t;
                tickets[s]         = 0;
            }
        }
    }

    __device__ __forceinline__ void seg_retire(int* sf, int s, int* gflags, int status, int conv)
    {
        sf[s * GF_N + GF_DONE]   = 1;
        sf[s * GF_N + GF_CONV]   = conv;
        sf[s * GF_N + GF_STATUS] = status;
        if(atomicSub(&gflags[1], 1) == 1)
            gflags[0] = 1;
    }

    // x += alpha p; r -= alpha q; ||r||_inf; stopping test, per segment.
    __global__ void __launch_bounds__(256)
        k_seg_update(const int64_t* off, double* __restrict__ x, double* __restrict__ r,
                     const double* __restrict__ p, const double* __restrict__ q, double* sc,
                     int* sf, int* gflags, double* partial, unsigned int* tickets, double rtol,
                     double atol)
    {
        const int s = blockIdx.y, k = blockIdx.x;
        if(gflags[0] || sf[s * GF_N + GF_DONE])
            return;
        const double alpha = sc[s * G_N + G_GAMMA] / sc[s * G_N + G_PQ];
        const double na    = -1.0 * alpha;
        int64_t      a, b;
        seg_range(off, s, k, a, b);
        double acc = 0.0;
        for(int64_t i = a + threadIdx.x; i < b; i += 256)
        {
            x[i]      = alpha == 1.0 ? __dadd_rn(p[i], x[i]) : __dadd_rn(__dmul_rn(alpha, p[i]), x[i]);
            double ri = na == 1.0 ? __dadd_rn(q[i], r[i]) : __dadd_rn(__dmul_rn(na, q[i]), r[i]);
            r[i]      = ri;
            acc       = nanmax(acc, fabs(ri));
        }
        double bs = block_max<256>(acc);
        if(threadIdx.x == 0)
            partial[(size_t)s * kSegK + k] = bs;
        if(seg_ticket(&tickets[s]))
        {
            if(threadIdx.x == 0)
            {
                double t = 0.0;
                for(int j = 0; j < kSegK; j++)
                    t = nanmax(t, __ldcg(partial + (size_t)s * kSegK + j));
                tickets[s]          = 0;
                sc[s * G_N + G_RN]  = t;
                double r0           = sc[s * G_N + G_R0];
                bool   nan          = isnan(t) || isnan(r0);
                if(!nan && (t <= atol || t / r0 <= rtol))
                    seg_retire(sf, s, gflags, LAB_OK, 1);
                else if(nan)
                    seg_retire(sf, s, gflags, LAB_NAN, 0);
            }
        }
    }

    // p = z + beta p, gamma <- gnew, iteration count, max_iter test, per segment.
    __global__ void __launch_bounds__(256)
        k_seg_pupdate(const int64_t* off, double* __restrict__ p, const double* __restrict__ z,
                      double* sc, int* sf, int* gflags, unsigned int* tickets)
    {
        const int s = blockIdx.y, k = blockIdx.x;
        if(gflags[0] || sf[s * GF_N + GF_DONE])
            return;
        const double beta = sc[s * G_N + G_GNEW] / sc[s * G_N + G_GAMMA];
        int64_t      a, b;
        seg_range(off, s, k, a, b);
        for(int64_t i = a + threadIdx.x; i < b; i += 256)
            p[i] = beta == 0.0 ? z[i] : __dadd_rn(z[i], __dmul_rn(beta, p[i]));
        if(seg_ticket(&tickets[s]))
        {
            if(threadIdx.x == 0)
            {
                tickets[s]            = 0;
                sc[s * G_N + G_GAMMA] = sc[s * G_N + G_GNEW];
                int it                = sf[s * GF_N + GF_ITER] + 1;
                sf[s * GF_N + GF_ITER] = it;
                if(it > gflags[2])
                    seg_retire(sf, s, gflags, LAB_NOT_CONVERGED, 0);
            }
        }
    }

    __global__ void k_seg_init(double* sc, int* sf, int* gflags, int nseg, int max_iter)
    {
        int active = 0;
        for(int s = 0; s < nseg; s++)
        {
            sc[s * G_N + G_GAMMA]    = sc[s * G_N + G_GNEW];
            sc[s * G_N + G_RN]       = sc[s * G_N + G_R0];
            sf[s * GF_N + GF_ITER]   = 0;
            bool zero                = sc[s * G_N + G_R0] == 0.0;
            sf[s * GF_N + GF_DONE]   = zero;
            sf[s * GF_N + GF_CONV]   = zero;
            sf[s * GF_N + GF_STATUS] = zero ? LAB_OK : LAB_NOT_CONVERGED;
            active += !zero;
        }
        gflags[1] = active;
        gflags[2] = max_iter;
        gflags[0] = active == 0;
    }

    // Operator products for the two segmentations.
    struct seg_ops
    {
        lab_csr_impl* A     = nullptr;
        precond_impl* M     = nullptr;
        int           multi = 0; // 0: stacked systems, 1: nseg columns of one matrix
        int64_t       n     = 0; // rows of A (multi-RHS column length)
        int           block = 0; // multi-RHS: block V-cycle over up to 8 columns per pass
    };

    static lab_status seg_apply_A(const seg_ops& o, seg_ws& w, const double* in, double* out,
                                  cudaStream_t s, const int* skip)
    {
        if(!o.multi)
        {
            op_spmv op{in, out, 1.0, 0.0};
            red_buf rb;
            rb.skip = skip;
            return launch_rowop(o.A, o.A->val, op, s, rb);
        }
        lab_csr_impl* A = o.A;
        for(int c = 0; c < w.nseg; c += 8)
        {
            int k = std::min(8, w.nseg - c);
            LAB_TRY(spmm_columns(A, k, in + (int64_t)c * o.n, o.n, out + (int64_t)c * o.n, o.n,
                                 s, skip));
        }
        return LAB_OK;
    }

    static lab_status seg_apply_M(const seg_ops& o, seg_ws& w, const double* r, double* z,
                                  cudaStream_t s, const int* skip)
    {
        if(!o.multi)
            return precond_apply(o.M, r, z, s, skip, red_buf());
        if(o.block)
        {
            cyc_ctx c{&o.M->o, s, skip};
            return cycle_precond_block(o.M->h, c, w.nseg, r, o.n, z, o.n);
        }
        for(int c = 0; c < w.nseg; c++)
            LAB_TRY(precond_apply(o.M, r + (int64_t)c * o.n, z + (int64_t)c * o.n, s, skip,
                                  red_buf()));
        return LAB_OK;
    }

    static lab_status seg_solve(const seg_ops& o, int nseg, const int64_t* offsets_h,
                                const double* b, double* x, const lab_iter_control* ctl,
                                int* iters_h, int* conv_h, lab_solve_info* info, cudaStream_t s)
    {
        seg_ws w;
        w.nseg  = nseg;
        w.total = offsets_h[nseg];
        lab_status st = LAB_OK;
        auto       al = [&](auto** p, size_t n) {
            if(st == LAB_OK)
                st = dalloc(p, n, s);
        };
        al(&w.off, (size_t)nseg + 1);
        al(&w.r, (size_t)w.total + 1);
        al(&w.z, (size_t)w.total + 1);
        al(&w.p, (size_t)w.total + 1);
        al(&w.q, (size_t)w.total + 1);
        al(&w.sc, (size_t)nseg * G_N);
        al(&w.sf, (size_t)nseg * GF_N);
        al(&w.gflags, 4);
        al(&w.partial, (size_t)4 * nseg * kSegK);
        al(&w.tickets, (size_t)4 * nseg);
        if(st != LAB_OK)
        {
            w.release();
            return st;
        }
        cudaMemcpyAsync(w.off, offsets_h, sizeof(int64_t) * (nseg + 1), cudaMemcpyHostToDevice, s);
        cudaMemsetAsync(w.tickets, 0, sizeof(unsigned int) * 4 * nseg, s);
        cudaMemsetAsync(w.gflags, 0, sizeof(int) * 4, s);
        cudaMemsetAsync(w.sf, 0, sizeof(int) * nseg * GF_N, s);
        const dim3 grid(kSegK, nseg);
        const int* skip = w.gflags;
        auto       red  = [&](int slotbuf) { return w.partial + (size_t)slotbuf * nseg * kSegK; };
        auto       tik  = [&](int slotbuf) { return w.tickets + (size_t)slotbuf * nseg; };

        cudaEvent_t t0, t1;
        cudaEventCreate(&t0);
        cudaEventCreate(&t1);
        cudaEventRecord(t0, s);
        cudaGraphExec_t gexec = nullptr;
        cudaStream_t    cap   = nullptr;
        int*            hf    = nullptr;
        cudaEvent_t     ev[2] = {nullptr, nullptr};
        do
        {
            // r = b - A x, r0 = ||r||, z = M r, gamma = (z, r), p = z
            if(!o.multi)
            {
                op_residual opr{x, b, w.r};
                st = launch_rowop(o.A, o.A->val, opr, s);
            }
            else
            {
                st = seg_apply_A(o, w, x, w.q, s, nullptr);
                if(st == LAB_OK)
                {
                    cudaMemcpyAsync(w.r, b, sizeof(double) * w.total, cudaMemcpyDeviceToDevice, s);
                    st = lab_axpy(w.total, -1.0, w.q, w.r, s); // r = b - A x
                }
            }
            if(st != LAB_OK)
                break;
            k_seg_reduce<1><<<grid, 256, 0, s>>>(w.off, w.r, nullptr, w.sc, G_R0, w.sf, w.gflags,
                                                 red(0), tik(0), 0);
            st = seg_apply_M(o, w, w.r, w.z, s, nullptr);
            if(st != LAB_OK)
                break;
            k_seg_reduce<0><<<grid, 256, 0, s>>>(w.off, w.z, w.r, w.sc, G_GNEW, w.sf, w.gflags,
                                                 red(1), tik(1), 0);
            cudaMemcpyAsync(w.p, w.z, sizeof(double) * w.total, cudaMemcpyDeviceToDevice, s);
            k_seg_init<<<1, 1, 0, s>>>(w.sc, w.sf, w.gflags, nseg, ctl->max_iter);
            g_launches.fetch_add(4);

            // the iterations as one graph launch (a device-side WHILE loop of at
            // most max_iter + 1 passes that stops once every system has retired);
            // where conditional nodes are unavailable, one launch per iteration
            if(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking) != cudaSuccess)
            {
                st = LAB_CUDA_ERROR;
                break;
            }
            auto iteration = [&](cudaStream_t c) -> lab_status {
                lab_status r = seg_apply_A(o, w, w.p, w.q, c, skip);
                k_seg_reduce<0><<<grid, 256, 0, c>>>(w.off, w.p, w.q, w.sc, G_PQ, w.sf, w.gflags,
                                                     red(2), tik(2), 1);
                k_seg_update<<<grid, 256, 0, c>>>(w.off, x, w.r, w.p, w.q, w.sc, w.sf, w.gflags,
                                                  red(3), tik(3), ctl->rel_tol, ctl->abs_tol);
                if(r == LAB_OK)
                    r = seg_apply_M(o, w, w.r, w.z, c, skip);
                k_seg_reduce<0><<<grid, 256, 0, c>>>(w.off, w.z, w.r, w.sc, G_GNEW, w.sf, w.gflags,
                                                     red(1), tik(1), 1);
                k_seg_pupdate<<<grid, 256, 0, c>>>(w.off, w.p, w.z, w.sc, w.sf, w.gflags, tik(0));
                return r;
            };
            const int     limit = ctl->max_iter + 1;
            const int64_t l0    = g_launches.load();
            int64_t       nodes = 0;
            st = build_loop_graph(cap, w.gflags, w.gflags + 3, limit, iteration, &gexec, &nodes);
            const bool device_loop = st == LAB_OK;
            if(st == LAB_NOT_SUPPORTED)
            {
                cudaGraph_t g = nullptr;
                if(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
                {
                    st = LAB_CUDA_ERROR;
                    break;
                }
                st             = iteration(cap);
                cudaError_t ce = cudaStreamEndCapture(cap, &g);
                if(st != LAB_OK || ce != cudaSuccess)
                {
                    if(g)
                        cudaGraphDestroy(g);
                    if(st == LAB_OK)
                        st = cuda_status(ce, "batched PCG capture", __FILE__, __LINE__);
                    break;
                }
                size_t n = 0;
                cudaGraphGetNodes(g, nullptr, &n);
                nodes = (int64_t)n;
                ce    = cudaGraphInstantiate(&gexec, g, 0);
                cudaGraphDestroy(g);
                if(ce != cudaSuccess)
                {
                    st = cuda_status(ce, "batched PCG instantiate", __FILE__, __LINE__);
                    break;
                }
            }
            if(st != LAB_OK)
                break;
            // launches counted while capturing are counted again as they run
            g_launches.fetch_sub(g_launches.load() - l0);
            if(device_loop)
            {
                if(cudaGraphLaunch(gexec, s) != cudaSuccess)
                {
                    st = LAB_CUDA_ERROR;
                    break;
                }
                int passes = 0;
                st         = copy_d2h_sync(&passes, w.gflags + 3, sizeof(int), s);
                g_launches.fetch_add(1 + (int64_t)passes * nodes);
                break;
            }
            if(cudaMallocHost(&hf, sizeof(int) * 8) != cudaSuccess)
            {
                st = LAB_OOM;
                break;
            }
            cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming);
            cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming);
            for(int it = 0; it < limit; it++)
            {
                if(cudaGraphLaunch(gexec, s) != cudaSuccess)
                {
                    st = LAB_CUDA_ERROR;
                    break;
                }
                g_launches.fetch_add(nodes);
                int slot = it & 1;
                cudaMemcpyAsync(hf + slot * 4, w.gflags, sizeof(int) * 4, cudaMemcpyDeviceToHost,
                                s);
                cudaEventRecord(ev[slot], s);
                if(it >= 1)
                {
                    cudaEventSynchronize(ev[(it - 1) & 1]);
                    if(hf[((it - 1) & 1) * 4])
                        break;
                }
            }
        } while(0);
        cudaEventRecord(t1, s);
        cudaStreamSynchronize(s);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, t0, t1);
        std::vector<int> sf((size_t)nseg * GF_N);
        if(st == LAB_OK)
            st = copy_d2h_sync(sf.data(), w.sf, sizeof(int) * sf.size(), s);
        if(gexec)
            cudaGraphExecDestroy(gexec);
        if(cap)
            cudaStreamDestroy(cap);
        if(hf)
            cudaFreeHost(hf);
        for(auto& e : ev)
            if(e)
                cudaEventDestroy(e);
        cudaEventDestroy(t0);
        cudaEventDestroy(t1);
        w.release();
        if(st != LAB_OK)
            return st;
        int maxit = 0, allconv = 1, nan = 0;
        for(int k = 0; k < nseg; k++)
        {
            if(iters_h)
                iters_h[k] = sf[k * GF_N + GF_ITER];
            if(conv_h)
                conv_h[k] = sf[k * GF_N + GF_CONV];
            maxit = std::max(maxit, sf[k * GF_N + GF_ITER]);
            allconv &= sf[k * GF_N + GF_CONV];
            nan |= sf[k * GF_N + GF_STATUS] == LAB_NAN;
        }
        lab_status status = allconv ? LAB_OK : (nan ? LAB_NAN : LAB_NOT_CONVERGED);
        if(status == LAB_NAN)
            set_error("segmented pcg: a system's residual became NaN/Inf");
        if(info)
        {
            info->iterations       = maxit;
            info->converged        = allconv;
            info->initial_residual = 0.0;
            info->final_residual   = 0.0;
            info->solve_ms         = ms;
            info->status           = status;
        }
        return status;
    }
}

using namespace lab;

struct lab_precond_s : precond_impl
{
};

extern "C" {

LAB_API void lab_amg_options_default(lab_amg_options* o)
{
    if(!o)
        return;
    o->n1        = 1;
    o->n2        = 1;
    o->cycle     = LAB_CYCLE_V;
    o->smoother  = LAB_SMOOTH_JACOBI;
    o->omega     = 1.0;
    o->omega_sor = 0.5;
    o->coarse    = LAB_COARSE_DIRECT;
    o->precision = LAB_PREC_FP64;
}

LAB_API void lab_iter_control_default(lab_iter_control* c)
{
    if(!c)
        return;
    c->rel_tol   = 1e-6;
    c->abs_tol   = 1e-6;
    c->max_iter  = 1000;
    c->max_cycle = 200;
}

static lab_status check_options(const lab_amg_options* o)
{
    LAB_ARG(o, "null options");
    LAB_ARG(o->n1 >= 0 && o->n2 >= 0 && o->n1 <= 64 && o->n2 <= 64, "smoothing sweeps in [0, 64]");
    LAB_ARG(o->cycle >= 0 && o->cycle <= 2, "unknown cycle");
    LAB_ARG(o->smoother >= 0 && o->smoother <= 4, "unknown smoother");
    LAB_ARG(o->coarse == 0 || o->coarse == 1, "unknown coarse solver");
    LAB_ARG(o->precision >= 0 && o->precision <= 2, "unknown precision");
    return LAB_OK;
}

LAB_API lab_status lab_amg_cycle(lab_hierarchy h, const lab_amg_options* o, const double* b,
                                 double* x, lab_stream ls)
{
    LAB_ARG(h && b && x, "null argument");
    LAB_TRY(check_options(o));
    LAB_TRY(ensure_init());
    cudaStream_t s = to_stream(ls);
    LAB_TRY(cycle_prepare(h, o, s));
    cyc_ctx c{o, s, nullptr};
    return cycle_iterate(h, c, b, x);
}

LAB_API lab_status lab_amg_solve(lab_hierarchy h, const lab_amg_options* o, const double* b,
                                 double* x, const lab_iter_control* c, lab_solve_info* info,
                                 lab_stream s)
{
    LAB_ARG(h && b && x && c, "null argument");
    LAB_TRY(check_options(o));
    LAB_TRY(ensure_init());
    return amg_solve(h, o, b, x, c, info, to_stream(s));
}

LAB_API lab_status lab_precond_create_amg(lab_hierarchy h, const lab_amg_options* o,
                                          lab_precond* out, lab_stream s)
{
    LAB_ARG(h && out, "null argument");
    LAB_TRY(check_options(o));
    LAB_TRY(ensure_init());
    lab_precond_s* M = new(std::nothrow) lab_precond_s();
    if(!M)
        return LAB_OOM;
    M->kind       = 0;
    M->h          = h;
    M->o          = *o;
    lab_status st = cycle_prepare(h, o, to_stream(s));
    if(st != LAB_OK)
    {
        delete M;
        return st;
    }
    *out = M;
    return LAB_OK;
}

LAB_API lab_status lab_precond_create_jacobi(lab_csr A, lab_precond* out, lab_stream s)
{
    LAB_ARG(A && out, "null argument");
    LAB_TRY(ensure_init());
    lab_precond_s* M = new(std::nothrow) lab_precond_s();
    if(!M)
        return LAB_OOM;
    M->kind       = 1;
    M->A          = A;
    lab_status st = csr_ensure_invdiag(A, to_stream(s));
    if(st != LAB_OK)
    {
        delete M;
        return st;
    }
    // a private copy: later value changes of A (lab_csr_values_changed frees and
    // rebuilds A's cached diagonal) leave the built preconditioner as it was
    st = dalloc(&M->diag, (size_t)A->m + 1, to_stream(s));
    if(st == LAB_OK && A->m > 0)
    {
        cudaError_t e = cudaMemcpyAsync(M->diag, A->diag, sizeof(double) * A->m,
                                        cudaMemcpyDeviceToDevice, to_stream(s));
        if(e != cudaSuccess)
            st = cuda_status(e, "jacobi diagonal copy", __FILE__, __LINE__);
    }
    if(st != LAB_OK)
    {
        delete M;
        return st;
    }
    *out = M;
    return LAB_OK;
}

// A triangular preconditioner's solves give up only if a row's dependencies never
// arrive (a bug, not an input property): report it over the solver's status.
static lab_status tri_status(lab_precond_s* M, lab_status st, cudaStream_t s)
{
    lab_status e = tri_check(M->F, s);
    if(e == LAB_OK && M->G)
        e = tri_check(M->G, s);
    return e != LAB_OK ? e : st;
}

// ILU(0) / IC(0): factor a copy of A (ilu_precond::build, preconditioner.cpp:432-450;
// ic_precond::build, 506-524).  Gauss-Seidel / SOR: solve with the lower part of
// a copy of A (gauss_seidel_precond::build 90-96, SOR_precond::build 137-147).
// SSOR: the two triangles L and U of SSOR_precond::build (283-353).
static lab_status create_tri_precond(lab_csr A, int kind, double omega, lab_precond* out,
                                     lab_stream ls)
{
    LAB_ARG(A && out, "null argument");
    LAB_ARG(A->m == A->n, "square matrix required");
    LAB_TRY(ensure_init());
    cudaStream_t   s = to_stream(ls);
    lab_precond_s* M = new(std::nothrow) lab_precond_s();
    if(!M)
        return LAB_OOM;
    M->kind       = kind;
    M->A          = A;
    M->dscale     = kind == 5 ? 1.0 / omega : 0.0; // SOR: scale_diagonal_by(1.0 / omega)
    // like the reference's build(), every kind works on its own copy of A (SSOR:
    // on the two triangles built from it)
    lab_csr    F  = nullptr;
    lab_status st = LAB_OK;
    if(kind == 6)
    {
        st = ssor_split(A, omega, &M->F, &M->G, s);
        if(st == LAB_OK)
            st = tri_analyse(M->G, s);
        if(st == LAB_OK)
            st = dalloc(&M->y, (size_t)A->m + 1, s);
    }
    else
    {
        st = lab_csr_clone(A, &F, ls);
        if(st == LAB_OK)
            M->F = F;
    }
    if(st == LAB_OK)
        st = tri_analyse(M->F, s);
    if(st == LAB_OK && (kind == 2 || kind == 3))
    {
        int sz = -1, nz = -1;
        st = tri_factor(M->F, kind == 3, &sz, &nz, s);
        if(st == LAB_OK)
            st = dalloc(&M->y, (size_t)A->m + 1, s);
    }
    if(st != LAB_OK)
    {
        delete M;
        return st;
    }
    *out = M;
    return LAB_OK;
}

LAB_API lab_status lab_precond_create_ilu0(lab_csr A, lab_precond* M, lab_stream s)
{
    return create_tri_precond(A, 2, 0.0, M, s);
}

LAB_API lab_status lab_precond_create_ic0(lab_csr A, lab_precond* M, lab_stream s)
{
    return create_tri_precond(A, 3, 0.0, M, s);
}

LAB_API lab_status lab_precond_create_gauss_seidel(lab_csr A, lab_precond* M, lab_stream s)
{
    return create_tri_precond(A, 4, 0.0, M, s);
}

LAB_API lab_status lab_precond_create_sor(lab_csr A, double omega, lab_precond* M, lab_stream s)
{
    LAB_ARG(omega > 0.0 && omega < 2.0, "SOR needs 0 < omega < 2");
    return create_tri_precond(A, 5, omega, M, s);
}

LAB_API lab_status lab_precond_create_ssor(lab_csr A, double omega, lab_precond* M, lab_stream s)
{
    LAB_ARG(omega > 0.0 && omega < 2.0, "SSOR needs 0 < omega < 2");
    return create_tri_precond(A, 6, omega, M, s);
}

LAB_API lab_status lab_precond_apply(lab_precond M, const double* r, double* z, lab_stream s)
{
    LAB_ARG(M && r && z, "null argument");
    LAB_TRY(ensure_init());
    return precond_apply(M, r, z, to_stream(s), nullptr, red_buf());
}

LAB_API lab_status lab_precond_destroy(lab_precond M)
{
    if(M)
    {
        cudaDeviceSynchronize();
        delete static_cast<lab_precond_s*>(M);
    }
    return LAB_OK;
}

LAB_API lab_status lab_pcg_solve(lab_csr A, lab_precond M, const double* b, double* x,
                                 const lab_iter_control* c, lab_solve_info* info, lab_stream s)
{
    LAB_ARG(A && b && x && c, "null argument");
    LAB_ARG(A->m == A->n, "CG needs a square matrix");
    LAB_ARG(c->max_iter >= 0, "negative max_iter");
    LAB_TRY(ensure_init());
    if(!M)
        return cg_plain(A, b, x, c, info, to_stream(s));
    if(M->kind == 0 && M->o.precision != LAB_PREC_FP64)
        return pcg_refine(A, M, b, x, c, info, to_stream(s));
    lab_status st = pcg_solve(A, M, b, x, c, info, to_stream(s));
    return M->kind >= 2 && st != LAB_BAD_ARG ? tri_status(M, st, to_stream(s)) : st;
}

LAB_API lab_status lab_pcg_solve_host(lab_csr A, lab_precond M, const double* bh, double* xh,
                                      const lab_iter_control* c, lab_solve_info* info, lab_stream ls)
{
    LAB_ARG(A && bh && xh && c, "null argument");
    LAB_TRY(ensure_init());
    cudaStream_t s = to_stream(ls);
    dbuf<double> b, x;
    LAB_TRY(b.alloc((size_t)A->m + 1, s));
    LAB_TRY(x.alloc((size_t)A->m + 1, s));
    LAB_CUDA(cudaMemcpyAsync(b.get(), bh, sizeof(double) * A->m, cudaMemcpyHostToDevice, s));
    LAB_CUDA(cudaMemcpyAsync(x.get(), xh, sizeof(double) * A->m, cudaMemcpyHostToDevice, s));
    lab_status st = !M ? cg_plain(A, b.get(), x.get(), c, info, s)
                       : (M->kind == 0 && M->o.precision != LAB_PREC_FP64)
                             ? pcg_refine(A, M, b.get(), x.get(), c, info, s)
                             : pcg_solve(A, M, b.get(), x.get(), c, info, s);
    if(M && M->kind >= 2 && st != LAB_BAD_ARG)
        st = tri_status(M, st, s);
    if(st != LAB_OK && st != LAB_NOT_CONVERGED && st != LAB_NAN)
        return st;
    LAB_CUDA(cudaMemcpyAsync(xh, x.get(), sizeof(double) * A->m, cudaMemcpyDeviceToHost, s));
    LAB_CUDA(cudaStreamSynchronize(s));
    return st;
}

LAB_API lab_status lab_gmres_solve(lab_csr A, lab_precond M, int restart, const double* b,
                                   double* x, const lab_iter_control* c, lab_solve_info* info,
                                   lab_stream s)
{
    LAB_ARG(A && b && x && c, "null argument");
    LAB_ARG(A->m == A->n, "GMRES needs a square matrix");
    LAB_ARG(restart >= 1, "restart must be >= 1");
    LAB_TRY(ensure_init());
    lab_status st = gmres_solve(A, M, restart, b, x, c, info, to_stream(s));
    return M && M->kind >= 2 && st != LAB_BAD_ARG ? tri_status(M, st, to_stream(s)) : st;
}

__global__ void k_block_copy(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                             const double* __restrict__ v, int64_t m, int64_t nnz, int32_t row_off,
                             int32_t col_off, int32_t nz_off, int32_t* orp, int32_t* oci,
                             double* ov)
{
    for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nnz + m;
        i += (int64_t)gridDim.x * blockDim.x)
    {
        if(i < nnz)
        {
            oci[nz_off + i] = ci[i] + col_off;
            ov[nz_off + i]  = v[i];
        }
        else
        {
            int64_t r        = i - nnz;
            orp[row_off + r] = rp[r] + nz_off;
        }
    }
}

LAB_API lab_status lab_csr_block_diag(const lab_csr* blocks, int nblocks, lab_csr* out,
                                      int64_t* offsets, lab_stream ls)
{
    LAB_ARG(blocks && out && offsets && nblocks > 0, "null argument");
    LAB_TRY(ensure_init());
    cudaStream_t s = to_stream(ls);
    int64_t      m = 0, n = 0, nnz = 0;
    for(int k = 0; k < nblocks; k++)
    {
        LAB_ARG(blocks[k], "null block");
        offsets[k] = m;
        m += blocks[k]->m;
        n += blocks[k]->n;
        nnz += blocks[k]->nnz;
    }
    offsets[nblocks] = m;
    LAB_ARG(m < INT32_MAX && nnz < INT32_MAX, "stacked matrix exceeds int32 indices");
    lab_csr_impl* C = nullptr;
    LAB_TRY(csr_alloc(&C, m, n, nnz, s));
    int64_t r0 = 0, c0 = 0, z0 = 0;
    for(int k = 0; k < nblocks; k++)
    {
        const lab_csr_impl* B = blocks[k];
        unsigned            g = grid_for(B->m + B->nnz);
        k_block_copy<<<g, 256, 0, s>>>(B->row_ptr, B->col_ind, B->val, B->m, B->nnz, (int32_t)r0,
                                       (int32_t)c0, (int32_t)z0, C->row_ptr, C->col_ind, C->val);
        g_launches.fetch_add(1);
        r0 += B->m;
        c0 += B->n;
        z0 += B->nnz;
    }
    int32_t last = (int32_t)nnz;
    cudaMemcpyAsync(C->row_ptr + m, &last, sizeof(int32_t), cudaMemcpyHostToDevice, s);
    cudaError_t e = cudaStreamSynchronize(s);
    if(e != cudaSuccess)
    {
        csr_release(C);
        return cuda_status(e, "lab_csr_block_diag", __FILE__, __LINE__);
    }
    *out = static_cast<lab_csr>(C);
    return LAB_OK;
}

LAB_API lab_status lab_batched_pcg_solve(lab_csr A, lab_precond M, int nsys,
                                         const int64_t* offsets, const double* b, double* x,
                                         const lab_iter_control* c, int* iterations,
                                         int* converged, lab_solve_info* info, lab_stream ls)
{
    LAB_ARG(A && M && offsets && b && x && c && nsys > 0, "null argument");
    LAB_ARG(offsets[0] == 0 && offsets[nsys] == A->m, "offsets must cover the rows of A");
    for(int k = 0; k < nsys; k++)
        LAB_ARG(offsets[k + 1] >= offsets[k], "offsets must be non-decreasing");
    LAB_TRY(ensure_init());
    cudaStream_t s = to_stream(ls);
    LAB_TRY(spmv_analyse(A, s));
    if(M->kind == 0)
        LAB_TRY(cycle_prepare(M->h, &M->o, s));
    seg_ops o;
    o.A = A;
    o.M = M;
    return seg_solve(o, nsys, offsets, b, x, c, iterations, converged, info, s);
}

LAB_API lab_status lab_multi_rhs_pcg_solve(lab_csr A, lab_precond M, int nrhs, const double* B,
                                           double* X, const lab_iter_control* c, int* iterations,
                                           int* converged, lab_solve_info* info, lab_stream ls)
{
    LAB_ARG(A && M && B && X && c && nrhs > 0, "null argument");
    LAB_ARG(A->m == A->n, "square matrix required");
    LAB_TRY(ensure_init());
    cudaStream_t s = to_stream(ls);
    LAB_TRY(spmv_analyse(A, s));
    if(M->kind == 0)
        LAB_TRY(cycle_prepare(M->h, &M->o, s));
    std::vector<int64_t> off((size_t)nrhs + 1);
    for(int k = 0; k <= nrhs; k++)
        off[k] = (int64_t)k * A->m;
    seg_ops o;
    o.A     = A;
    o.M     = M;
    o.multi = 1;
    o.n     = A->m;
    if(M->kind == 0 && cycle_block_supported(M->h, &M->o))
    {
        LAB_TRY(cycle_prepare_block(M->h, s));
        o.block = 1;
    }
    return seg_solve(o, nrhs, off.data(), B, X, c, iterations, converged, info, s);
}

LAB_API lab_status lab_adjoint_solve(lab_csr A, lab_precond M, int symmetric, const double* g,
                                     double* lambda, const lab_iter_control* c,
                                     lab_solve_info* info, lab_stream ls)
{
    LAB_ARG(A && g && lambda && c, "null argument");
    LAB_ARG(A->m == A->n, "adjoint needs a square matrix");
    LAB_TRY(ensure_init());
    cudaStream_t s = to_stream(ls);
    if(symmetric)
    {
        if(!M)
            return cg_plain(A, g, lambda, c, info, s);
        return pcg_solve(A, M, g, lambda, c, info, s);
    }
    lab_csr_impl* T = nullptr;
    LAB_TRY(transpose(A, &T, s));
    lab_status st = gmres_solve(T, M, 50, g, lambda, c, info, s);
    csr_release(T);
    return st;
}

LAB_API lab_status lab_adjoint_grad_A(lab_csr A, const double* lambda, const double* x,
                                      double* grad, lab_stream s)
{
    LAB_ARG(A && lambda && x && (grad || A->nnz == 0), "null argument");
    LAB_TRY(ensure_init());
    if(A->m == 0)
        return LAB_OK;
    LAB_LAUNCH(k_adjoint_grad, (unsigned)ceil_div<int64_t>(A->m, 256), 256, 0, to_stream(s),
               (const int32_t*)A->row_ptr, (const int32_t*)A->col_ind, A->m, lambda, x, grad);
    return LAB_OK;
}

} // extern "C"
