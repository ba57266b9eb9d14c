// Triangular path: sparse triangular solves, in-place ILU(0) and IC(0), behind
// the reference's csrtrsv / csrilu0 / csric0 and its ILU(0), IC(0), Gauss-Seidel
// and SOR preconditioners.
//
// Rows are grouped into dependency levels once per matrix pattern (on the host:
// a row's level is one more than the deepest row it reads).  A solve is one
// launch (after one that marks x pending): warps claim 32-row chunks in level
// order from an atomic counter, and each lane walks its row in the reference's
// order, reading a dependency once its value is no longer marked pending.  A
// chunk only waits on rows claimed before it, by warps that are running, so
// every wait ends; the waits are still bounded (an error flag is set and the
// kernel returns).  The factorizations run one launch per level.
// Every row is computed by one thread in exactly the reference's operation
// order (host_csrtrsv.cpp, host_csrilu0.cpp, host_csric0.cpp), so the results
// are bit-identical to the reference's sequential loops.
#include "internal.cuh"
#include "tri.cuh"
#include "amg.cuh"

#include <algorithm>
#include <climits>
#include <vector>

namespace lab
{
    struct tri_sched
    {
        std::vector<int> ptr;          // level k: rows[ptr[k] .. ptr[k+1])
        int32_t*         rows = nullptr; // device, rows ordered by level
    };

    struct tri_plan
    {
        tri_sched lower, upper;
        int32_t*  diag     = nullptr; // device: position of a_ii in row i, -1 if absent
        int32_t*  ctl      = nullptr; // device: claim counter, error flag of the solves
        double*   scratch  = nullptr; // device: copy of b for in-place solves
        bool      all_diag = true;
        // bounded wait: idle polling rounds before a warp gives up, and a row whose
        // value the solves never write (-1: none; set only to test that path)
        unsigned  idle_limit = 0;     // 0: kTriIdle
        int       held_row   = -1;
    };

    void tri_release(lab_csr_impl* A)
    {
        if(!A->tri)
            return;
        if(A->tri->lower.rows)
            cudaFree(A->tri->lower.rows);
        if(A->tri->upper.rows)
            cudaFree(A->tri->upper.rows);
        if(A->tri->diag)
            cudaFree(A->tri->diag);
        if(A->tri->ctl)
            cudaFree(A->tri->ctl);
        if(A->tri->scratch)
            cudaFree(A->tri->scratch);
        delete A->tri;
        A->tri = nullptr;
    }

    // ------------------------------------------------------------ level analysis
    // Dependency levels of the lower (row i reads columns < i) or upper (columns > i)
    // triangle, on the device, by Kahn's algorithm: the rows with no dependency are
    // level 0; processing level L decrements the pending-dependency count of every
    // row that reads one of its rows, and a row whose count reaches 0 joins level
    // L + 1.  One cooperative launch runs all levels, separated by a grid barrier;
    // order[] receives the rows level by level (any order within a level: a
    // level's rows are independent, so results do not depend on it).
    __global__ void k_iota(int32_t* __restrict__ p, int n)
    {
        const int i = blockIdx.x * blockDim.x + threadIdx.x;
        if(i < n)
            p[i] = i;
    }

    __global__ void k_dep_count(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                int m, int lower, int32_t* __restrict__ indeg,
                                int32_t* __restrict__ tcnt)
    {
        const int i = blockIdx.x * blockDim.x + threadIdx.x;
        if(i >= m)
            return;
        int d = 0;
        for(int j = rp[i]; j < rp[i + 1]; j++)
        {
            const int c = ci[j];
            if(lower ? c < i : c > i)
            {
                d++;
                atomicAdd(&tcnt[c], 1);
            }
        }
        indeg[i] = d;
    }

    __global__ void k_dep_fill(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                               int m, int lower, int32_t* __restrict__ tcur,
                               int32_t* __restrict__ tadj)
    {
        const int i = blockIdx.x * blockDim.x + threadIdx.x;
        if(i >= m)
            return;
        for(int j = rp[i]; j < rp[i + 1]; j++)
        {
            const int c = ci[j];
            if(lower ? c < i : c > i)
                tadj[atomicAdd(&tcur[c], 1)] = i;
        }
    }

    __global__ void k_diag_pos(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                               int m, int32_t* __restrict__ dpos, int* missing)
    {
        const int i = blockIdx.x * blockDim.x + threadIdx.x;
        if(i >= m)
            return;
        int d = -1;
        for(int j = rp[i]; j < rp[i + 1]; j++)
            if(ci[j] == i)
            {
                d = j;
                break;
            }
        dpos[i] = d;
        if(d < 0)
            atomicExch(missing, 1);
    }

    struct kahn_ctl
    {
        unsigned arrive, gen;
        int      tail, err, nlev;
    };

    __device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p)
    {
        unsigned v;
        asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
        return v;
    }
    __device__ __forceinline__ void st_release_u32(unsigned* p, unsigned v)
    {
        asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
    }

    constexpr unsigned kKahnSpin = 1u << 22; // bounded barrier wait (then the error flag)

    // Grid barrier (all blocks are co-resident: cooperative launch).  The last
    // block to arrive records the level boundary lptr[slot] = rows appended so far
    // and releases the others; a block that waits kKahnSpin rounds sets the error
    // flag.  Returns false on error.
    __device__ bool kahn_barrier(kahn_ctl* c, int slot, int32_t* lptr)
    {
        __shared__ int ok;
        __syncthreads();
        if(threadIdx.x == 0)
        {
            __threadfence();
            const unsigned g = ld_acquire_u32(&c->gen);
            ok               = 1;
            if(atomicAdd(&c->arrive, 1u) == gridDim.x - 1)
            {
                atomicExch(&c->arrive, 0u);
                lptr[slot] = atomicAdd(&c->tail, 0);
                __threadfence();
                st_release_u32(&c->gen, g + 1u);
            }
            else
            {
                unsigned it = 0;
                while(ld_acquire_u32(&c->gen) == g)
                {
                    if(++it > kKahnSpin)
                    {
                        atomicExch(&c->err, 1);
                        break;
                    }
                    __nanosleep(64);
                }
            }
            if(atomicAdd(&c->err, 0))
                ok = 0;
        }
        __syncthreads();
        return ok != 0;
    }

    __global__ void __launch_bounds__(512)
        k_kahn(const int32_t* __restrict__ tptr, const int32_t* __restrict__ tadj,
               int32_t* indeg, int m, int32_t* order, int32_t* lptr, kahn_ctl* c)
    {
        const int nt  = gridDim.x * blockDim.x;
        const int tid = blockIdx.x * blockDim.x + threadIdx.x;
        for(int i = tid; i < m; i += nt)
            if(indeg[i] == 0)
                order[atomicAdd(&c->tail, 1)] = i;
        int L = 0, lo = 0;
        if(!kahn_barrier(c, 1, lptr))
            return;
        for(;;)
        {
            const int hi = __ldcg(lptr + L + 1);
            if(hi == lo)
            {
                if(tid == 0)
                    c->nlev = L;
                return;
            }
            for(int t = lo + tid; t < hi; t += nt)
            {
                const int r = __ldcg(order + t);
                for(int q = tptr[r]; q < tptr[r + 1]; q++)
                {
                    const int j = tadj[q];
                    if(atomicSub(&indeg[j], 1) == 1)
                        order[atomicAdd(&c->tail, 1)] = j;
                }
            }
            lo = hi;
            L++;
            if(!kahn_barrier(c, L + 1, lptr))
                return;
        }
    }

    // Row -> level of the level order.
    __global__ void k_row_level(const int32_t* __restrict__ order, const int32_t* __restrict__ lptr,
                                int m, int nlev, int32_t* __restrict__ lev)
    {
        const int t = blockIdx.x * blockDim.x + threadIdx.x;
        if(t >= m)
            return;
        int lo = 0, hi = nlev - 1; // the level L with lptr[L] <= t < lptr[L + 1]
        while(lo < hi)
        {
            const int mid = (lo + hi + 1) >> 1;
            if(lptr[mid] <= t)
                lo = mid;
            else
                hi = mid - 1;
        }
        lev[order[t]] = lo;
    }

    // Rows of each level in ascending order (neighbouring rows of a level then load
    // neighbouring matrix rows): the level order is the transpose of the m x nlev
    // row -> level incidence, and the library's transpose keeps each output row in
    // source-row order.
    static lab_status order_levels(tri_sched& out, const int32_t* lptr, int m, int nlev,
                                   cudaStream_t s)
    {
        if(m == 0 || nlev <= 1)
            return LAB_OK;
        lab_csr_impl* T = nullptr;
        LAB_TRY(csr_alloc(&T, m, nlev, m, s));
        lab_status st = LAB_OK;
        k_iota<<<(unsigned)ceil_div(m + 1, 256), 256, 0, s>>>(T->row_ptr, m + 1);
        k_row_level<<<(unsigned)ceil_div(m, 256), 256, 0, s>>>(out.rows, lptr, m, nlev, T->col_ind);
        g_launches.fetch_add(2);
        if(cudaGetLastError() != cudaSuccess ||
           cudaMemsetAsync(T->val, 0, sizeof(double) * (size_t)m, s) != cudaSuccess)
            st = LAB_CUDA_ERROR;
        lab_csr_impl* Tt = nullptr;
        if(st == LAB_OK)
            st = transpose(T, &Tt, s);
        if(st == LAB_OK &&
           cudaMemcpyAsync(out.rows, Tt->col_ind, sizeof(int32_t) * (size_t)m,
                           cudaMemcpyDeviceToDevice, s) != cudaSuccess)
            st = LAB_CUDA_ERROR;
        if(Tt)
        {
            cudaStreamSynchronize(s);
            csr_release(Tt);
        }
        cudaStreamSynchronize(s);
        csr_release(T);
        return st;
    }

    static lab_status level_sched_dev(const lab_csr_impl* A, bool lower, tri_sched& out,
                                      cudaStream_t s)
    {
        const int      m = (int)A->m;
        dbuf<int32_t>  indeg, tptr, tcur, tadj, lptr;
        dbuf<kahn_ctl> ctl;
        int64_t        ndep = 0;
        LAB_TRY(indeg.alloc((size_t)m, s));
        LAB_TRY(tptr.alloc((size_t)m + 1, s));
        LAB_CUDA(cudaMemsetAsync(tptr.get(), 0, sizeof(int32_t) * ((size_t)m + 1), s));
        const unsigned g = (unsigned)ceil_div(m, 256);
        LAB_LAUNCH(k_dep_count, g, 256, 0, s, A->row_ptr, A->col_ind, m, (int)lower, indeg.get(),
                   tptr.get());
        LAB_TRY(counts_to_rowptr(tptr.get(), tptr.get(), m, &ndep, s));
        LAB_TRY(tcur.alloc((size_t)m + 1, s));
        LAB_TRY(tadj.alloc((size_t)std::max<int64_t>(ndep, 1), s));
        LAB_CUDA(cudaMemcpyAsync(tcur.get(), tptr.get(), sizeof(int32_t) * ((size_t)m + 1),
                                 cudaMemcpyDeviceToDevice, s));
        LAB_LAUNCH(k_dep_fill, g, 256, 0, s, A->row_ptr, A->col_ind, m, (int)lower, tcur.get(),
                   tadj.get());
        LAB_TRY(dalloc(&out.rows, (size_t)std::max(m, 1), s));
        LAB_TRY(lptr.alloc((size_t)m + 2, s));
        LAB_TRY(ctl.alloc(1, s));
        LAB_CUDA(cudaMemsetAsync(lptr.get(), 0, sizeof(int32_t) * ((size_t)m + 2), s));
        LAB_CUDA(cudaMemsetAsync(ctl.get(), 0, sizeof(kahn_ctl), s));
        static int occ = 0;
        if(!occ)
        {
            if(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_kahn, 512, 0) != cudaSuccess ||
               occ < 1)
            {
                cudaGetLastError();
                occ = 1;
            }
        }
        const int32_t* tp     = tptr.get();
        const int32_t* ta     = tadj.get();
        int32_t*       id     = indeg.get();
        int32_t*       od     = out.rows;
        int32_t*       lp     = lptr.get();
        kahn_ctl*      cp     = ctl.get();
        int            mm     = m;
        void*          args[] = {(void*)&tp, (void*)&ta, (void*)&id, (void*)&mm,
                                 (void*)&od, (void*)&lp, (void*)&cp};
        unsigned grid = (unsigned)std::max(1, std::min(num_sms() * occ, (int)ceil_div(m, 512)));
        // every block must be resident at once: a device shared with other work may
        // not fit the occupancy-derived grid, so halve it until the launch is accepted
        cudaError_t le = cudaErrorCooperativeLaunchTooLarge;
        while(true)
        {
            le = cudaLaunchCooperativeKernel((const void*)k_kahn, dim3(grid), dim3(512), args, 0, s);
            if(le != cudaErrorCooperativeLaunchTooLarge || grid == 1)
                break;
            cudaGetLastError();
            grid = std::max(1u, grid / 2);
        }
        LAB_CUDA(le);
        g_launches.fetch_add(1);
        kahn_ctl hc{};
        LAB_TRY(copy_d2h_sync(&hc, ctl.get(), sizeof(hc), s));
        if(hc.err || hc.tail != m)
        {
            set_error("triangular analysis: level computation failed (%s)",
                      hc.err ? "barrier wait" : "a row never became ready");
            return LAB_CUDA_ERROR;
        }
        out.ptr.assign((size_t)hc.nlev + 1, 0);
        LAB_TRY(copy_d2h_sync(out.ptr.data(), lptr.get(), sizeof(int32_t) * out.ptr.size(), s));
        return order_levels(out, lptr.get(), m, hc.nlev, s);
    }

    lab_status tri_analyse(lab_csr_impl* A, cudaStream_t s)
    {
        if(A->tri)
            return LAB_OK;
        const int m = (int)A->m;
        tri_plan* p = new(std::nothrow) tri_plan();
        if(!p)
            return LAB_OOM;
        A->tri        = p;
        lab_status st = dalloc(&p->diag, (size_t)std::max(m, 1), s);
        dbuf<int>  missing;
        if(st == LAB_OK)
            st = missing.alloc(1, s);
        if(st == LAB_OK && cudaMemsetAsync(missing.get(), 0, sizeof(int), s) != cudaSuccess)
            st = LAB_CUDA_ERROR;
        if(st == LAB_OK && m > 0)
        {
            k_diag_pos<<<(unsigned)ceil_div(m, 256), 256, 0, s>>>(A->row_ptr, A->col_ind, m,
                                                                 p->diag, missing.get());
            g_launches.fetch_add(1);
            if(cudaGetLastError() != cudaSuccess)
                st = LAB_CUDA_ERROR;
        }
        if(st == LAB_OK && m > 0)
            st = level_sched_dev(A, true, p->lower, s);
        if(st == LAB_OK && m > 0)
            st = level_sched_dev(A, false, p->upper, s);
        if(st == LAB_OK)
            st = dalloc(&p->ctl, 2, s);
        if(st == LAB_OK && cudaMemsetAsync(p->ctl, 0, sizeof(int32_t) * 2, s) != cudaSuccess)
            st = LAB_CUDA_ERROR;
        int miss = 0;
        if(st == LAB_OK)
            st = copy_d2h_sync(&miss, missing.get(), sizeof(int), s);
        p->all_diag = miss == 0;
        if(st != LAB_OK)
            tri_release(A);
        return st;
    }

    // ------------------------------------------------------------ solves
    // x is filled with kTriPending before a solve and every x_i is written once,
    // by the row's lane, as the result of a double operation.  Such a result is
    // never a signalling NaN (arithmetic returns a quiet NaN), so a value other
    // than kTriPending is the solved x_i: the value is its own "solved" flag and
    // a dependency costs one L2 round trip (relaxed 64-bit loads and stores at
    // GPU scope, single-copy atomic).
    constexpr uint64_t kTriPending = 0x7ff4d1b0c0de0001ull; // signalling NaN
    constexpr int      kTriBlock   = 256;
    constexpr int      kTriPf      = 8;        // entries of a row held in registers
    constexpr unsigned kTriIdle    = 1u << 26; // default idle rounds before a warp gives up

    __device__ __forceinline__ uint64_t ld_relaxed(const double* p)
    {
        uint64_t v;
        asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
        return v;
    }
    __device__ __forceinline__ void st_relaxed(double* p, double v)
    {
        asm volatile("st.relaxed.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(__double_as_longlong(v))
                     : "memory");
    }
    __device__ __forceinline__ int ld_acquire(const int32_t* p)
    {
        int v;
        asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
        return v;
    }

    __global__ void k_trsv_prep(double* x, int m, int32_t* counter, const int* skip)
    {
        if(skip && *skip)
            return;
        uint64_t* u = reinterpret_cast<uint64_t*>(x);
        for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
            u[i] = kTriPending;
        if(blockIdx.x == 0 && threadIdx.x == 0)
            *counter = 0;
    }

    // One entry of a lane's row, in the reference's order, given the entry's
    // dependency value xv (kTriPending: not solved yet -> false).  LOWER,
    // host_forward_solve_impl (host_csrtrsv.cpp:36-64): fma over the entries left
    // of the diagonal in CSR order, stop at the first entry right of it (or at the
    // diagonal when unit); dscale != 0 scales the diagonal (SOR_precond's M,
    // preconditioner.cpp:137-147).  Upper, host_backward_solve_impl (66-90): walk
    // the row right to left subtracting a_ij x_j (multiply, then subtract), keep
    // the diagonal.
    template <bool LOWER>
    __device__ __forceinline__ bool tri_entry(int c, double a, uint64_t xv, int i, int unit,
                                              double dscale, int len, int& k, double& acc,
                                              double& d)
    {
        if(LOWER ? c < i : c > i)
        {
            if(xv == kTriPending)
                return false;
            const double xc = __longlong_as_double((long long)xv);
            acc             = LOWER ? fma(a, xc, acc) : __dsub_rn(acc, __dmul_rn(a, xc));
            k++;
        }
        else if(c == i && !unit)
        {
            d = (LOWER && dscale != 0.0) ? __dmul_rn(a, dscale) : a;
            k++;
        }
        else
            k = LOWER ? len : k + 1; // the forward loop breaks here
        return true;
    }

    // Warps claim 32-row chunks of `order` (rows by level) from ctl[0]; each lane
    // polls the dependencies of its row's next entries at once, consumes the solved
    // prefix in order, and writes x_i when the row is done.  ctl[1] is the error
    // flag, set when a warp waited idle_limit rounds without progress; the other
    // warps see it when they claim their next chunk or every 1024 idle rounds and
    // return.  held (>= 0) is a row whose value is never written: the rows that
    // depend on it can only run out of their wait (the test of this path).
    template <bool LOWER>
    __global__ void __launch_bounds__(kTriBlock)
        k_trsv(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
               const double* __restrict__ v, const int32_t* __restrict__ order, int m, int unit,
               double dscale, const double* __restrict__ b, double* x, int32_t* ctl,
               const int* skip, unsigned idle_limit, int held)
    {
        if(skip && *skip)
            return;
        const int lane = threadIdx.x & 31;
        for(;;)
        {
            int base = 0;
            if(lane == 0)
                base = ld_acquire(ctl + 1) ? m : atomicAdd(ctl, 32);
            base = __shfl_sync(0xffffffffu, base, 0);
            if(base >= m)
                return;
            const int t    = base + lane;
            bool      done = t >= m;
            int       i = 0, a = 0, e = 0, len = 0, k = 0;
            double    acc = 0.0, d = 1.0, bi = 0.0;
            int       pc[kTriPf];
            double    pv[kTriPf];
            if(!done)
            {
                i   = order[t];
                a   = rp[i];
                e   = rp[i + 1];
                len = e - a;
#pragma unroll
                for(int q = 0; q < kTriPf; q++)
                {
                    const int j = LOWER ? a + q : e - 1 - q;
                    pc[q]       = q < len ? ci[j] : i;
                    pv[q]       = q < len ? v[j] : 0.0;
                }
                if(LOWER)
                    bi = b[i];
                else
                    acc = b[i];
            }
            unsigned idle = 0;
            for(;;)
            {
                bool progress = false;
                if(!done)
                {
                    const int k0 = k;
                    // all outstanding dependencies of the held entries in flight at once
                    uint64_t xv[kTriPf];
#pragma unroll
                    for(int q = 0; q < kTriPf; q++)
                        xv[q] = (q >= k && q < len && (LOWER ? pc[q] < i : pc[q] > i))
                                    ? ld_relaxed(x + pc[q])
                                    : 0;
                    bool blocked = false;
#pragma unroll
                    for(int q = 0; q < kTriPf; q++)
                        if(!blocked && q == k && k < len)
                            blocked = !tri_entry<LOWER>(pc[q], pv[q], xv[q], i, unit, dscale, len,
                                                        k, acc, d);
                    while(!blocked && k < len) // entries beyond the held ones
                    {
                        const int j  = LOWER ? a + k : e - 1 - k;
                        const int c  = ci[j];
                        uint64_t  xc = (LOWER ? c < i : c > i) ? ld_relaxed(x + c) : 0;
                        blocked = !tri_entry<LOWER>(c, v[j], xc, i, unit, dscale, len, k, acc, d);
                    }
                    progress = k != k0;
                    if(!blocked && i == held)
                    {
                        done     = true; // x_i stays pending
                        progress = true;
                    }
                    else if(!blocked)
                    {
                        st_relaxed(x + i,
                                   LOWER ? __ddiv_rn(__dsub_rn(bi, acc), d) : __ddiv_rn(acc, d));
                        done     = true;
                        progress = true;
                    }
                }
                if(__all_sync(0xffffffffu, done))
                    break;
                if(__any_sync(0xffffffffu, progress))
                    idle = 0;
                else
                {
                    if(++idle >= idle_limit)
                    {
                        if(lane == 0)
                            atomicExch(ctl + 1, 1);
                        return;
                    }
                    if((idle & 1023u) == 0 && __any_sync(0xffffffffu, ld_acquire(ctl + 1) != 0))
                        return;
                    __nanosleep(idle < 8 ? 0 : 64);
                }
            }
        }
    }

    // One CTA (8 warps) per SM: 37,888 rows in flight on 148 SMs, more than the
    // widest level of the 128^3 7-point solve; more warps only add polling traffic
    // (measured: 740 us per 128^3 solve at 1 CTA per SM, 860 us at 3).
    static int trsv_grid(int m)
    {
        return (int)std::max<int64_t>(1, std::min<int64_t>(num_sms(), ceil_div(m, kTriBlock)));
    }

    lab_status tri_solve(lab_csr_impl* A, bool lower, bool unit, double dscale, const double* b,
                         double* x, cudaStream_t s, const int* skip)
    {
        if(A->m == 0)
            return LAB_OK;
        LAB_TRY(tri_analyse(A, s));
        tri_plan& p = *A->tri;
        const int m = (int)A->m;
        if(b < x + m && x < b + m) // in place: x is overwritten by the pending marks first
        {
            if(!p.scratch)
                LAB_TRY(dalloc(&p.scratch, (size_t)m, s));
            LAB_CUDA(cudaMemcpyAsync(p.scratch, b, sizeof(double) * m, cudaMemcpyDeviceToDevice, s));
            b = p.scratch;
        }
        LAB_LAUNCH(k_trsv_prep, (unsigned)std::min<int64_t>(ceil_div(m, 256), 4 * num_sms()), 256,
                   0, s, x, m, p.ctl, skip);
        const unsigned idle = p.idle_limit ? p.idle_limit : kTriIdle;
        if(lower)
            LAB_LAUNCH(k_trsv<true>, trsv_grid(m), kTriBlock, 0, s, A->row_ptr, A->col_ind,
                       (const double*)A->val, (const int32_t*)p.lower.rows, m, (int)unit, dscale,
                       b, x, p.ctl, skip, idle, p.held_row);
        else
            LAB_LAUNCH(k_trsv<false>, trsv_grid(m), kTriBlock, 0, s, A->row_ptr,
                       A->col_ind, (const double*)A->val, (const int32_t*)p.upper.rows, m,
                       (int)unit, 0.0, b, x, p.ctl, skip, idle, p.held_row);
        return LAB_OK;
    }

    lab_status tri_check(lab_csr_impl* A, cudaStream_t s)
    {
        if(!A->tri || A->m == 0)
            return LAB_OK;
        int32_t e = 0;
        LAB_TRY(copy_d2h_sync(&e, A->tri->ctl + 1, sizeof(e), s));
        if(e)
        {
            LAB_CUDA(cudaMemsetAsync(A->tri->ctl + 1, 0, sizeof(int32_t), s));
            set_error("triangular solve: a row waited longer than the wait limit for its "
                      "dependencies");
            return LAB_TIMEOUT;
        }
        return LAB_OK;
    }

    // ------------------------------------------------------------ factorizations
    // get_diagonal_value_local (host_csrilu0.cpp:35-54): the pivot of column col,
    // 1.0 (recorded) when it is missing or zero.
    __device__ __forceinline__ double tri_pivot(int col, int di, const double* v, int* sz, int* nz)
    {
        if(di == -1)
        {
            atomicMin(sz, col);
            return 1.0;
        }
        const double d = v[di];
        if(d == 0.0)
        {
            atomicMin(nz, col);
            return 1.0;
        }
        return d;
    }

    // One row of host_csrilu0_impl (host_csrilu0.cpp:66-100).  The reference looks
    // entries of the row up through a column->position map; both rows are sorted
    // by column, so a forward walk finds the same positions.  A missing pivot
    // (di = -1) keeps the reference's k loop from position 0 of the whole array and
    // searches the row for each column.
    __device__ void ilu0_row(int row, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                             double* v, const int32_t* __restrict__ diag, int* sz, int* nz)
    {
        const int a = rp[row], b = rp[row + 1];
        for(int j = a; j < b; j++)
        {
            const int cj = ci[j];
            if(cj > row)
                break;
            if(cj == row)
                break;
            const int    di  = diag[cj];
            const double piv = tri_pivot(cj, di, v, sz, nz);
            const int    end = rp[cj + 1];
            v[j]             = __ddiv_rn(v[j], piv);
            int          p   = a;
            for(int k = di + 1; k < end; k++)
            {
                const int ck = ci[k];
                int       t  = -1;
                if(di >= 0)
                {
                    while(p < b && ci[p] < ck)
                        p++;
                    if(p < b && ci[p] == ck)
                        t = p;
                }
                else
                {
                    for(int q = b - 1; q >= a; q--) // the map keeps the last position
                        if(ci[q] == ck)
                        {
                            t = q;
                            break;
                        }
                }
                // v[j] is re-read: with a missing pivot t can be j itself
                if(t != -1)
                    v[t] = __dsub_rn(v[t], __dmul_rn(v[j], v[k]));
            }
        }
    }

    // One row of host_csric0_impl (host_csric0.cpp:68-106).
    __device__ void ic0_row(int row, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                            double* v, const int32_t* __restrict__ diag, int* sz, int* nz)
    {
        const int a = rp[row], b = rp[row + 1];
        double    sum = 0.0;
        for(int j = a; j < b; j++)
        {
            const int cj = ci[j];
            if(cj < row)
            {
                const int di = diag[cj];
                double    s  = 0.0;
                int       p  = a;
                for(int k = rp[cj]; k < di; k++)
                {
                    const int ck = ci[k];
                    while(p < b && ci[p] < ck)
                        p++;
                    if(p < b && ci[p] == ck)
                        s = fma(v[p], v[k], s);
                }
                const double piv = tri_pivot(cj, di, v, sz, nz);
                const double val = __ddiv_rn(__dsub_rn(v[j], s), piv);
                sum              = fma(val, val, sum);
                v[j]             = val;
            }
            else if(cj == row)
            {
                v[j] = __dsqrt_rn(fabs(__dsub_rn(v[j], sum)));
                break;
            }
            else
                break;
        }
    }

    template <int IC>
    __global__ void k_factor_level(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                   double* v, const int32_t* __restrict__ diag,
                                   const int32_t* __restrict__ rows, int n, int* flags)
    {
        const int t = blockIdx.x * blockDim.x + threadIdx.x;
        if(t >= n)
            return;
        if(IC)
            ic0_row(rows[t], rp, ci, v, diag, flags, flags + 1);
        else
            ilu0_row(rows[t], rp, ci, v, diag, flags, flags + 1);
    }

    // Rows in order on one thread: ILU(0) with a missing pivot reads rows of any
    // level (the reference's k loop from position 0).
    __global__ void k_ilu0_sequential(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                      double* v, const int32_t* __restrict__ diag, int m, int* flags)
    {
        for(int row = 0; row < m; row++)
            ilu0_row(row, rp, ci, v, diag, flags, flags + 1);
    }

    lab_status tri_factor(lab_csr_impl* A, bool ic, int* structural_zero, int* numeric_zero,
                          cudaStream_t s)
    {
        LAB_TRY(tri_analyse(A, s));
        dbuf<int> flags;
        LAB_TRY(flags.alloc(2, s));
        const int init[2] = {INT_MAX, INT_MAX};
        LAB_CUDA(cudaMemcpyAsync(flags.get(), init, sizeof(init), cudaMemcpyHostToDevice, s));
        const tri_plan& p = *A->tri;
        if(A->m > 0)
        {
            if(!ic && !p.all_diag)
                LAB_LAUNCH(k_ilu0_sequential, 1, 1, 0, s, A->row_ptr, A->col_ind, A->val,
                           (const int32_t*)p.diag, (int)A->m, flags.get());
            else
                for(size_t k = 0; k + 1 < p.lower.ptr.size(); k++)
                {
                    const int      r0 = p.lower.ptr[k], n = p.lower.ptr[k + 1] - r0;
                    const unsigned g  = (unsigned)ceil_div(n, 128);
                    if(ic)
                        LAB_LAUNCH(k_factor_level<1>, g, 128, 0, s, A->row_ptr, A->col_ind, A->val,
                                   (const int32_t*)p.diag, (const int32_t*)(p.lower.rows + r0), n,
                                   flags.get());
                    else
                        LAB_LAUNCH(k_factor_level<0>, g, 128, 0, s, A->row_ptr, A->col_ind, A->val,
                                   (const int32_t*)p.diag, (const int32_t*)(p.lower.rows + r0), n,
                                   flags.get());
                }
        }
        int h[2];
        LAB_TRY(copy_d2h_sync(h, flags.get(), sizeof(h), s));
        if(structural_zero)
            *structural_zero = h[0] == INT_MAX ? -1 : h[0];
        if(numeric_zero)
            *numeric_zero = h[1] == INT_MAX ? -1 : h[1];
        return LAB_OK;
    }
}

namespace lab
{
    // ------------------------------------------------------------ SSOR split
    // SSOR_precond::build (preconditioner.cpp:283-353): L = (beta D - E) D^-1 holds
    // a_ij / d_j left of the diagonal and beta on it; U = beta D - F holds a_ij
    // right of it and beta * a_ii on it (host_ssor.cpp:52-142; d = the row's first
    // diagonal entry, 0 if none).  Entries keep A's order within each row.
    __global__ void k_ssor_count(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                 const double* __restrict__ v, int m, int32_t* cl, int32_t* cu,
                                 double* d)
    {
        const int i = blockIdx.x * blockDim.x + threadIdx.x;
        if(i >= m)
            return;
        int    nl = 0, nu = 0;
        double di = 0.0;
        bool   found = false;
        for(int j = rp[i]; j < rp[i + 1]; j++)
        {
            const int c = ci[j];
            nl += c <= i;
            nu += c >= i;
            if(c == i && !found)
            {
                di    = v[j];
                found = true;
            }
        }
        cl[i] = nl;
        cu[i] = nu;
        d[i]  = di;
    }

    __global__ void k_ssor_fill(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                const double* __restrict__ v, int m, const double* __restrict__ d,
                                double beta, const int32_t* __restrict__ lrp, int32_t* lci,
                                double* lv, const int32_t* __restrict__ urp, int32_t* uci,
                                double* uv)
    {
        const int i = blockIdx.x * blockDim.x + threadIdx.x;
        if(i >= m)
            return;
        int kl = lrp[i], ku = urp[i];
        for(int j = rp[i]; j < rp[i + 1]; j++)
        {
            const int    c = ci[j];
            const double a = v[j];
            if(c < i)
            {
                lci[kl]  = c;
                lv[kl++] = __ddiv_rn(a, d[c]);
            }
            else if(c > i)
            {
                uci[ku]  = c;
                uv[ku++] = a;
            }
            else
            {
                lci[kl]  = c;
                lv[kl++] = beta;
                uci[ku]  = c;
                uv[ku++] = __dmul_rn(beta, a);
            }
        }
    }

    // ------------------------------------------------------------ csr_matrix members
    // The triangle of A with columns <= i (lower) or >= i (upper), diagonal
    // included, rows kept in CSR order (host_extract.cpp:54-181; the reference
    // passes its unit_diag flag nowhere, so neither does this).
    __global__ void k_tri_count(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                int m, int upper, int32_t* __restrict__ cnt)
    {
        const int i = blockIdx.x * blockDim.x + threadIdx.x;
        if(i >= m)
            return;
        int c = 0;
        for(int j = rp[i]; j < rp[i + 1]; j++)
            c += upper ? ci[j] >= i : ci[j] <= i;
        cnt[i] = c;
    }

    __global__ void k_tri_fill(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                               const double* __restrict__ v, int m, int upper,
                               const int32_t* __restrict__ trp, int32_t* __restrict__ tci,
                               double* __restrict__ tv)
    {
        const int i = blockIdx.x * blockDim.x + threadIdx.x;
        if(i >= m)
            return;
        int o = trp[i];
        for(int j = rp[i]; j < rp[i + 1]; j++)
            if(upper ? ci[j] >= i : ci[j] <= i)
            {
                tci[o] = ci[j];
                tv[o]  = v[j];
                o++;
            }
    }

    // host_scale.cpp:34-52: the first stored a_ii of each row times the scalar
    __global__ void k_scale_diag(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                 double* __restrict__ v, int m, double scalar)
    {
        const int i = blockIdx.x * blockDim.x + threadIdx.x;
        if(i >= m)
            return;
        for(int j = rp[i]; j < rp[i + 1]; j++)
            if(ci[j] == i)
            {
                v[j] = __dmul_rn(v[j], scalar);
                break;
            }
    }

    // host_scale.cpp:54-69: every entry a_ij times (1 / d_j), d the diagonal of
    // extract_diagonal (first stored a_jj, 0 if none: the factor is then inf)
    __global__ void k_scale_inv_diag(const int32_t* __restrict__ ci, double* __restrict__ v,
                                     int64_t nnz, const double* __restrict__ d)
    {
        for(int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < nnz;
            j += (int64_t)gridDim.x * blockDim.x)
            v[j] = __dmul_rn(v[j], __ddiv_rn(1.0, d[ci[j]]));
    }

    static lab_status triangle(lab_csr_impl* A, bool upper, lab_csr_impl** T, cudaStream_t s)
    {
        const int     m = (int)A->m;
        dbuf<int32_t> cnt;
        LAB_TRY(cnt.alloc((size_t)m + 1, s));
        if(m > 0)
            LAB_LAUNCH(k_tri_count, (unsigned)ceil_div(m, 256), 256, 0, s, A->row_ptr, A->col_ind,
                       m, (int)upper, cnt.get());
        int64_t nt = 0;
        LAB_TRY(counts_to_rowptr(cnt.get(), cnt.get(), m, &nt, s));
        lab_csr_impl* t = nullptr;
        LAB_TRY(csr_alloc(&t, A->m, A->n, nt, s));
        lab_status st = LAB_OK;
        if(cudaMemcpyAsync(t->row_ptr, cnt.get(), sizeof(int32_t) * ((size_t)m + 1),
                           cudaMemcpyDeviceToDevice, s) != cudaSuccess)
            st = LAB_CUDA_ERROR;
        if(st == LAB_OK && m > 0)
        {
            k_tri_fill<<<(unsigned)ceil_div(m, 256), 256, 0, s>>>(
                A->row_ptr, A->col_ind, (const double*)A->val, m, (int)upper, t->row_ptr,
                t->col_ind, (double*)t->val);
            g_launches.fetch_add(1);
            if(cudaGetLastError() != cudaSuccess)
                st = LAB_CUDA_ERROR;
        }
        if(st != LAB_OK)
        {
            set_error("triangle extraction failed");
            csr_release(t);
            return st;
        }
        *T = t;
        return LAB_OK;
    }

    lab_status ssor_split(lab_csr_impl* A, double omega, lab_csr_impl** L, lab_csr_impl** U,
                          cudaStream_t s)
    {
        const int m = (int)A->m;
        // build() hands 1 / omega to the fill routines, which take its inverse again
        const double beta_in = 1.0 / omega;
        const double beta    = 1.0 / beta_in;
        dbuf<int32_t> cl, cu;
        dbuf<double>  d;
        LAB_TRY(cl.alloc((size_t)m + 1, s));
        LAB_TRY(cu.alloc((size_t)m + 1, s));
        LAB_TRY(d.alloc((size_t)m, s));
        LAB_CUDA(cudaMemsetAsync(cl.get() + m, 0, sizeof(int32_t), s));
        LAB_CUDA(cudaMemsetAsync(cu.get() + m, 0, sizeof(int32_t), s));
        if(m > 0)
            LAB_LAUNCH(k_ssor_count, (unsigned)ceil_div(m, 256), 256, 0, s, A->row_ptr, A->col_ind,
                       (const double*)A->val, m, cl.get(), cu.get(), d.get());
        LAB_TRY(scan_i32(cl.get(), (int64_t)m + 1, s));
        LAB_TRY(scan_i32(cu.get(), (int64_t)m + 1, s));
        int32_t nl = 0, nu = 0;
        LAB_TRY(copy_d2h_sync(&nl, cl.get() + m, sizeof(nl), s));
        LAB_TRY(copy_d2h_sync(&nu, cu.get() + m, sizeof(nu), s));
        lab_csr_impl *l = nullptr, *u = nullptr;
        LAB_TRY(csr_alloc(&l, A->m, A->n, nl, s));
        lab_status st = csr_alloc(&u, A->m, A->n, nu, s);
        if(st == LAB_OK &&
           (cudaMemcpyAsync(l->row_ptr, cl.get(), sizeof(int32_t) * ((size_t)m + 1),
                            cudaMemcpyDeviceToDevice, s) != cudaSuccess ||
            cudaMemcpyAsync(u->row_ptr, cu.get(), sizeof(int32_t) * ((size_t)m + 1),
                            cudaMemcpyDeviceToDevice, s) != cudaSuccess))
            st = LAB_CUDA_ERROR;
        if(st == LAB_OK && m > 0)
        {
            k_ssor_fill<<<(unsigned)ceil_div(m, 256), 256, 0, s>>>(
                A->row_ptr, A->col_ind, (const double*)A->val, m, d.get(), beta, l->row_ptr,
                l->col_ind, (double*)l->val, u->row_ptr, u->col_ind, (double*)u->val);
            g_launches.fetch_add(1);
            if(cudaGetLastError() != cudaSuccess)
                st = LAB_CUDA_ERROR;
        }
        if(st != LAB_OK)
        {
            csr_release(l);
            if(u)
                csr_release(u);
            return st;
        }
        *L = l;
        *U = u;
        return LAB_OK;
    }
}

using namespace lab;

extern "C" {

LAB_API lab_status lab_csrtrsv(lab_csr A, int lower, int unit_diag, const double* b, double* x,
                               lab_stream s)
{
    LAB_ARG(A && (A->m == 0 || (b && x)), "null argument");
    LAB_ARG(A->m == A->n, "triangular solve needs a square matrix");
    LAB_TRY(ensure_init());
    LAB_TRY(tri_solve(A, lower != 0, unit_diag != 0, 0.0, b, x, to_stream(s), nullptr));
    return tri_check(A, to_stream(s));
}

LAB_API lab_status lab_csrtrsv_wait_control(lab_csr A, int64_t idle_rounds, int64_t held_row,
                                            lab_stream s)
{
    LAB_ARG(A, "null matrix");
    LAB_ARG(idle_rounds >= 0 && idle_rounds <= 0xffffffffll, "idle_rounds out of range");
    LAB_ARG(held_row >= -1 && held_row < A->m, "held_row out of range");
    LAB_TRY(ensure_init());
    if(A->m == 0)
        return LAB_OK;
    LAB_TRY(tri_analyse(A, to_stream(s)));
    A->tri->idle_limit = (unsigned)idle_rounds;
    A->tri->held_row   = (int)held_row;
    return LAB_OK;
}

LAB_API lab_status lab_csr_triangle(lab_csr A, int upper, lab_csr* T, lab_stream s)
{
    LAB_ARG(A && T, "null argument");
    LAB_TRY(ensure_init());
    lab_csr_impl* t = nullptr;
    LAB_TRY(triangle(A, upper != 0, &t, to_stream(s)));
    *T = static_cast<lab_csr_s*>(t);
    return LAB_OK;
}

LAB_API lab_status lab_csrtrsv_analysis(lab_csr A, lab_stream s)
{
    LAB_ARG(A, "null matrix");
    LAB_ARG(A->m == A->n, "triangular analysis needs a square matrix");
    LAB_TRY(ensure_init());
    return A->m == 0 ? LAB_OK : tri_analyse(A, to_stream(s));
}

LAB_API lab_status lab_csr_scale_diagonal(lab_csr A, double scalar, lab_stream s)
{
    LAB_ARG(A, "null matrix");
    LAB_TRY(ensure_init());
    if(A->m > 0)
        LAB_LAUNCH(k_scale_diag, (unsigned)ceil_div<int64_t>(A->m, 256), 256, 0, to_stream(s),
                   A->row_ptr, A->col_ind, A->val, (int)A->m, scalar);
    return lab_csr_values_changed(A, s);
}

LAB_API lab_status lab_csr_scale_by_inverse_diagonal(lab_csr A, lab_stream ls)
{
    LAB_ARG(A, "null matrix");
    LAB_ARG(A->m == A->n, "square matrix required (columns index the diagonal)");
    LAB_TRY(ensure_init());
    cudaStream_t s = to_stream(ls);
    if(A->nnz > 0)
    {
        dbuf<double> d;
        LAB_TRY(d.alloc((size_t)A->m, s));
        LAB_TRY(diag_into(A, d.get(), nullptr, s));
        LAB_LAUNCH(k_scale_inv_diag,
                   (unsigned)std::min<int64_t>(ceil_div<int64_t>(A->nnz, 256), 8 * num_sms()), 256,
                   0, s, A->col_ind, A->val, A->nnz, (const double*)d.get());
    }
    return lab_csr_values_changed(A, ls);
}

LAB_API lab_status lab_csrilu0(lab_csr A, int* structural_zero, int* numeric_zero, lab_stream s)
{
    LAB_ARG(A, "null matrix");
    LAB_ARG(A->m == A->n, "ILU(0) needs a square matrix");
    LAB_TRY(ensure_init());
    LAB_TRY(tri_factor(A, false, structural_zero, numeric_zero, to_stream(s)));
    return lab_csr_values_changed(A, s);
}

LAB_API lab_status lab_csric0(lab_csr A, int* structural_zero, int* numeric_zero, lab_stream s)
{
    LAB_ARG(A, "null matrix");
    LAB_ARG(A->m == A->n, "IC(0) needs a square matrix");
    LAB_TRY(ensure_init());
    LAB_TRY(tri_factor(A, true, structural_zero, numeric_zero, to_stream(s)));
    return lab_csr_values_changed(A, s);
}

} // extern "C"
