// SpMV front end: analysis (row statistics -> schedule), y = alpha*A*x + beta*y,
// residual, multi-vector SpMM.
#include "spmv_engine.cuh"

#include <climits>
#include <vector>

namespace lab
{
    __global__ void k_row_stats(const int32_t* __restrict__ rp, int64_t m, int* maxlen)
    {
        int local = 0;
        for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m;
            i += (int64_t)gridDim.x * blockDim.x)
            local = max(local, rp[i + 1] - rp[i]);
#pragma unroll
        for(int o = 16; o > 0; o >>= 1)
            local = max(local, __shfl_xor_sync(0xffffffffu, local, o));
        if((threadIdx.x & 31) == 0)
            atomicMax(maxlen, local);
    }

    // Largest number of entries in a tile of `rows` consecutive rows.
    __global__ void k_tile_max(const int32_t* __restrict__ rp, int64_t m, int rows, int* out)
    {
        int           local  = 0;
        const int64_t ntiles = (m + rows - 1) / rows;
        for(int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < ntiles;
            t += (int64_t)gridDim.x * blockDim.x)
        {
            const int64_t r0 = t * rows;
            const int64_t r1 = r0 + rows < m ? r0 + rows : m;
            local            = max(local, rp[r1] - rp[r0]);
        }
#pragma unroll
        for(int o = 16; o > 0; o >>= 1)
            local = max(local, __shfl_xor_sync(0xffffffffu, local, o));
        if((threadIdx.x & 31) == 0)
            atomicMax(out, local);
    }

    // 16-bit column offsets col - row, W lanes per row (coalesced over the row's
    // entries); *wide = 1 when some offset leaves the int16 range (the copy is
    // then discarded).
    template <int W>
    __global__ void k_dcol_build(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                 int64_t m, int16_t* __restrict__ dcol, int* wide)
    {
        const int lane = threadIdx.x & (W - 1);
        int       bad  = 0;
        for(int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / W; i < m;
            i += (int64_t)gridDim.x * blockDim.x / W)
            for(int j = rp[i] + lane; j < rp[i + 1]; j += W)
            {
                const int64_t d = (int64_t)ci[j] - i;
                bad |= d < INT16_MIN || d > INT16_MAX;
                dcol[j] = (int16_t)d;
            }
        if(__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0)
            atomicOr(wide, 1);
    }

    // ------------------------------------------------------------ halo plan
    // Reductions over one CTA (every thread gets the result).
    template <int NT, class F>
    __device__ __forceinline__ int block_reduce(int v, int* red, F f)
    {
#pragma unroll
        for(int o = 16; o > 0; o >>= 1)
            v = f(v, __shfl_xor_sync(0xffffffffu, v, o));
        if((threadIdx.x & 31) == 0)
            red[threadIdx.x >> 5] = v;
        __syncthreads();
        int r = red[0];
#pragma unroll
        for(int k = 1; k < NT / 32; k++)
            r = f(r, red[k]);
        __syncthreads();
        return r;
    }

    // Marks chunk c's columns (rows [c*rows, c*rows + rows)) in a bitmap over
    // [lo, lo + 32*words); returns false (uniformly) when the chunk has no entries
    // or its span exceeds kHaloBits.
    template <int NT>
    __device__ bool halo_mark(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                              int64_t m, int rows, unsigned* bm, int* red, int& lo, int& words,
                              int& j0, int& j1)
    {
        const int64_t r0 = (int64_t)blockIdx.x * rows;
        const int64_t r1 = r0 + rows < m ? r0 + rows : m;
        j0               = rp[r0];
        j1               = rp[r1];
        int l = INT_MAX, h = -1;
        for(int j = j0 + threadIdx.x; j < j1; j += NT)
        {
            const int c = __ldg(ci + j);
            l           = min(l, c);
            h           = max(h, c);
        }
        lo = block_reduce<NT>(l, red, [](int a, int b) { return min(a, b); });
        h  = block_reduce<NT>(h, red, [](int a, int b) { return max(a, b); });
        if(j1 <= j0 || (int64_t)h - lo + 1 > kHaloBits)
            return false;
        words = (int)(((int64_t)h - lo + 1 + 31) >> 5);
        for(int w = threadIdx.x; w < words; w += NT)
            bm[w] = 0u;
        __syncthreads();
        for(int j = j0 + threadIdx.x; j < j1; j += NT)
        {
            const int off = __ldg(ci + j) - lo;
            atomicOr(bm + (off >> 5), 1u << (off & 31));
        }
        __syncthreads();
        return true;
    }

    // Distinct columns per chunk: hcnt[c] = count (0 for an empty chunk), or -1
    // (span beyond kHaloBits or more than kHaloCap columns).  stats: [0] largest
    // count, [1] chunks at -1, [2] sum of counts.
    template <int NT>
    __global__ void __launch_bounds__(NT)
        k_halo_count(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, int64_t m,
                     int rows, int32_t* __restrict__ hcnt, int* stats)
    {
        extern __shared__ unsigned halo_bm[];
        __shared__ int red[NT / 32];
        int            lo = 0, words = 0, j0 = 0, j1 = 0;
        const int      c  = blockIdx.x;
        if(!halo_mark<NT>(rp, ci, m, rows, halo_bm, red, lo, words, j0, j1))
        {
            if(threadIdx.x == 0)
            {
                hcnt[c] = j1 <= j0 ? 0 : -1;
                if(j1 > j0)
                    atomicAdd(stats + 1, 1);
            }
            return;
        }
        int cnt = 0;
        for(int w = threadIdx.x; w < words; w += NT)
            cnt += __popc(halo_bm[w]);
        cnt = block_reduce<NT>(cnt, red, [](int a, int b) { return a + b; });
        if(threadIdx.x == 0)
        {
            if(cnt > kHaloCap)
            {
                hcnt[c] = -1;
                atomicAdd(stats + 1, 1);
            }
            else
            {
                hcnt[c] = cnt;
                atomicMax(stats, cnt);
                atomicAdd(stats + 2, cnt);
            }
        }
    }

    // Chunk c's distinct columns in ascending order into hcol[c * slot ...] and,
    // for every entry, the position of its column in that list (hloc).
    template <int NT>
    __global__ void __launch_bounds__(NT)
        k_halo_fill(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, int64_t m,
                    int rows, const int32_t* __restrict__ hcnt, int slot,
                    int32_t* __restrict__ hcol, uint16_t* __restrict__ hloc)
    {
        extern __shared__ unsigned halo_bm[];
        uint16_t*  pre = reinterpret_cast<uint16_t*>(halo_bm + kHaloBits / 32);
        __shared__ int red[NT / 32];
        const int      c = blockIdx.x;
        if(hcnt[c] <= 0)
            return;
        int lo = 0, words = 0, j0 = 0, j1 = 0;
        if(!halo_mark<NT>(rp, ci, m, rows, halo_bm, red, lo, words, j0, j1))
            return; // not reached: the count pass staged this chunk
        // exclusive prefix of the per-word counts: contiguous word runs per thread
        const int per = (words + NT - 1) / NT;
        const int w0 = min(words, (int)threadIdx.x * per), w1 = min(words, w0 + per);
        int       own = 0;
        for(int w = w0; w < w1; w++)
            own += __popc(halo_bm[w]);
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        int       inc  = own;
#pragma unroll
        for(int o = 1; o < 32; o <<= 1)
        {
            const int t = __shfl_up_sync(0xffffffffu, inc, o);
            if(lane >= o)
                inc += t;
        }
        if(lane == 31)
            red[wid] = inc;
        __syncthreads();
        int run = inc - own;
        for(int k = 0; k < wid; k++)
            run += red[k];
        for(int w = w0; w < w1; w++)
        {
            pre[w] = (uint16_t)run;
            run += __popc(halo_bm[w]);
        }
        __syncthreads();
        int32_t* hc = hcol + (size_t)c * slot;
        for(int w = threadIdx.x; w < words; w += NT)
        {
            unsigned b = halo_bm[w];
            int      k = pre[w];
            while(b)
            {
                hc[k++] = lo + (w << 5) + (__ffs(b) - 1);
                b &= b - 1u;
            }
        }
        for(int j = j0 + threadIdx.x; j < j1; j += NT)
        {
            const int off = __ldg(ci + j) - lo;
            const int w   = off >> 5;
            hloc[j] = (uint16_t)(pre[w] + __popc(halo_bm[w] & ((1u << (off & 31)) - 1u)));
        }
    }

    // Rows per halo chunk: about kHaloEntries entries, at least four chunks per SM,
    // a whole number of VECTOR passes (256 / W rows) for the matrix's lane count.
    constexpr int kHaloEntries = 8192;
    static int halo_rows(const lab_csr_impl* A, int w)
    {
        const double avg    = (double)A->nnz / (double)A->m;
        const double target = std::min<double>(kHaloEntries,
                                                (double)A->nnz / (4.0 * (double)num_sms()));
        const int    pass   = std::max(1, kVectorNT / w);
        const int    r      = (int)(target / avg) / pass * pass;
        return std::max(pass, r);
    }

    // Largest power of two <= v, clamped to 2..32.
    static int pow2_at_most(double v)
    {
        int w = 2;
        while(w < 32 && 2 * w <= v)
            w <<= 1;
        return w;
    }

    // Halo plan of a square matrix (LAB_SPMV_VECTOR_HALO, and the autotuner's halo
    // candidates): distinct columns per chunk counted on the device and read back
    // (their largest count sizes the lists and the launch's shared memory), then the
    // lists and the per-entry positions written.  Built once per pattern; a matrix
    // whose chunks all read x directly gets none (halo_state -1).
    lab_status halo_build(lab_csr_impl* A, cudaStream_t s)
    {
        spmv_plan& p = A->plan;
        if(p.halo_state != 0)
            return LAB_OK;
        p.halo_state = -1;
        if(A->m != A->n || A->m == 0 || A->nnz == 0 || A->m > INT32_MAX)
            return LAB_OK;
        const double avg     = (double)A->nnz / (double)A->m;
        const int    w       = p.alg == LAB_SPMV_VECTOR ? p.lanes : pow2_at_most(avg / 5.0);
        const int    hrows   = halo_rows(A, w);
        const int    hchunks = (int)ceil_div<int64_t>(A->m, hrows);
        int          stats[3] = {0, 0, 0};
        int*         d        = nullptr;
        LAB_TRY(dalloc(&d, 3, s));
        LAB_CUDA(cudaMemsetAsync(d, 0, 3 * sizeof(int), s));
        LAB_TRY(dalloc(&p.hcnt, (size_t)hchunks, s));
        static const cudaError_t count_attr = cudaFuncSetAttribute(
            k_halo_count<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, kHaloBits / 8);
        LAB_CUDA(count_attr);
        LAB_LAUNCH(k_halo_count<256>, (unsigned)hchunks, 256, kHaloBits / 8, s, A->row_ptr,
                   A->col_ind, A->m, hrows, p.hcnt, d);
        const lab_status st = copy_d2h_sync(stats, d, sizeof(stats), s);
        dfree(d, s);
        LAB_TRY(st);
        const int slot = stats[0];
        if(slot == 0)
        {
            dfree(p.hcnt, s);
            p.hcnt = nullptr;
            return LAB_OK;
        }
        LAB_TRY(dalloc(&p.hcol, (size_t)hchunks * slot, s));
        LAB_TRY(dalloc(&p.hloc, (size_t)A->nnz, s));
        static const cudaError_t fill_attr =
            cudaFuncSetAttribute(k_halo_fill<256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 kHaloBits / 8 + kHaloBits / 16);
        LAB_CUDA(fill_attr);
        LAB_LAUNCH(k_halo_fill<256>, (unsigned)hchunks, 256, kHaloBits / 8 + kHaloBits / 16, s,
                   A->row_ptr, A->col_ind, A->m, hrows, p.hcnt, slot, p.hcol, p.hloc);
        p.halo_state = 1;
        p.hrows      = hrows;
        p.hchunks    = hchunks;
        p.hslot      = slot;
        p.hdirect    = stats[1];
        p.hdistinct  = stats[2];
        return LAB_OK;
    }

    // Schedule choice from row statistics.  Rows of at most 32 entries (stencils up
    // to 27 points) take the one-thread-per-row order (ROWSEQ: staged tiles for
    // <= 16, warp tiles for <= 32), whose fma chain matches the reference's host
    // SpMV bit for bit.  Longer rows (coarse AMG levels) take W lanes per row with
    // W the largest power of two <= mean row / 5 -- the fastest lane count measured
    // on B200 across the SA levels of 7- and 27-point operators (W = 4 at 23
    // entries, 8 at 41-73, 16 at 143-178, 16-32 beyond); lab_spmv_autotune times
    // every choice on the actual matrix instead.  vlanes is also the lane count of
    // SpMM and multicolour Gauss-Seidel on long rows.
    //
    // The same pass checks whether every column offset col - row fits in 16 bits;
    // then a 16-bit offset copy is built once per pattern and the row kernels read
    // it in place of the int32 columns in every precision (2 instead of 4 index
    // bytes per entry; the column, and so the arithmetic, is the same).
    // Analysis of several matrices with one host round trip: every matrix's statistics
    // kernels (and 16-bit offset copy) are enqueued, all statistics come back in one
    // copy, then each plan is finished.  Matrices already analysed are skipped.
    lab_status spmv_analyse_batch(lab_csr_impl* const* mats, int count, cudaStream_t s)
    {
        struct item
        {
            lab_csr_impl* A;
            int           st_rows = 0;
            bool          build   = false; // 16-bit offset copy enqueued
        };
        std::vector<item> todo;
        for(int k = 0; k < count; k++)
            if(mats[k] && !mats[k]->plan.analysed)
            {
                bool dup = false;
                for(const item& t : todo)
                    dup = dup || t.A == mats[k];
                if(!dup)
                    todo.push_back(item{mats[k]});
            }
        if(todo.empty())
            return LAB_OK;
        // per matrix: longest row, offsets too wide for 16 bits, largest stream tile
        const int        nt = (int)todo.size();
        std::vector<int> stats(3 * (size_t)nt, 0);
        int*             d  = nullptr;
        LAB_TRY(dalloc(&d, 3 * (size_t)nt, s));
        LAB_CUDA(cudaMemsetAsync(d, 0, 3 * sizeof(int) * (size_t)nt, s));
        lab_status st = LAB_OK;
        for(int k = 0; k < nt && st == LAB_OK; k++)
        {
            lab_csr_impl* A  = todo[k].A;
            int*          dk = d + 3 * k;
            if(A->m == 0)
                continue;
            st = [&]() -> lab_status {
                spmv_plan&     p    = A->plan;
                const unsigned grid = (unsigned)std::min<int64_t>(ceil_div<int64_t>(A->m, 256), 2048);
                LAB_LAUNCH(k_row_stats, grid, 256, 0, s, A->row_ptr, A->m, dk);
                if(A->m >= kStreamMinRows && A->nnz > 0)
                {
                    // tiles of at most about kStreamTileEntries entries and a whole
                    // number of consumer passes (8 warps x 32 / W rows, W the lane count
                    // the VECTOR plan takes), so every consumer warp has rows in every
                    // tile; a multiple of 4 rows keeps the row-pointer copy 16-byte aligned
                    const double avg = (double)A->nnz / (double)A->m;
                    const int    w   = p.forced && p.alg == LAB_SPMV_VECTOR ? p.lanes
                                                                           : pow2_at_most(avg / 5.0);
                    const int    rpp = kStreamConsumers * 32 / w;
                    const int    str =
                        std::min(1024, rpp * std::max(1, (int)(kStreamTileEntries / avg / rpp)));
                    todo[k].st_rows   = str;
                    const int64_t ntl = ceil_div<int64_t>(A->m, str);
                    LAB_LAUNCH(k_tile_max,
                               (unsigned)std::min<int64_t>(ceil_div<int64_t>(ntl, 256), 1024), 256, 0,
                               s, A->row_ptr, A->m, str, dk + 2);
                }
                // square matrices only: a prolongation's or restriction's col - row
                // spans the ratio of the two grids and does not fit
                if(A->lp.dcol_state == 0 && A->nnz > 0 && A->m == A->n)
                {
                    LAB_TRY(dalloc(&A->lp.dcol, (size_t)A->nnz, s));
                    todo[k].build = true;
                    // lanes per row: the largest power of two <= the mean row length
                    const double avg = (double)A->nnz / (double)A->m;
                    int          w   = 1;
                    while(w < 32 && 2 * w <= avg)
                        w <<= 1;
                    const unsigned g = (unsigned)std::min<int64_t>(
                        ceil_div<int64_t>(A->m * (int64_t)w, 256), (int64_t)num_sms() * 8);
                    switch(w)
                    {
                    case 1: LAB_LAUNCH(k_dcol_build<1>, g, 256, 0, s, A->row_ptr, A->col_ind, A->m, A->lp.dcol, dk + 1); break;
                    case 2: LAB_LAUNCH(k_dcol_build<2>, g, 256, 0, s, A->row_ptr, A->col_ind, A->m, A->lp.dcol, dk + 1); break;
                    case 4: LAB_LAUNCH(k_dcol_build<4>, g, 256, 0, s, A->row_ptr, A->col_ind, A->m, A->lp.dcol, dk + 1); break;
                    case 8: LAB_LAUNCH(k_dcol_build<8>, g, 256, 0, s, A->row_ptr, A->col_ind, A->m, A->lp.dcol, dk + 1); break;
                    case 16: LAB_LAUNCH(k_dcol_build<16>, g, 256, 0, s, A->row_ptr, A->col_ind, A->m, A->lp.dcol, dk + 1); break;
                    default: LAB_LAUNCH(k_dcol_build<32>, g, 256, 0, s, A->row_ptr, A->col_ind, A->m, A->lp.dcol, dk + 1); break;
                    }
                }
                return LAB_OK;
            }();
        }
        if(st == LAB_OK)
            st = copy_d2h_sync(stats.data(), d, sizeof(int) * stats.size(), s);
        dfree(d, s);
        if(st != LAB_OK)
        {
            // an enqueued offset copy whose check did not come back is dropped
            for(const item& t : todo)
                if(t.build)
                {
                    dfree(t.A->lp.dcol, s);
                    t.A->lp.dcol = nullptr;
                }
            return st;
        }
        for(int k = 0; k < nt; k++)
        {
            lab_csr_impl* A  = todo[k].A;
            spmv_plan&    p  = A->plan;
            const int*    sk = stats.data() + 3 * k;
            if(A->m > 0)
            {
                // stage capacity: the largest tile plus the alignment slack of its
                // copies (start rounded down to 16 bytes, quads read past the row end)
                const int cap = sk[2] + 16;
                p.st_rows     = todo[k].st_rows > 0 && cap <= kStreamMaxCap ? todo[k].st_rows : 0;
                p.st_cap      = p.st_rows ? cap : 0;
                if(todo[k].build)
                {
                    A->lp.dcol_state = sk[1] ? -1 : 1;
                    if(sk[1])
                    {
                        dfree(A->lp.dcol, s);
                        A->lp.dcol = nullptr;
                    }
                }
            }
            const int maxlen = sk[0];
            p.max_row        = maxlen;
            p.avg_row        = A->m > 0 ? (double)A->nnz / (double)A->m : 0.0;
            p.vlanes         = pow2_at_most(p.avg_row / 5.0);
            if(!p.forced)
            {
                p.alg   = maxlen <= 32 ? LAB_SPMV_ROWSEQ : LAB_SPMV_VECTOR;
                p.lanes = maxlen <= 32 ? 1 : p.vlanes;
            }
            p.analysed = 1;
            if(p.forced && p.alg == LAB_SPMV_VECTOR && p.halo_use && !p.stream &&
               p.halo_state == 0)
                LAB_TRY(halo_build(A, s));
        }
        return LAB_OK;
    }

    lab_status spmv_analyse(lab_csr_impl* A, cudaStream_t s)
    {
        return spmv_analyse_batch(&A, 1, s);
    }

    // SpMM: column-major X (n x k), Y (m x k); one pass over A per column block of
    // up to 8 right-hand sides, so A's bytes are read once per 8 columns.
    template <int K>
    __global__ void __launch_bounds__(256)
        k_spmm(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
               const double* __restrict__ v, int32_t m, const double* __restrict__ X,
               int64_t ldx, double* __restrict__ Y, int64_t ldy, double alpha, double beta,
               int lanes, const int* skip = nullptr)
    {
        if(skip && *skip)
            return;
        int64_t t    = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
        int     lane = (int)(t % lanes);
        int64_t row  = t / lanes;
        double  s[K];
#pragma unroll
        for(int k = 0; k < K; k++)
            s[k] = 0.0;
        if(row < m)
        {
            for(int j = rp[row] + lane; j < rp[row + 1]; j += lanes)
            {
                double  a = v[j];
                int64_t c = ci[j];
#pragma unroll
                for(int k = 0; k < K; k++)
                    s[k] = fma(a, __ldg(X + c + k * ldx), s[k]);
            }
        }
#pragma unroll
        for(int k = 0; k < K; k++)
            for(int o = lanes / 2; o > 0; o >>= 1)
                s[k] += __shfl_xor_sync(0xffffffffu, s[k], o, lanes);
        if(row < m && lane == 0)
        {
#pragma unroll
            for(int k = 0; k < K; k++)
            {
                double* y = Y + row + k * ldy;
                *y = beta == 0.0 ? alpha * s[k] : fma(alpha, s[k], beta * *y);
            }
        }
    }
}

namespace lab
{
    // Y[:, 0:k] = A X[:, 0:k] for k <= 8 columns in one pass over A (enqueue only).
    lab_status spmm_columns(const lab_csr_impl* A, int k, const double* X, int64_t ldx, double* Y,
                            int64_t ldy, cudaStream_t s, const int* skip)
    {
        if(A->m == 0 || k <= 0)
            return LAB_OK;
        int      lanes = A->plan.alg == LAB_SPMV_VECTOR ? A->plan.lanes
                       : (A->plan.max_row <= 32 ? 4 : A->plan.vlanes);
        unsigned grid  = (unsigned)ceil_div<int64_t>(A->m * (int64_t)lanes, 256);
        int32_t  m     = (int32_t)A->m;
        if(k == 8)
            LAB_LAUNCH(k_spmm<8>, grid, 256, 0, s, A->row_ptr, A->col_ind, A->val, m, X, ldx, Y,
                       ldy, 1.0, 0.0, lanes, skip);
        else if(k == 4)
            LAB_LAUNCH(k_spmm<4>, grid, 256, 0, s, A->row_ptr, A->col_ind, A->val, m, X, ldx, Y,
                       ldy, 1.0, 0.0, lanes, skip);
        else
            for(int q = 0; q < k; q++)
                LAB_LAUNCH(k_spmm<1>, grid, 256, 0, s, A->row_ptr, A->col_ind, A->val, m,
                           X + q * ldx, ldx, Y + q * ldy, ldy, 1.0, 0.0, lanes, skip);
        return LAB_OK;
    }
}

using namespace lab;

extern "C" {

LAB_API lab_status lab_spmv_analysis(lab_csr A, lab_stream s)
{
    LAB_ARG(A, "null matrix");
    LAB_TRY(ensure_init());
    return spmv_analyse(A, to_stream(s));
}

LAB_API lab_status lab_spmv_set_algorithm(lab_csr A, lab_spmv_alg alg, int lanes)
{
    LAB_ARG(A, "null matrix");
    LAB_ARG(lanes == 0 || lanes == 1 || lanes == 2 || lanes == 4 || lanes == 8 || lanes == 16 ||
                lanes == 32,
            "lanes must be a power of two <= 32");
    if(alg == LAB_SPMV_AUTO)
    {
        A->plan.forced   = 0;
        A->plan.analysed = 0;
        A->plan.stream   = 0;
        A->plan.halo_use = 0;
        return LAB_OK;
    }
    LAB_ARG(alg == LAB_SPMV_ROWSEQ || alg == LAB_SPMV_VECTOR || alg == LAB_SPMV_MERGE ||
                alg == LAB_SPMV_VECTOR_STREAM || alg == LAB_SPMV_VECTOR_HALO,
            "unknown algorithm");
    A->plan.forced   = 1;
    A->plan.analysed = 0;
    A->plan.stream   = alg == LAB_SPMV_VECTOR_STREAM;
    A->plan.halo_use = alg == LAB_SPMV_VECTOR_HALO;
    if(alg == LAB_SPMV_ROWSEQ)
    {
        A->plan.alg   = LAB_SPMV_ROWSEQ;
        A->plan.lanes = 1;
    }
    else
    {
        // The merge-path schedule is served by the 32-lane vector kernel.
        A->plan.alg   = LAB_SPMV_VECTOR;
        A->plan.lanes = alg == LAB_SPMV_MERGE ? 32 : (lanes > 1 ? lanes : 8);
    }
    return LAB_OK;
}

LAB_API lab_status lab_spmv_get_algorithm(lab_csr A, int* alg, int* lanes)
{
    LAB_ARG(A, "null matrix");
    const spmv_plan& p = A->plan;
    if(alg)
        *alg = p.alg == LAB_SPMV_VECTOR && p.stream && p.st_rows > 0 ? LAB_SPMV_VECTOR_STREAM
               : p.alg == LAB_SPMV_VECTOR && !p.stream && p.halo_use && p.halo_state == 1
                   ? LAB_SPMV_VECTOR_HALO
                   : p.alg;
    if(lanes)
        *lanes = p.lanes;
    return LAB_OK;
}

LAB_API lab_status lab_spmv_halo_info(lab_csr A, int64_t* chunks, int64_t* rows_per_chunk,
                                      int64_t* distinct, int64_t* direct_chunks)
{
    LAB_ARG(A, "null matrix");
    const spmv_plan& p    = A->plan;
    const bool       have = p.halo_state == 1;
    if(chunks)
        *chunks = have ? p.hchunks : 0;
    if(rows_per_chunk)
        *rows_per_chunk = have ? p.hrows : 0;
    if(distinct)
        *distinct = have ? p.hdistinct : 0;
    if(direct_chunks)
        *direct_chunks = have ? p.hdirect : 0;
    return LAB_OK;
}

LAB_API lab_status lab_spmv(double alpha, lab_csr A, const double* x, double beta, double* y,
                            lab_stream ls)
{
    LAB_ARG(A, "null matrix");
    LAB_ARG(A->m == 0 || y, "null y");
    LAB_ARG(A->n == 0 || x, "null x");
    LAB_TRY(ensure_init());
    cudaStream_t s = to_stream(ls);
    LAB_TRY(spmv_analyse(A, s));
    op_spmv op{x, y, alpha, beta};
    return launch_rowop(A, A->val, op, s);
}

LAB_API lab_status lab_residual(lab_csr A, const double* x, const double* b, double* r,
                                lab_stream ls)
{
    LAB_ARG(A, "null matrix");
    LAB_ARG(A->m == 0 || (b && r), "null vector");
    LAB_TRY(ensure_init());
    cudaStream_t s = to_stream(ls);
    LAB_TRY(spmv_analyse(A, s));
    op_residual op{x, b, r};
    return launch_rowop(A, A->val, op, s);
}

LAB_API lab_status lab_spmm(double alpha, lab_csr A, int nrhs, const double* X, int64_t ldx,
                            double beta, double* Y, int64_t ldy, lab_stream ls)
{
    LAB_ARG(A, "null matrix");
    LAB_ARG(nrhs >= 0, "negative nrhs");
    LAB_ARG(ldx >= A->n && ldy >= A->m, "leading dimension too small");
    LAB_TRY(ensure_init());
    cudaStream_t s = to_stream(ls);
    LAB_TRY(spmv_analyse(A, s));
    if(A->m == 0)
        return LAB_OK;
    int      lanes = A->plan.alg == LAB_SPMV_VECTOR ? A->plan.lanes
                       : (A->plan.max_row <= 32 ? 4 : A->plan.vlanes);
    unsigned grid  = (unsigned)ceil_div<int64_t>(A->m * (int64_t)lanes, 256);
    for(int c = 0; c < nrhs; c += 8)
    {
        int           k  = std::min(8, nrhs - c);
        const double* Xc = X + (int64_t)c * ldx;
        double*       Yc = Y + (int64_t)c * ldy;
        int32_t       m  = (int32_t)A->m;
        switch(k)
        {
        case 8:
            LAB_LAUNCH(k_spmm<8>, grid, 256, 0, s, A->row_ptr, A->col_ind, A->val, m, Xc, ldx, Yc,
                       ldy, alpha, beta, lanes);
            break;
        case 4:
            LAB_LAUNCH(k_spmm<4>, grid, 256, 0, s, A->row_ptr, A->col_ind, A->val, m, Xc, ldx, Yc,
                       ldy, alpha, beta, lanes);
            break;
        default:
            for(int q = 0; q < k; q++)
                LAB_LAUNCH(k_spmm<1>, grid, 256, 0, s, A->row_ptr, A->col_ind, A->val, m,
                           Xc + q * ldx, ldx, Yc + q * ldy, ldy, alpha, beta, lanes);
            break;
        }
    }
    return LAB_OK;
}

} // extern "C"
