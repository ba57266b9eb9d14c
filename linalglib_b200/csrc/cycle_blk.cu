// Block V-cycle: the AMG preconditioner applied to up to 8 right-hand sides in
// one pass over every level operator.  Block vectors hold K columns interleaved
// per row (entry (i, k) at i*K + k), so one gather fetches the K values of a
// column index with 16-byte loads and each matrix entry read from HBM serves K
// products.  Every column sees exactly the arithmetic of the single-vector FP64
// cycle (same fused passes, same schedule and accumulation order per level), so a
// block application equals K single applications bit for bit (a level forced onto
// one thread per row with rows longer than 32 entries is the exception: there the
// block pass uses W lanes per row).  Covered: V-cycle, Jacobi smoothing (any n1,
// n2, omega), FP64, 1x1 or dense-inverse coarsest solve; anything else is applied
// column by column by the caller.
#include "cycle.cuh"

#include <map>
#include <mutex>

namespace lab
{
    constexpr int kBlkMax = 8;

    template <int K>
    __device__ __forceinline__ void ldk(const double* __restrict__ p, double (&o)[K])
    {
        if constexpr(K % 2 == 0)
        {
#pragma unroll
            for(int k = 0; k < K; k += 2)
            {
                const double2 t = __ldg(reinterpret_cast<const double2*>(p + k));
                o[k]            = t.x;
                o[k + 1]        = t.y;
            }
        }
        else
        {
#pragma unroll
            for(int k = 0; k < K; k++)
                o[k] = __ldg(p + k);
        }
    }

    // ------------------------------------------------------------ block ops
    // Same formulas as op_pre0 / op_jacobi / op_res / op_prolong / op_restrict.
    template <int K>
    struct bop_pre0
    {
        const double* __restrict__ b;
        const double* __restrict__ invd;
        double omega;
        double* __restrict__ x;
        double* __restrict__ r;
        __device__ __forceinline__ void gather(int c, double (&g)[K]) const
        {
            double bv[K];
            ldk<K>(b + (size_t)c * K, bv);
            const double ic = __ldg(invd + c);
#pragma unroll
            for(int k = 0; k < K; k++)
                g[k] = omega * (ic * bv[k]);
        }
        __device__ __forceinline__ void finish(int i, const double (&s)[K]) const
        {
            double bv[K];
            ldk<K>(b + (size_t)i * K, bv);
            const double ii = __ldg(invd + i);
#pragma unroll
            for(int k = 0; k < K; k++)
            {
                x[(size_t)i * K + k] = omega * (ii * bv[k]);
                r[(size_t)i * K + k] = bv[k] - s[k];
            }
        }
    };

    template <int K>
    struct bop_jacobi
    {
        const double* __restrict__ x;
        const double* __restrict__ b;
        const double* __restrict__ invd;
        double omega;
        double* __restrict__ y;
        __device__ __forceinline__ void gather(int c, double (&g)[K]) const
        {
            ldk<K>(x + (size_t)c * K, g);
        }
        __device__ __forceinline__ void finish(int i, const double (&s)[K]) const
        {
            double xv[K], bv[K];
            ldk<K>(x + (size_t)i * K, xv);
            ldk<K>(b + (size_t)i * K, bv);
            const double ii = __ldg(invd + i);
#pragma unroll
            for(int k = 0; k < K; k++)
                y[(size_t)i * K + k] = xv[k] + omega * (ii * (bv[k] - s[k]));
        }
    };

    template <int K>
    struct bop_res
    {
        const double* __restrict__ x;
        const double* __restrict__ b;
        double* __restrict__ r;
        __device__ __forceinline__ void gather(int c, double (&g)[K]) const
        {
            ldk<K>(x + (size_t)c * K, g);
        }
        __device__ __forceinline__ void finish(int i, const double (&s)[K]) const
        {
            double bv[K];
            ldk<K>(b + (size_t)i * K, bv);
#pragma unroll
            for(int k = 0; k < K; k++)
                r[(size_t)i * K + k] = bv[k] - s[k];
        }
    };

    // y = x + P e; x and y may alias (each row reads and writes only its own entries)
    template <int K>
    struct bop_prolong
    {
        const double* __restrict__ e;
        const double* x;
        double*       y;
        __device__ __forceinline__ void gather(int c, double (&g)[K]) const
        {
            ldk<K>(e + (size_t)c * K, g);
        }
        __device__ __forceinline__ void finish(int i, const double (&s)[K]) const
        {
#pragma unroll
            for(int k = 0; k < K; k++)
                y[(size_t)i * K + k] = x[(size_t)i * K + k] + s[k];
        }
    };

    template <int K>
    struct bop_restrict
    {
        const double* __restrict__ r;
        double* __restrict__ y;
        __device__ __forceinline__ void gather(int c, double (&g)[K]) const
        {
            ldk<K>(r + (size_t)c * K, g);
        }
        __device__ __forceinline__ void finish(int i, const double (&s)[K]) const
        {
#pragma unroll
            for(int k = 0; k < K; k++)
                y[(size_t)i * K + k] = s[k];
        }
    };

    // ------------------------------------------------------------ block row kernels
    // One thread per row over staged tiles (the ROWSEQ schedule of k_pipe, with K
    // accumulators): CSR-order fma chains, gathers issued CH entries at a time.
    template <class Op, int NT, int MAXR, int K>
    __global__ void __launch_bounds__(NT)
        k_blk_pipe(csr_view<double> A, Op op, int cap, int ntiles, const int* skip)
    {
        constexpr int VPC = 2;
        constexpr int CH  = (16 / K) > 0 ? 16 / K : 1;
        extern __shared__ __align__(16) unsigned char smem_raw[];
        const size_t sv_b    = ((size_t)(cap + 16) * sizeof(double) + 15) / 16 * 16;
        const size_t sc_b    = ((size_t)(cap + 16) * 4 + 15) / 16 * 16;
        const size_t stage_b = pipe_stage_bytes<double>(cap, NT);
        if(skip && *skip)
            return;
        auto issue = [&](int tile, int stage) {
            const int      r0   = tile * NT;
            const int      r1   = min(r0 + NT, A.m);
            const int      j0   = A.rp[r0];
            const int      j1   = A.rp[r1];
            const int      j0v  = j0 & ~(VPC - 1), j0c = j0 & ~3;
            unsigned char* base = smem_raw + stage * stage_b;
            int32_t*       sr   = reinterpret_cast<int32_t*>(base + sv_b + sc_b);
            const int      nr   = (r1 - r0 + 1 + 3) / 4;
            for(int k = threadIdx.x; k < nr; k += NT)
                cp_async16(sr + 4 * k, A.rp + r0 + 4 * k);
            if((j1 - j0v) <= cap + 8 && (j1 - j0c) <= cap + 4)
            {
                double*   sv = reinterpret_cast<double*>(base);
                int32_t*  sc = reinterpret_cast<int32_t*>(base + sv_b);
                const int nv = (j1 - j0v + VPC - 1) / VPC;
                const int nc = (j1 - j0c + 3) / 4;
                for(int k = threadIdx.x; k < nv; k += NT)
                    cp_async16(sv + (size_t)k * VPC, A.v + j0v + (size_t)k * VPC);
                for(int k = threadIdx.x; k < nc; k += NT)
                    cp_async16(sc + (size_t)k * 4, A.ci + j0c + (size_t)k * 4);
            }
        };
        int tile = blockIdx.x;
        if(tile < ntiles)
            issue(tile, 0);
        cp_async_commit();
        for(int it = 0; tile < ntiles; it++, tile += gridDim.x)
        {
            const int nxt = tile + gridDim.x;
            if(nxt < ntiles)
                issue(nxt, (it + 1) & 1);
            cp_async_commit();
            cp_async_wait_group<1>();
            __syncthreads();
            const unsigned char* base   = smem_raw + (it & 1) * stage_b;
            const double*        sv     = reinterpret_cast<const double*>(base);
            const int32_t*       sc     = reinterpret_cast<const int32_t*>(base + sv_b);
            const int32_t*       sr     = reinterpret_cast<const int32_t*>(base + sv_b + sc_b);
            const int            r0     = tile * NT;
            const int            r1     = min(r0 + NT, A.m);
            const int            j0     = sr[0], j1 = sr[r1 - r0];
            const int            j0v    = j0 & ~(VPC - 1), j0c = j0 & ~3;
            const bool           staged = (j1 - j0v) <= cap + 8 && (j1 - j0c) <= cap + 4;
            const int            row    = r0 + threadIdx.x;
            if(row < r1)
            {
                const int a = sr[row - r0], b = sr[row - r0 + 1];
                double    s[K];
#pragma unroll
                for(int k = 0; k < K; k++)
                    s[k] = 0.0;
                if(staged)
                {
                    for(int c0 = a; c0 < b; c0 += CH)
                    {
                        double g[CH][K];
#pragma unroll
                        for(int q = 0; q < CH; q++)
                            if(c0 + q < b)
                                op.gather(sc[c0 + q - j0c], g[q]);
#pragma unroll
                        for(int q = 0; q < CH; q++)
                            if(c0 + q < b)
                            {
                                const double v = sv[c0 + q - j0v];
#pragma unroll
                                for(int k = 0; k < K; k++)
                                    s[k] = fma(v, g[q][k], s[k]);
                            }
                    }
                }
                else
                {
                    for(int j = a; j < b; j++)
                    {
                        double g[K];
                        op.gather(A.ci[j], g);
                        const double v = A.v[j];
#pragma unroll
                        for(int k = 0; k < K; k++)
                            s[k] = fma(v, g[k], s[k]);
                    }
                }
                op.finish(row, s);
            }
            __syncthreads();
        }
        cp_async_wait_group<0>();
    }

    // W lanes per row, lane-strided partial sums and an xor-shuffle reduction per
    // column (the VECTOR schedule of k_vector with K accumulators).
    template <class Op, int NT, int W, int K>
    __global__ void __launch_bounds__(NT)
        k_blk_vector(csr_view<double> A, Op op, const int* skip)
    {
        if(skip && *skip)
            return;
        const int lane = threadIdx.x & (W - 1);
        const int row  = (int)(((int64_t)blockIdx.x * NT + threadIdx.x) / W);
        double    s[K];
#pragma unroll
        for(int k = 0; k < K; k++)
            s[k] = 0.0;
        if(row < A.m)
        {
            const int a = A.rp[row], b = A.rp[row + 1];
            for(int j = a + lane; j < b; j += W)
            {
                double g[K];
                op.gather(A.ci[j], g);
                const double v = A.v[j];
#pragma unroll
                for(int k = 0; k < K; k++)
                    s[k] = fma(v, g[k], s[k]);
            }
        }
#pragma unroll
        for(int k = 0; k < K; k++)
#pragma unroll
            for(int o = W / 2; o > 0; o >>= 1)
                s[k] += __shfl_xor_sync(0xffffffffu, s[k], o, W);
        if(row < A.m && lane == 0)
            op.finish(row, s);
    }

    template <class Op, int MAXR, int K>
    static int blk_pipe_occupancy(size_t smem)
    {
        const auto                   kernel = k_blk_pipe<Op, kRowseqNT, MAXR, K>;
        static std::mutex            mu;
        static std::map<size_t, int> cache;
        static const cudaError_t     attr = cudaFuncSetAttribute(
            kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        (void)attr;
        std::lock_guard<std::mutex> g(mu);
        auto                        it = cache.find(smem);
        if(it != cache.end())
            return it->second;
        int occ = 0;
        if(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, kRowseqNT, smem) !=
           cudaSuccess)
        {
            cudaGetLastError();
            occ = 1;
        }
        occ         = std::max(occ, 1);
        cache[smem] = occ;
        return occ;
    }

    template <class Op, int MAXR, int K>
    static lab_status blk_pipe(const csr_view<double>& V, const Op& op, int cap, cudaStream_t s,
                               const int* skip)
    {
        const int      ntiles = (int)ceil_div<int64_t>(V.m, kRowseqNT);
        const size_t   smem   = 2 * pipe_stage_bytes<double>(cap, kRowseqNT);
        const int      occ    = blk_pipe_occupancy<Op, MAXR, K>(smem);
        const unsigned grid   = (unsigned)std::min<int64_t>(ntiles, (int64_t)num_sms() * occ);
        LAB_LAUNCH((k_blk_pipe<Op, kRowseqNT, MAXR, K>), grid, kRowseqNT, smem, s, V, op, cap,
                   ntiles, skip);
        return LAB_OK;
    }

    template <class Op, int W, int K>
    static lab_status blk_vector(const csr_view<double>& V, const Op& op, cudaStream_t s,
                                 const int* skip)
    {
        const unsigned grid = (unsigned)ceil_div<int64_t>((int64_t)V.m * W, kVectorNT);
        LAB_LAUNCH((k_blk_vector<Op, kVectorNT, W, K>), grid, kVectorNT, 0, s, V, op, skip);
        return LAB_OK;
    }

    // The schedule of the matrix's SpMV plan, with K accumulators.
    template <int K, class Op>
    static lab_status blk_rowop(const lab_csr_impl* A, const Op& op, cudaStream_t s,
                                const int* skip)
    {
        if(A->m == 0)
            return LAB_OK;
        csr_view<double> V{A->row_ptr, A->col_ind, A->val, (int32_t)A->m};
        const spmv_plan& p = A->plan;
        if(p.alg == LAB_SPMV_ROWSEQ)
        {
            const int mr = std::max(1, p.max_row);
            if(mr <= 8)
                return blk_pipe<Op, 8, K>(V, op, kRowseqNT * mr, s, skip);
            if(mr <= 16)
                return blk_pipe<Op, 16, K>(V, op, kRowseqNT * mr, s, skip);
            if(mr <= 32)
                return blk_pipe<Op, 32, K>(V, op, kRowseqNT * mr, s, skip);
        }
        // long rows: W lanes per row, as the single-vector VECTOR schedule
        switch(p.alg == LAB_SPMV_VECTOR ? p.lanes : p.vlanes)
        {
        case 2:
            return blk_vector<Op, 2, K>(V, op, s, skip);
        case 4:
            return blk_vector<Op, 4, K>(V, op, s, skip);
        case 8:
            return blk_vector<Op, 8, K>(V, op, s, skip);
        case 16:
            return blk_vector<Op, 16, K>(V, op, s, skip);
        default:
            return blk_vector<Op, 32, K>(V, op, s, skip);
        }
    }

    // ------------------------------------------------------------ small kernels
    template <int K>
    __global__ void k_to_blk(const double* __restrict__ r, int64_t ld, int64_t n,
                             double* __restrict__ rb, const int* skip)
    {
        if(skip && *skip)
            return;
        for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
            i += (int64_t)gridDim.x * blockDim.x)
#pragma unroll
            for(int k = 0; k < K; k++)
                rb[i * K + k] = r[k * ld + i];
    }

    template <int K>
    __global__ void k_from_blk(const double* __restrict__ zb, int64_t n, double* __restrict__ z,
                               int64_t ld, const int* skip)
    {
        if(skip && *skip)
            return;
        for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
            i += (int64_t)gridDim.x * blockDim.x)
#pragma unroll
            for(int k = 0; k < K; k++)
                z[k * ld + i] = zb[i * K + k];
    }

    __global__ void k_blk_zero(double* x, int64_t n, const int* skip)
    {
        if(skip && *skip)
            return;
        for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
            i += (int64_t)gridDim.x * blockDim.x)
            x[i] = 0.0;
    }

    template <int K>
    __global__ void k_blk_coarse1(const double* a, const double* b, double* x, const int* skip)
    {
        if(skip && *skip)
            return;
        if(threadIdx.x < K)
            x[threadIdx.x] = __ddiv_rn(b[threadIdx.x], a[0]);
    }

    // x = Ainv b per column, the single-vector kernel's order (lane-strided fma, warp sum)
    template <int K>
    __global__ void k_blk_coarse_dense(const double* __restrict__ Ainv, const double* __restrict__ b,
                                       double* __restrict__ x, int n, const int* skip)
    {
        if(skip && *skip)
            return;
        const int row  = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
        const int lane = threadIdx.x & 31;
        if(row >= n)
            return;
        double s[K];
#pragma unroll
        for(int k = 0; k < K; k++)
            s[k] = 0.0;
        for(int j = lane; j < n; j += 32)
        {
            const double a = Ainv[(size_t)row * n + j];
#pragma unroll
            for(int k = 0; k < K; k++)
                s[k] = fma(a, b[(size_t)j * K + k], s[k]);
        }
#pragma unroll
        for(int k = 0; k < K; k++)
        {
            const double t = warp_sum(s[k]);
            if(lane == 0)
                x[(size_t)row * K + k] = t;
        }
    }

    // ------------------------------------------------------------ the recursion
    template <int K>
    static lab_status cycle_blk(hierarchy_impl* h, int l, double* x, const double* b,
                                const cyc_ctx& c)
    {
        const lab_amg_options* o = c.o;
        if(l == h->levels)
        {
            const lab_csr_impl* A = h->A[l];
            if(A->m == 1)
                LAB_LAUNCH(k_blk_coarse1<K>, 1, 32, 0, c.s, (const double*)A->val, b, x, c.skip);
            else if(A->m > 1)
                LAB_LAUNCH(k_blk_coarse_dense<K>, (unsigned)ceil_div<int64_t>(A->m, 8), 256, 0, c.s,
                           (const double*)h->coarse_inv, b, x, (int)A->m, c.skip);
            return LAB_OK;
        }
        lab_csr_impl* A    = h->A[l];
        lab_csr_impl* P    = h->P[l];
        lab_csr_impl* R    = h->R[l];
        level_ws&     w    = h->ws[l];
        level_ws&     wc   = h->ws[l + 1];
        const int64_t m    = A->m;
        const int     n1   = o->n1, n2 = o->n2;
        const double  om   = o->omega;
        const double* invd = A->invdiag;
        double*       r    = w.rk;
        // start in the buffer that makes the last write land in x
        double*   cur   = x;
        double*   oth   = w.tk;
        const int flips = (n1 >= 1 ? n1 - 1 : n1) + 1 + n2;
        if(flips & 1)
        {
            cur = w.tk;
            oth = x;
        }
        auto jacobi = [&]() -> lab_status {
            bop_jacobi<K> op{cur, b, invd, om, oth};
            LAB_TRY(blk_rowop<K>(A, op, c.s, c.skip));
            std::swap(cur, oth);
            return LAB_OK;
        };
        if(n1 >= 1)
        {
            bop_pre0<K> op{b, invd, om, cur, r};
            LAB_TRY(blk_rowop<K>(A, op, c.s, c.skip));
            for(int k = 1; k < n1; k++)
                LAB_TRY(jacobi());
            if(n1 > 1)
            {
                bop_res<K> opr{cur, b, r};
                LAB_TRY(blk_rowop<K>(A, opr, c.s, c.skip));
            }
        }
        else
        {
            LAB_LAUNCH(k_blk_zero, grid_for(m * K), 256, 0, c.s, cur, m * K, c.skip);
            bop_res<K> opr{cur, b, r};
            LAB_TRY(blk_rowop<K>(A, opr, c.s, c.skip));
        }
        bop_restrict<K> opr{r, wc.bk};
        LAB_TRY(blk_rowop<K>(R, opr, c.s, c.skip));
        LAB_TRY(cycle_blk<K>(h, l + 1, wc.xk, wc.bk, c));
        bop_prolong<K> opp{wc.xk, cur, oth};
        LAB_TRY(blk_rowop<K>(P, opp, c.s, c.skip));
        std::swap(cur, oth);
        for(int k = 0; k < n2; k++)
            LAB_TRY(jacobi());
        if(cur != x)
        {
            set_error("block cycle: internal buffer parity");
            return LAB_BAD_ARG;
        }
        return LAB_OK;
    }

    bool cycle_block_supported(const hierarchy_impl* h, const lab_amg_options* o)
    {
        if(o->cycle != LAB_CYCLE_V || o->smoother != LAB_SMOOTH_JACOBI ||
           o->precision != LAB_PREC_FP64 || o->n1 < 0 || o->n2 < 0)
            return false;
        const lab_csr_impl* Ac = h->A[h->levels];
        return Ac->m <= 1 || (o->coarse == LAB_COARSE_DIRECT && h->coarse_inv);
    }

    lab_status cycle_prepare_block(hierarchy_impl* h, cudaStream_t s)
    {
        for(int l = 0; l <= h->levels; l++)
        {
            level_ws&    w = h->ws[l];
            const size_t n = (size_t)h->A[l]->m * kBlkMax + 8;
            if(!w.xk)
            {
                LAB_TRY(dalloc(&w.xk, n, s));
                LAB_TRY(dalloc(&w.bk, n, s));
                LAB_TRY(dalloc(&w.rk, n, s));
                LAB_TRY(dalloc(&w.tk, n, s));
            }
        }
        return LAB_OK;
    }

    template <int K>
    static lab_status precond_group(hierarchy_impl* h, const cyc_ctx& c, const double* r,
                                    int64_t ldr, double* z, int64_t ldz)
    {
        const int64_t n  = h->A[0]->m;
        level_ws&     w0 = h->ws[0];
        const unsigned g = grid_for(n);
        LAB_LAUNCH(k_to_blk<K>, g, 256, 0, c.s, r, ldr, n, w0.bk, c.skip);
        LAB_TRY(cycle_blk<K>(h, 0, w0.xk, w0.bk, c));
        LAB_LAUNCH(k_from_blk<K>, g, 256, 0, c.s, (const double*)w0.xk, n, z, ldz, c.skip);
        return LAB_OK;
    }

    lab_status cycle_precond_block(hierarchy_impl* h, const cyc_ctx& c, int ncols, const double* r,
                                   int64_t ldr, double* z, int64_t ldz)
    {
        int col = 0;
        while(col < ncols)
        {
            const int left = ncols - col;
            const int k    = left >= 8 ? 8 : left >= 4 ? 4 : left >= 2 ? 2 : 1;
            const double* rc = r + (int64_t)col * ldr;
            double*       zc = z + (int64_t)col * ldz;
            switch(k)
            {
            case 8:
                LAB_TRY(precond_group<8>(h, c, rc, ldr, zc, ldz));
                break;
            case 4:
                LAB_TRY(precond_group<4>(h, c, rc, ldr, zc, ldz));
                break;
            case 2:
                LAB_TRY(precond_group<2>(h, c, rc, ldr, zc, ldz));
                break;
            default:
                LAB_TRY(precond_group<1>(h, c, rc, ldr, zc, ldz));
                break;
            }
            col += k;
        }
        return LAB_OK;
    }
}
