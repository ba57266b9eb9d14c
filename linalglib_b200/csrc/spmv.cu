// SpMV front end: analysis (row statistics -> schedule), y = alpha*A*x + beta*y,
// residual, multi-vector SpMM.
#include "spmv_engine.cuh"

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

    // Largest power of two <= v, clamped to 2..32.
    static int pow2_at_most(double v)
    {
        int w = 2;
        while(w < 32 && 2 * w <= v)
            w <<= 1;
        return w;
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
    lab_status spmv_analyse(lab_csr_impl* A, cudaStream_t s)
    {
        spmv_plan& p = A->plan;
        if(p.analysed)
            return LAB_OK;
        // longest row, offsets too wide for 16 bits, largest stream tile
        int stats[3] = {0, 0, 0};
        int st_rows  = 0;
        if(A->m > 0)
        {
            int* d = nullptr;
            LAB_TRY(dalloc(&d, 3, s));
            LAB_CUDA(cudaMemsetAsync(d, 0, 3 * sizeof(int), s));
            unsigned grid = (unsigned)std::min<int64_t>(ceil_div<int64_t>(A->m, 256), 2048);
            LAB_LAUNCH(k_row_stats, grid, 256, 0, s, A->row_ptr, A->m, d);
            if(A->m >= kStreamMinRows && A->nnz > 0)
            {
                // tiles of at most about kStreamTileEntries entries and a whole number
                // of consumer passes (8 warps x 32 / W rows, W the lane count the
                // VECTOR plan takes), so every consumer warp has rows in every tile;
                // a multiple of 4 rows keeps the row-pointer copy 16-byte aligned
                const double avg = (double)A->nnz / (double)A->m;
                const int    w   = p.forced && p.alg == LAB_SPMV_VECTOR ? p.lanes
                                                                       : pow2_at_most(avg / 5.0);
                const int    rpp = kStreamConsumers * 32 / w;
                st_rows = std::min(1024, rpp * std::max(1, (int)(kStreamTileEntries / avg / rpp)));
                const int64_t nt = ceil_div<int64_t>(A->m, st_rows);
                LAB_LAUNCH(k_tile_max, (unsigned)std::min<int64_t>(ceil_div<int64_t>(nt, 256), 1024),
                           256, 0, s, A->row_ptr, A->m, st_rows, d + 2);
            }
            // square matrices only: a prolongation's or restriction's col - row
            // spans the ratio of the two grids and does not fit
            const bool build = A->lp.dcol_state == 0 && A->nnz > 0 && A->m == A->n;
            if(build)
            {
                LAB_TRY(dalloc(&A->lp.dcol, (size_t)A->nnz, s));
                // lanes per row: the largest power of two <= the mean row length
                const double avg = (double)A->nnz / (double)A->m;
                int          w   = 1;
                while(w < 32 && 2 * w <= avg)
                    w <<= 1;
                const unsigned g = (unsigned)std::min<int64_t>(
                    ceil_div<int64_t>(A->m * (int64_t)w, 256), (int64_t)num_sms() * 8);
                switch(w)
                {
                case 1: LAB_LAUNCH(k_dcol_build<1>, g, 256, 0, s, A->row_ptr, A->col_ind, A->m, A->lp.dcol, d + 1); break;
                case 2: LAB_LAUNCH(k_dcol_build<2>, g, 256, 0, s, A->row_ptr, A->col_ind, A->m, A->lp.dcol, d + 1); break;
                case 4: LAB_LAUNCH(k_dcol_build<4>, g, 256, 0, s, A->row_ptr, A->col_ind, A->m, A->lp.dcol, d + 1); break;
                case 8: LAB_LAUNCH(k_dcol_build<8>, g, 256, 0, s, A->row_ptr, A->col_ind, A->m, A->lp.dcol, d + 1); break;
                case 16: LAB_LAUNCH(k_dcol_build<16>, g, 256, 0, s, A->row_ptr, A->col_ind, A->m, A->lp.dcol, d + 1); break;
                default: LAB_LAUNCH(k_dcol_build<32>, g, 256, 0, s, A->row_ptr, A->col_ind, A->m, A->lp.dcol, d + 1); break;
                }
            }
            lab_status st = copy_d2h_sync(stats, d, sizeof(stats), s);
            dfree(d, s);
            LAB_TRY(st);
            // stage capacity: the largest tile plus the alignment slack of its copies
            // (start rounded down to 16 bytes, quads read past the row end)
            const int cap = stats[2] + 16;
            p.st_rows     = st_rows > 0 && cap <= kStreamMaxCap ? st_rows : 0;
            p.st_cap      = p.st_rows ? cap : 0;
            if(build)
            {
                A->lp.dcol_state = stats[1] ? -1 : 1;
                if(stats[1])
                {
                    dfree(A->lp.dcol, s);
                    A->lp.dcol = nullptr;
                }
            }
        }
        const int maxlen = stats[0];
        p.max_row = maxlen;
        p.avg_row = A->m > 0 ? (double)A->nnz / (double)A->m : 0.0;
        p.vlanes  = pow2_at_most(p.avg_row / 5.0);
        if(!p.forced)
        {
            p.alg   = maxlen <= 32 ? LAB_SPMV_ROWSEQ : LAB_SPMV_VECTOR;
            p.lanes = maxlen <= 32 ? 1 : p.vlanes;
        }
        p.analysed = 1;
        return LAB_OK;
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
        return LAB_OK;
    }
    LAB_ARG(alg == LAB_SPMV_ROWSEQ || alg == LAB_SPMV_VECTOR || alg == LAB_SPMV_MERGE ||
                alg == LAB_SPMV_VECTOR_STREAM,
            "unknown algorithm");
    A->plan.forced   = 1;
    A->plan.analysed = 0;
    A->plan.stream   = alg == LAB_SPMV_VECTOR_STREAM;
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
    if(alg)
        *alg = A->plan.alg == LAB_SPMV_VECTOR && A->plan.stream && A->plan.st_rows > 0
                   ? LAB_SPMV_VECTOR_STREAM
                   : A->plan.alg;
    if(lanes)
        *lanes = A->plan.lanes;
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
