// Solve phase: fused multigrid cycles, preconditioners, PCG (device-resident
// scalars, one CUDA graph per iteration), stationary AMG and GMRES.
#include "amg.cuh"
#include "spmv_engine.cuh"

#include <cmath>
#include <map>
#include <mutex>
#include <tuple>

namespace lab
{
    lab_status dot_device(int64_t n, const double* x, const double* y, red_buf r, cudaStream_t s);

    // ================================================================ cycle ops
    // Pre-smoothing from a zero guess fused with the residual:
    //   x = omega * D^-1 b          (first Jacobi sweep from x = 0)
    //   r = b - A x                 (x gathered on the fly, never re-read from memory)
    struct op_pre0
    {
        using val_t                   = double;
        using acc_t                   = double;
        static constexpr bool kFma    = true;
        static constexpr bool kReduce = false;
        const double* __restrict__ b;
        const double* __restrict__ invd;
        double omega;
        double* __restrict__ x;
        double* __restrict__ r;
        __device__ __forceinline__ double gather(int c) const
        {
            return omega * (__ldg(invd + c) * __ldg(b + c));
        }
        __device__ __forceinline__ double finish(int i, double s) const
        {
            x[i] = gather(i);
            r[i] = b[i] - s;
            return 0.0;
        }
    };

    // Weighted Jacobi sweep y = x + omega * D^-1 (b - A x); optionally returns
    // y_i * dv_i for a fused dot product.
    template <bool DOT>
    struct op_jacobi
    {
        using val_t                   = double;
        using acc_t                   = double;
        static constexpr bool kFma    = true;
        static constexpr bool kReduce = DOT;
        const double* __restrict__ x;
        const double* __restrict__ b;
        const double* __restrict__ invd;
        double omega;
        double* __restrict__ y;
        const double* __restrict__ dv;
        __device__ __forceinline__ double gather(int c) const
        {
            return __ldg(x + c);
        }
        __device__ __forceinline__ double finish(int i, double s) const
        {
            double yi = x[i] + omega * (invd[i] * (b[i] - s));
            y[i]      = yi;
            return DOT ? yi * dv[i] : 0.0;
        }
    };

    // Residual r = b - A x (fma accumulation; used inside cycles).
    struct op_res_fma
    {
        using val_t                   = double;
        using acc_t                   = double;
        static constexpr bool kFma    = true;
        static constexpr bool kReduce = false;
        const double* __restrict__ x;
        const double* __restrict__ b;
        double* __restrict__ r;
        __device__ __forceinline__ double gather(int c) const
        {
            return __ldg(x + c);
        }
        __device__ __forceinline__ double finish(int i, double s) const
        {
            r[i] = b[i] - s;
            return 0.0;
        }
    };

    // Prolongation and correction y = x + P e; optionally returns y_i * dv_i.
    template <bool DOT>
    struct op_prolong
    {
        using val_t                   = double;
        using acc_t                   = double;
        static constexpr bool kFma    = true;
        static constexpr bool kReduce = DOT;
        const double* __restrict__ e;
        const double* x; // may alias y (in-place correction for GS-type smoothers)
        double*       y;
        const double* __restrict__ dv;
        __device__ __forceinline__ double gather(int c) const
        {
            return __ldg(e + c);
        }
        __device__ __forceinline__ double finish(int i, double s) const
        {
            double yi = x[i] + s;
            y[i]      = yi;
            return DOT ? yi * dv[i] : 0.0;
        }
    };

    // Restriction y = R r.
    struct op_restrict
    {
        using val_t                   = double;
        using acc_t                   = double;
        static constexpr bool kFma    = true;
        static constexpr bool kReduce = false;
        const double* __restrict__ r;
        double* __restrict__ y;
        __device__ __forceinline__ double gather(int c) const
        {
            return __ldg(r + c);
        }
        __device__ __forceinline__ double finish(int i, double s) const
        {
            y[i] = s;
            return 0.0;
        }
    };

    // ================================================================ small kernels
    __global__ void k_zero(double* x, int64_t n, const int* skip)
    {
        if(skip && *skip)
            return;
        for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
            i += (int64_t)gridDim.x * blockDim.x)
            x[i] = 0.0;
    }

    __global__ void k_copy(double* __restrict__ y, const double* __restrict__ x, int64_t n,
                           const int* skip)
    {
        if(skip && *skip)
            return;
        for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
            i += (int64_t)gridDim.x * blockDim.x)
            y[i] = x[i];
    }

    // Coarsest 1x1 level: x = b / a (amg.cpp:211-216).
    __global__ void k_coarse1(const double* a, const double* b, double* x, const int* skip)
    {
        if(skip && *skip)
            return;
        x[0] = __ddiv_rn(b[0], a[0]);
    }

    // Coarse solve through the dense inverse: x = Ainv b (one warp per row).
    __global__ void k_coarse_dense(const double* __restrict__ Ainv, const double* __restrict__ b,
                                   double* __restrict__ x, int n, const int* skip)
    {
        if(skip && *skip)
            return;
        int row  = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
        int lane = threadIdx.x & 31;
        if(row >= n)
            return;
        double s = 0.0;
        for(int k = lane; k < n; k += 32)
            s = fma(Ainv[(size_t)row * n + k], b[k], s);
        s = warp_sum(s);
        if(lane == 0)
            x[row] = s;
    }

    // The reference's coarsest solve: `sweeps` lexicographic Gauss-Seidel sweeps
    // (amg.cpp:238-264, 362-388, 485-511), one thread, same operation order.
    __global__ void k_coarse_gs(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                const double* __restrict__ v, int n, const double* __restrict__ b,
                                double* __restrict__ x, int sweeps, const int* skip)
    {
        if(skip && *skip)
            return;
        if(threadIdx.x != 0 || blockIdx.x != 0)
            return;
        for(int it = 0; it < sweeps; it++)
            for(int j = 0; j < n; j++)
            {
                double sigma = 0.0, ajj = 0.0;
                for(int k = rp[j]; k < rp[j + 1]; k++)
                {
                    int c = ci[k];
                    if(c != j)
                        sigma = __dadd_rn(sigma, __dmul_rn(v[k], x[c]));
                    else
                        ajj = v[k];
                }
                x[j] = __ddiv_rn(__dsub_rn(b[j], sigma), ajj);
            }
    }

    // Dense inverse by Gauss-Jordan with partial pivoting, one CTA (n <= 1024).
    __global__ void __launch_bounds__(1024)
        k_gauss_jordan(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                       const double* __restrict__ v, int n, double* M, double* I, int* singular)
    {
        const int t  = threadIdx.x;
        const int NT = blockDim.x;
        for(size_t k = t; k < (size_t)n * n; k += NT)
        {
            M[k] = 0.0;
            I[k] = 0.0;
        }
        __syncthreads();
        for(int i = t; i < n; i += NT)
        {
            I[(size_t)i * n + i] = 1.0;
            for(int j = rp[i]; j < rp[i + 1]; j++)
                M[(size_t)i * n + ci[j]] += v[j];
        }
        __syncthreads();
        __shared__ int    s_piv;
        __shared__ double s_pv;
        for(int c = 0; c < n; c++)
        {
            if(t == 0)
            {
                int    p  = c;
                double pv = fabs(M[(size_t)c * n + c]);
                for(int r = c + 1; r < n; r++)
                {
                    double a = fabs(M[(size_t)r * n + c]);
                    if(a > pv)
                    {
                        pv = a;
                        p  = r;
                    }
                }
                s_piv = p;
                s_pv  = pv;
            }
            __syncthreads();
            if(s_pv == 0.0)
            {
                if(t == 0)
                    *singular = 1;
                return;
            }
            int p = s_piv;
            if(p != c)
                for(int k = t; k < n; k += NT)
                {
                    double a = M[(size_t)c * n + k];
                    M[(size_t)c * n + k] = M[(size_t)p * n + k];
                    M[(size_t)p * n + k] = a;
                    a                    = I[(size_t)c * n + k];
                    I[(size_t)c * n + k] = I[(size_t)p * n + k];
                    I[(size_t)p * n + k] = a;
                }
            __syncthreads();
            const double inv = 1.0 / M[(size_t)c * n + c];
            __syncthreads();
            for(int k = t; k < n; k += NT)
            {
                M[(size_t)c * n + k] *= inv;
                I[(size_t)c * n + k] *= inv;
            }
            __syncthreads();
            for(size_t q = t; q < (size_t)n * n; q += NT)
            {
                int r = (int)(q / n), k = (int)(q % n);
                if(r == c)
                    continue;
                double f = M[(size_t)r * n + c];
                if(k == c)
                    continue; // column c of M is zeroed after the sweep
                M[q] -= f * M[(size_t)c * n + k];
                I[q] -= f * I[(size_t)c * n + k];
            }
            __syncthreads();
            for(int r = t; r < n; r += NT)
                if(r != c)
                {
                    double f             = M[(size_t)r * n + c];
                    I[(size_t)r * n + c] -= f * I[(size_t)c * n + c];
                    M[(size_t)r * n + c] = 0.0;
                }
            __syncthreads();
        }
    }

    // ---------------------------------------------------------------- multicolour GS
    __device__ __forceinline__ unsigned int colour_hash(unsigned int x)
    {
        x ^= 0x9e3779b9u;
        x = ((x >> 16) ^ x) * 0x45d9f3bu;
        x = ((x >> 16) ^ x) * 0x45d9f3bu;
        return (x >> 16) ^ x;
    }

    // Jones-Plassmann-Luby: an uncoloured row takes colour c when its (hash, index)
    // beats every uncoloured neighbour of the symmetrised pattern.
    __global__ void k_jpl_round(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                int64_t m, int32_t* colour, int c, int* remaining)
    {
        int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
        if(i >= m || colour[i] >= 0)
            return;
        unsigned hi = colour_hash((unsigned)i);
        for(int j = rp[i]; j < rp[i + 1]; j++)
        {
            int k = ci[j];
            if(k == i)
                continue;
            int ck = colour[k];
            if(ck >= 0 && ck != c)
                continue;
            unsigned hk = colour_hash((unsigned)k);
            if(hk > hi || (hk == hi && k > i))
            {
                atomicAdd(remaining, 1);
                return;
            }
        }
        colour[i] = c;
    }

    __global__ void k_colour_count(const int32_t* colour, int64_t m, int32_t* cnt)
    {
        int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
        if(i < m)
            atomicAdd(&cnt[colour[i]], 1);
    }

    __global__ void k_colour_scatter(const int32_t* colour, int64_t m, int32_t* cursor,
                                     int32_t* perm)
    {
        int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
        if(i < m)
            perm[atomicAdd(&cursor[colour[i]], 1)] = (int32_t)i;
    }

    // One colour of a (S)SOR / GS sweep: x_i += omega * (b_i - (A x)_i) / a_ii
    // for the rows of that colour (mutually independent).
    template <int LANES>
    __global__ void k_gs_colour(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                const double* __restrict__ v, const double* __restrict__ invd,
                                const int32_t* __restrict__ rows, int nrows,
                                const double* __restrict__ b, double* x, double omega,
                                const int* skip)
    {
        if(skip && *skip)
            return;
        int64_t t    = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
        int64_t q    = t / LANES;
        int     lane = (int)(t % LANES);
        int     i    = q < nrows ? rows[q] : -1;
        double  s    = 0.0;
        if(i >= 0)
            for(int j = rp[i] + lane; j < rp[i + 1]; j += LANES)
                s = fma(v[j], x[ci[j]], s);
#pragma unroll
        for(int o = LANES / 2; o > 0; o >>= 1)
            s += __shfl_xor_sync(0xffffffffu, s, o, LANES);
        if(i >= 0 && lane == 0)
            x[i] = x[i] + omega * (invd[i] * (b[i] - s));
    }

    // ================================================================ workspace
    struct cyc_ctx
    {
        const lab_amg_options* o;
        cudaStream_t           s;
        const int*             skip; // early exit flag (PCG graph), may be null
    };

    static lab_status build_colouring(lab_csr_impl* A, level_ws& w, cudaStream_t s)
    {
        if(w.colour)
            return LAB_OK;
        const int64_t m = A->m;
        // symmetrised pattern A + A^T
        lab_csr_impl* T = nullptr;
        LAB_TRY(transpose(A, &T, s));
        lab_csr_impl* G = nullptr;
        lab_status st = spgeam(1.0, A, 1.0, T, &G, s);
        csr_release(T);
        LAB_TRY(st);
        dbuf<int32_t> colour, cnt, cursor;
        dbuf<int>     rem;
        st = colour.alloc((size_t)m + 1, s);
        if(st == LAB_OK)
            st = rem.alloc(1, s);
        int ncol = 0;
        if(st == LAB_OK)
        {
            cudaMemsetAsync(colour.get(), 0xff, sizeof(int32_t) * m, s);
            // every round colours at least the highest-priority uncoloured row,
            // so m rounds always suffice
            for(int64_t c = 0; c <= m; c++)
            {
                cudaMemsetAsync(rem.get(), 0, sizeof(int), s);
                k_jpl_round<<<(unsigned)ceil_div<int64_t>(m, 256), 256, 0, s>>>(
                    G->row_ptr, G->col_ind, m, colour.get(), c, rem.get());
                g_launches.fetch_add(1);
                int h = 0;
                st    = copy_d2h_sync(&h, rem.get(), sizeof(int), s);
                if(st != LAB_OK)
                    break;
                ncol = (int)c + 1;
                if(h == 0)
                    break;
            }
        }
        csr_release(G);
        LAB_TRY(st);
        LAB_TRY(cnt.alloc((size_t)ncol + 1, s));
        LAB_TRY(cursor.alloc((size_t)ncol + 1, s));
        LAB_CUDA(cudaMemsetAsync(cnt.get(), 0, sizeof(int32_t) * (ncol + 1), s));
        LAB_LAUNCH(k_colour_count, (unsigned)ceil_div<int64_t>(m, 256), 256, 0, s, colour.get(), m,
                   cnt.get());
        LAB_TRY(counts_to_rowptr(cnt.get(), cursor.get(), ncol, nullptr, s));
        w.colour_ptr_h = new int32_t[ncol + 1];
        LAB_TRY(copy_d2h_sync(w.colour_ptr_h, cursor.get(), sizeof(int32_t) * (ncol + 1), s));
        LAB_TRY(dalloc(&w.colour, (size_t)m + 1, s));
        LAB_LAUNCH(k_colour_scatter, (unsigned)ceil_div<int64_t>(m, 256), 256, 0, s, colour.get(),
                   m, cursor.get(), w.colour);
        w.ncolours = ncol;
        return LAB_OK;
    }

    static lab_status build_coarse(hierarchy_impl* h, int coarse_mode, cudaStream_t s)
    {
        lab_csr_impl* A = h->A[h->levels];
        const int     n = (int)A->m;
        if(n <= 1 || coarse_mode != LAB_COARSE_DIRECT || h->coarse_inv || h->coarse_singular)
            return LAB_OK;
        if(n > 1024)
        {
            h->coarse_singular = 2; // too large for the dense path: GS sweeps are used
            return LAB_OK;
        }
        dbuf<double> M;
        dbuf<int>    sing;
        LAB_TRY(M.alloc((size_t)n * n, s));
        LAB_TRY(sing.alloc(1, s));
        LAB_TRY(dalloc(&h->coarse_inv, (size_t)n * n, s));
        LAB_CUDA(cudaMemsetAsync(sing.get(), 0, sizeof(int), s));
        LAB_LAUNCH(k_gauss_jordan, 1, 1024, 0, s, A->row_ptr, A->col_ind, A->val, n, M.get(),
                   h->coarse_inv, sing.get());
        int hs = 0;
        LAB_TRY(copy_d2h_sync(&hs, sing.get(), sizeof(int), s));
        if(hs)
        {
            h->coarse_singular = 1;
            dfree(h->coarse_inv, s);
            h->coarse_inv = nullptr;
        }
        h->coarse_n = n;
        return LAB_OK;
    }

    // Allocate every per-level vector and analyse every operator once, so the
    // cycle itself never allocates or synchronises (it is captured in graphs).
    static lab_status prepare(hierarchy_impl* h, const lab_amg_options* o, cudaStream_t s)
    {
        const int L = h->levels;
        for(int l = 0; l <= L; l++)
        {
            lab_csr_impl* A = h->A[l];
            level_ws&     w = h->ws[l];
            LAB_TRY(spmv_analyse(A, s));
            LAB_TRY(csr_ensure_invdiag(A, s));
            if(l < L)
            {
                LAB_TRY(spmv_analyse(h->P[l], s));
                LAB_TRY(spmv_analyse(h->R[l], s));
            }
            if(!w.x)
            {
                size_t m = (size_t)A->m + 1;
                LAB_TRY(dalloc(&w.x, m, s));
                LAB_TRY(dalloc(&w.b, m, s));
                LAB_TRY(dalloc(&w.r, m, s));
                LAB_TRY(dalloc(&w.t, m, s));
            }
            if(o->smoother != LAB_SMOOTH_JACOBI && l < L)
                LAB_TRY(build_colouring(A, w, s));
        }
        LAB_TRY(build_coarse(h, o->coarse, s));
        h->ws_ready = 1;
        return LAB_OK;
    }

    static inline unsigned grid_for(int64_t n)
    {
        return (unsigned)std::max<int64_t>(1, std::min<int64_t>(ceil_div<int64_t>(n, 256),
                                                                (int64_t)num_sms() * 8));
    }

    // ---------------------------------------------------------------- smoothing sweeps
    // One smoothing sweep reading xin, producing the new iterate in xout (Jacobi
    // needs two buffers; GS-type sweeps update xin in place and return it).
    static lab_status smooth(const lab_csr_impl* A, level_ws& w, const double* b, double* xin,
                             double* xout, double** result, const cyc_ctx& c, bool reverse,
                             red_buf dot = red_buf(), const double* dv = nullptr)
    {
        const lab_amg_options* o = c.o;
        red_buf                rb;
        rb.skip = c.skip;
        if(o->smoother != LAB_SMOOTH_JACOBI && !w.colour_ptr_h)
        {
            set_error("multicolour smoother without a colouring of level of size %lld",
                      (long long)A->m);
            return LAB_BAD_ARG;
        }
        if(o->smoother == LAB_SMOOTH_JACOBI)
        {
            if(dv)
            {
                dot.skip = c.skip;
                op_jacobi<true> op{xin, b, A->invdiag, o->omega, xout, dv};
                LAB_TRY(launch_rowop(A, A->val, op, c.s, dot));
            }
            else
            {
                op_jacobi<false> op{xin, b, A->invdiag, o->omega, xout, nullptr};
                LAB_TRY(launch_rowop(A, A->val, op, c.s, rb));
            }
            *result = xout;
            return LAB_OK;
        }
        // GS family.  The reference maps SGS to plain GS (amg.cpp:130-132) and uses
        // omega 0.5 for SOR / SSOR (amg.cpp:133-137); SSOR sweeps forward then back.
        const double omega = (o->smoother == LAB_SMOOTH_SOR || o->smoother == LAB_SMOOTH_SSOR)
                                 ? o->omega_sor
                                 : 1.0;
        const bool   sym   = o->smoother == LAB_SMOOTH_SSOR;
        const int    lanes = A->plan.alg == LAB_SPMV_ROWSEQ ? 1 : std::min(A->plan.lanes, 32);
        auto         pass  = [&](int col) -> lab_status {
            int r0 = w.colour_ptr_h[col], r1 = w.colour_ptr_h[col + 1];
            int nr = r1 - r0;
            if(nr == 0)
                return LAB_OK;
            unsigned g = (unsigned)ceil_div<int64_t>((int64_t)nr * lanes, 256);
            switch(lanes)
            {
            case 1:
                LAB_LAUNCH(k_gs_colour<1>, g, 256, 0, c.s, A->row_ptr, A->col_ind, A->val,
                           A->invdiag, w.colour + r0, nr, b, xin, omega, c.skip);
                break;
            case 2:
                LAB_LAUNCH(k_gs_colour<2>, g, 256, 0, c.s, A->row_ptr, A->col_ind, A->val,
                           A->invdiag, w.colour + r0, nr, b, xin, omega, c.skip);
                break;
            case 4:
                LAB_LAUNCH(k_gs_colour<4>, g, 256, 0, c.s, A->row_ptr, A->col_ind, A->val,
                           A->invdiag, w.colour + r0, nr, b, xin, omega, c.skip);
                break;
            case 8:
                LAB_LAUNCH(k_gs_colour<8>, g, 256, 0, c.s, A->row_ptr, A->col_ind, A->val,
                           A->invdiag, w.colour + r0, nr, b, xin, omega, c.skip);
                break;
            case 16:
                LAB_LAUNCH(k_gs_colour<16>, g, 256, 0, c.s, A->row_ptr, A->col_ind, A->val,
                           A->invdiag, w.colour + r0, nr, b, xin, omega, c.skip);
                break;
            default:
                LAB_LAUNCH(k_gs_colour<32>, g, 256, 0, c.s, A->row_ptr, A->col_ind, A->val,
                           A->invdiag, w.colour + r0, nr, b, xin, omega, c.skip);
                break;
            }
            return LAB_OK;
        };
        if(!reverse)
            for(int col = 0; col < w.ncolours; col++)
                LAB_TRY(pass(col));
        else
            for(int col = w.ncolours - 1; col >= 0; col--)
                LAB_TRY(pass(col));
        if(sym)
        {
            if(!reverse)
                for(int col = w.ncolours - 1; col >= 0; col--)
                    LAB_TRY(pass(col));
            else
                for(int col = 0; col < w.ncolours; col++)
                    LAB_TRY(pass(col));
        }
        *result = xin;
        if(dv)
        {
            // fused dot unavailable for in-place sweeps: separate reduction
            dot.skip = c.skip;
            LAB_TRY(dot_device(A->m, xin, dv, dot, c.s));
        }
        return LAB_OK;
    }

    // ---------------------------------------------------------------- coarse solve
    static lab_status coarse_solve(hierarchy_impl* h, const double* b, double* x, bool zero_guess,
                                   int sweeps, const cyc_ctx& c)
    {
        lab_csr_impl* A = h->A[h->levels];
        const int     n = (int)A->m;
        if(n == 0)
            return LAB_OK;
        if(n == 1)
        {
            LAB_LAUNCH(k_coarse1, 1, 1, 0, c.s, (const double*)A->val, b, x, c.skip);
            return LAB_OK;
        }
        if(c.o->coarse == LAB_COARSE_DIRECT && h->coarse_inv)
        {
            unsigned g = (unsigned)ceil_div(n, 8);
            LAB_LAUNCH(k_coarse_dense, g, 256, 0, c.s, (const double*)h->coarse_inv, b, x, n,
                       c.skip);
            return LAB_OK;
        }
        if(zero_guess)
            LAB_LAUNCH(k_zero, grid_for(n), 256, 0, c.s, x, (int64_t)n, c.skip);
        LAB_LAUNCH(k_coarse_gs, 1, 1, 0, c.s, A->row_ptr, A->col_ind, A->val, n, b, x, sweeps,
                   c.skip);
        return LAB_OK;
    }

    // ---------------------------------------------------------------- cycles
    // cycle(l): x <- cycle(x; b) on level l.  kind 0 = V (amg.cpp:144-267),
    // 1 = W (269-390), 2 = F (392-513).  zero_guess: x enters as 0 (not read).
    // When `dv` is given (level 0 of a PCG preconditioner), the kernel writing the
    // final x also accumulates dot(x, dv) into dot.out.
    static lab_status cycle(hierarchy_impl* h, int l, int kind, double* x, const double* b,
                            bool zero_guess, const cyc_ctx& c, red_buf dot = red_buf(),
                            const double* dv = nullptr)
    {
        const lab_amg_options* o = c.o;
        red_buf                rb;
        rb.skip = c.skip;
        if(l == h->levels)
        {
            LAB_TRY(coarse_solve(h, b, x, zero_guess, kind == 0 ? 1000 : 100, c));
            if(dv)
            {
                dot.skip = c.skip;
                LAB_TRY(dot_device(h->A[l]->m, x, dv, dot, c.s));
            }
            return LAB_OK;
        }
        lab_csr_impl* A  = h->A[l];
        lab_csr_impl* P  = h->P[l];
        lab_csr_impl* R  = h->R[l];
        level_ws&     w  = h->ws[l];
        level_ws&     wc = h->ws[l + 1];
        const int64_t m  = A->m;
        const int     n1 = o->n1, n2 = o->n2;
        const bool    jac = o->smoother == LAB_SMOOTH_JACOBI;

        // Buffers: the level iterate alternates between x and w.t for Jacobi.
        double* cur = x;
        double* oth = w.t;
        auto    flip = [&](double* res) {
            if(res != cur)
            {
                oth = cur;
                cur = res;
            }
        };

        // ---- pre-smoothing + residual
        // Jacobi alternates between x and w.t; start in the buffer that makes the
        // last write land in x (GS-type sweeps and the prolongation work in place).
        const int visits = kind == 0 ? 1 : 2;
        if(jac)
        {
            int flips = (zero_guess && n1 >= 1) ? (n1 - 1) + visits * (1 + n2)
                                                : n1 + visits * (1 + n2);
            if(zero_guess && (flips & 1))
            {
                cur = w.t;
                oth = x;
            }
        }
        if(zero_guess && n1 >= 1 && jac)
        {
            op_pre0 op{b, A->invdiag, o->omega, cur, w.r};
            LAB_TRY(launch_rowop(A, A->val, op, c.s, rb));
            for(int k = 1; k < n1; k++)
            {
                double* res = nullptr;
                LAB_TRY(smooth(A, w, b, cur, oth, &res, c, false));
                flip(res);
            }
            if(n1 > 1)
            {
                op_res_fma op2{cur, b, w.r};
                LAB_TRY(launch_rowop(A, A->val, op2, c.s, rb));
            }
        }
        else
        {
            if(zero_guess)
                LAB_LAUNCH(k_zero, grid_for(m), 256, 0, c.s, cur, m, c.skip);
            for(int k = 0; k < n1; k++)
            {
                double* res = nullptr;
                LAB_TRY(smooth(A, w, b, cur, oth, &res, c, false));
                flip(res);
            }
            op_res_fma op2{cur, b, w.r};
            LAB_TRY(launch_rowop(A, A->val, op2, c.s, rb));
        }

        // ---- restrict, recurse, correct
        auto coarse_correct = [&](bool cz, int ckind, bool last) -> lab_status {
            op_restrict opr{w.r, wc.b};
            LAB_TRY(launch_rowop(R, R->val, opr, c.s, rb));
            LAB_TRY(cycle(h, l + 1, ckind, wc.x, wc.b, cz, c));
            bool    fuse = last && dv && n2 == 0 && kind == 0;
            double* dst  = jac ? oth : cur;
            if(fuse)
            {
                dot.skip = c.skip;
                op_prolong<true> opp{wc.x, cur, dst, dv};
                LAB_TRY(launch_rowop(P, P->val, opp, c.s, dot));
            }
            else
            {
                op_prolong<false> opp{wc.x, cur, dst, nullptr};
                LAB_TRY(launch_rowop(P, P->val, opp, c.s, rb));
            }
            flip(dst);
            return LAB_OK;
        };

        auto post = [&](int sweeps, bool last) -> lab_status {
            for(int k = 0; k < sweeps; k++)
            {
                double* res      = nullptr;
                bool    fuse_dot = last && dv && k == sweeps - 1;
                LAB_TRY(smooth(A, w, b, cur, oth, &res, c, false, fuse_dot ? dot : red_buf(),
                               fuse_dot ? dv : nullptr));
                flip(res);
            }
            return LAB_OK;
        };

        if(kind == 0)
        {
            LAB_TRY(coarse_correct(true, 0, true));
            LAB_TRY(post(n2, true));
        }
        else
        {
            // W: second visit recurses with W again; F: with V (amg.cpp:463).
            // The second coarse solve starts from the first one's result.
            LAB_TRY(coarse_correct(true, kind, false));
            LAB_TRY(post(n2, false));
            op_res_fma op2{cur, b, w.r};
            LAB_TRY(launch_rowop(A, A->val, op2, c.s, rb));
            LAB_TRY(coarse_correct(false, kind == 1 ? 1 : 0, false));
            LAB_TRY(post(n2, true)); // n3 = n2 (amg.cpp:537)
            if(dv && n2 == 0)
            {
                dot.skip = c.skip;
                LAB_TRY(dot_device(m, cur, dv, dot, c.s));
            }
        }
        if(cur != x)
            LAB_LAUNCH(k_copy, grid_for(m), 256, 0, c.s, x, (const double*)cur, m, c.skip);
        return LAB_OK;
    }

    // ================================================================ reductions on device
    template <int OP>
    __global__ void __launch_bounds__(256)
        k_red_dev(int64_t n, const double* __restrict__ x, const double* __restrict__ y,
                  double* partial, unsigned int* counter, double* out, const int* skip)
    {
        if(skip && *skip)
            return;
        double acc = 0.0;
        for(int64_t i = blockIdx.x * 256ll + threadIdx.x; i < n; i += (int64_t)gridDim.x * 256)
            acc = OP == 0 ? acc + x[i] * y[i] : nanmax(acc, fabs(x[i]));
        if(OP == 0)
            reduce_finish_sum<256>(acc, partial, counter, out);
        else
            reduce_finish_max<256>(acc, partial, counter, out);
    }

    static unsigned red_grid(int64_t n)
    {
        return (unsigned)std::max<int64_t>(1, std::min<int64_t>(kRedBlocks, ceil_div<int64_t>(n, 256)));
    }

    lab_status dot_device(int64_t n, const double* x, const double* y, red_buf r, cudaStream_t s)
    {
        LAB_LAUNCH(k_red_dev<0>, red_grid(n), 256, 0, s, n, x, y, r.partial, r.counter, r.out,
                   r.skip);
        return LAB_OK;
    }

    static lab_status norm_inf_device(int64_t n, const double* x, red_buf r, cudaStream_t s)
    {
        LAB_LAUNCH(k_red_dev<1>, red_grid(n), 256, 0, s, n, x, (const double*)nullptr, r.partial,
                   r.counter, r.out, r.skip);
        return LAB_OK;
    }

    // ================================================================ preconditioners
    struct precond_impl
    {
        uint64_t         uid  = next_uid();
        int              kind = 0; // 0 = AMG, 1 = Jacobi
        hierarchy_impl*  h    = nullptr;
        lab_amg_options  o;
        lab_csr_impl*    A    = nullptr; // Jacobi
        double*          diag = nullptr; // Jacobi: the reference divides by the diagonal
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
        if(M->kind == 1)
        {
            int64_t n = M->A->m;
            LAB_LAUNCH(k_jacobi_dot, red_grid(n), 256, 0, s, n, r, (const double*)M->diag, z,
                       dot.partial, dot.counter, dot.out, skip);
            return LAB_OK;
        }
        cyc_ctx c{&M->o, s, skip};
        if(dot.out)
            return cycle(M->h, 0, M->o.cycle, z, r, true, c, dot, r);
        return cycle(M->h, 0, M->o.cycle, z, r, true, c);
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
        S_COUNT = 8
    };
    enum
    {
        F_DONE   = 0,
        F_ITER   = 1,
        F_STATUS = 2,
        F_CONV   = 3,
        F_MAXIT  = 4,
        F_COUNT  = 8
    };

    struct pcg_ws
    {
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
        cudaGraphExec_t graph = nullptr;
        uint64_t      key_M   = 0;
        const double* key_x   = nullptr;
        uint64_t      key_A   = 0;
        cudaStream_t  key_s   = nullptr;
        ~pcg_ws()
        {
            if(graph)
                cudaGraphExecDestroy(graph);
            void* dp[] = {r, z, p, q, sc, flags, partial, counters};
            for(void* x : dp)
                if(x)
                    cudaFree(x);
            if(hflags)
                cudaFreeHost(hflags);
            for(auto& e : ev)
                if(e)
                    cudaEventDestroy(e);
            if(cap)
                cudaStreamDestroy(cap);
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
    __global__ void __launch_bounds__(256)
        k_pcg_pupdate(int64_t n, double* __restrict__ p, const double* __restrict__ z, double* sc,
                      int* flags, unsigned int* counter)
    {
        if(flags[F_DONE])
            return;
        const double beta = sc[S_GNEW] / sc[S_GAMMA];
        for(int64_t i = blockIdx.x * 256ll + threadIdx.x; i < n; i += (int64_t)gridDim.x * 256)
            p[i] = beta == 0.0 ? z[i] : __dadd_rn(z[i], __dmul_rn(beta, p[i]));
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
        LAB_CUDA(cudaMallocHost(&w->hflags, sizeof(int) * F_COUNT * 2));
        LAB_CUDA(cudaEventCreateWithFlags(&w->ev[0], cudaEventDisableTiming));
        LAB_CUDA(cudaEventCreateWithFlags(&w->ev[1], cudaEventDisableTiming));
        LAB_CUDA(cudaStreamCreateWithFlags(&w->cap, cudaStreamNonBlocking));
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
        LAB_TRY(precond_apply(M, w->r, w->z, s, skip, rbuf(w, 2, w->sc + S_GNEW, skip)));
        LAB_LAUNCH(k_pcg_pupdate, red_grid(A->m), 256, 0, s, A->m, w->p, (const double*)w->z,
                   w->sc, w->flags, w->counters + 3);
        return LAB_OK;
    }

    static lab_status pcg_solve(lab_csr_impl* A, precond_impl* M, const double* b, double* x,
                                const lab_iter_control* ctl, lab_solve_info* info, cudaStream_t s)
    {
        LAB_TRY(spmv_analyse(A, s));
        if(M && M->kind == 0)
            LAB_TRY(prepare(M->h, &M->o, s));
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

        // iteration graph (rebuilt when the operands change)
        if(!w->graph || w->key_M != M->uid || w->key_x != x || w->key_A != A->uid)
        {
            if(w->graph)
                cudaGraphExecDestroy(w->graph);
            w->graph = nullptr;
            cudaGraph_t g = nullptr;
            LAB_CUDA(cudaStreamBeginCapture(w->cap, cudaStreamCaptureModeThreadLocal));
            lab_status  st = pcg_iteration(A, M, x, w, w->cap);
            cudaError_t ce = cudaStreamEndCapture(w->cap, &g);
            if(st != LAB_OK && g)
                cudaGraphDestroy(g);
            LAB_TRY(st);
            LAB_CUDA(ce);
            ce = cudaGraphInstantiate(&w->graph, g, 0);
            cudaGraphDestroy(g);
            LAB_CUDA(ce);
            w->key_M = M->uid;
            w->key_x = x;
            w->key_A = A->uid;
            w->key_s = s;
        }
        // Pipelined host loop: iteration k+1 is queued before the flags of
        // iteration k are inspected; a queued iteration after convergence is a
        // no-op because every kernel checks flags[F_DONE] first.
        const int max_launch = ctl->max_iter + 1;
        int       launched   = 0;
        for(; launched < max_launch; launched++)
        {
            LAB_CUDA(cudaGraphLaunch(w->graph, s));
            int slot = launched & 1;
            LAB_CUDA(cudaMemcpyAsync(w->hflags + slot * F_COUNT, w->flags, sizeof(int) * F_COUNT,
                                     cudaMemcpyDeviceToHost, s));
            LAB_CUDA(cudaEventRecord(w->ev[slot], s));
            if(launched >= 1)
            {
                int prev = (launched - 1) & 1;
                LAB_CUDA(cudaEventSynchronize(w->ev[prev]));
                if(w->hflags[prev * F_COUNT + F_DONE])
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

    // Unpreconditioned CG as the reference runs it (cg.cpp:60-134): with
    // restart_iter = -1, `iter % restart_iter == 0` holds for every iter > 0, so
    // each iteration restarts from the true residual (steepest descent).
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
                LAB_LAUNCH(k_copy, grid_for(A->m), 256, 0, s, w->p, (const double*)w->r, A->m,
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
            LAB_LAUNCH(k_pcg_pupdate, red_grid(A->m), 256, 0, s, A->m, w->p, (const double*)w->r,
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
        LAB_TRY(prepare(h, o, s));
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
            LAB_TRY(cycle(h, 0, o->cycle, x, b, false, c));
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
            LAB_TRY(prepare(M->h, &M->o, s));
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
                    op_restrict ops{qkm1, w.get()};
                    LAB_TRY(launch_rowop(A, A->val, ops, s));
                    LAB_TRY(precond_apply(M, w.get(), qk, s, nullptr, red_buf()));
                }
                else
                {
                    op_restrict ops{qkm1, qk};
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
    LAB_TRY(prepare(h, o, s));
    cyc_ctx c{o, s, nullptr};
    return cycle(h, 0, o->cycle, x, b, false, c);
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
    lab_status st = prepare(h, o, to_stream(s));
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
    M->diag = A->diag;
    *out    = M;
    return LAB_OK;
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
    return pcg_solve(A, M, b, x, c, info, to_stream(s));
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
    lab_status st = M ? pcg_solve(A, M, b.get(), x.get(), c, info, s)
                      : cg_plain(A, b.get(), x.get(), c, info, s);
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
    return gmres_solve(A, M, restart, b, x, c, info, to_stream(s));
}

} // extern "C"
