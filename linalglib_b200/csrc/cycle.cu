// Multigrid cycles on the device: fused smoother / residual / restriction /
// prolongation kernels, multicolour Gauss-Seidel, coarsest-level solves, and
// the V / W / F recursion (amg.cpp:144-513), in FP64 or in reduced precision
// (FP32 arithmetic over FP32 or BF16 stored values) for the mixed-precision
// preconditioner.
#include "cycle.cuh"

#include <cuda_bf16.h>
#include <type_traits>

namespace lab
{
    // ================================================================ ops
    // Pre-smoothing from a zero guess fused with the residual:
    //   x = omega D^-1 b   (first Jacobi sweep from x = 0)
    //   r = b - A x        (x recomputed from b and D^-1 at every gather)
    template <class VT, class T>
    struct op_pre0
    {
        using val_t                   = VT;
        using acc_t                   = T;
        static constexpr bool kFma    = true;
        static constexpr bool kReduce = false;
        const T* __restrict__ b;
        const T* __restrict__ invd;
        T omega;
        T* __restrict__ x;
        T* __restrict__ r;
        __device__ __forceinline__ T gather(int c) const
        {
            return omega * (__ldg(invd + c) * __ldg(b + c));
        }
        __device__ __forceinline__ double finish(int i, T s) const
        {
            x[i] = gather(i);
            r[i] = b[i] - s;
            return 0.0;
        }
        struct pre_t
        {
            T b, invd;
        };
        __device__ __forceinline__ pre_t pre(int i) const
        {
            return {__ldg(b + i), __ldg(invd + i)};
        }
        __device__ __forceinline__ double finish(int i, T s, const pre_t& p) const
        {
            x[i] = omega * (p.invd * p.b);
            r[i] = p.b - s;
            return 0.0;
        }
    };

    // Weighted Jacobi sweep y = x + omega D^-1 (b - A x); with DOT returns y_i dv_i.
    template <class VT, class T, bool DOT>
    struct op_jacobi
    {
        using val_t                   = VT;
        using acc_t                   = T;
        static constexpr bool kFma    = true;
        static constexpr bool kReduce = DOT;
        const T* __restrict__ x;
        const T* __restrict__ b;
        const T* __restrict__ invd;
        T omega;
        T* __restrict__ y;
        const T* __restrict__ dv;
        __device__ __forceinline__ T gather(int c) const
        {
            return __ldg(x + c);
        }
        __device__ __forceinline__ double finish(int i, T s) const
        {
            T yi = x[i] + omega * (invd[i] * (b[i] - s));
            y[i] = yi;
            return DOT ? (double)yi * (double)dv[i] : 0.0;
        }
        struct pre_t
        {
            T x, b, invd, dv;
        };
        __device__ __forceinline__ pre_t pre(int i) const
        {
            return {__ldg(x + i), __ldg(b + i), __ldg(invd + i), DOT ? __ldg(dv + i) : T(0)};
        }
        __device__ __forceinline__ double finish(int i, T s, const pre_t& p) const
        {
            T yi = p.x + omega * (p.invd * (p.b - s));
            y[i] = yi;
            return DOT ? (double)yi * (double)p.dv : 0.0;
        }
    };

    template <class VT, class T>
    struct op_res
    {
        using val_t                   = VT;
        using acc_t                   = T;
        static constexpr bool kFma    = true;
        static constexpr bool kReduce = false;
        const T* __restrict__ x;
        const T* __restrict__ b;
        T* __restrict__ r;
        __device__ __forceinline__ T gather(int c) const
        {
            return __ldg(x + c);
        }
        __device__ __forceinline__ double finish(int i, T s) const
        {
            r[i] = b[i] - s;
            return 0.0;
        }
        using pre_t = T; // b_i
        __device__ __forceinline__ T pre(int i) const
        {
            return __ldg(b + i);
        }
        __device__ __forceinline__ double finish(int i, T s, T bi) const
        {
            r[i] = bi - s;
            return 0.0;
        }
    };

    // y = x + P e (x may alias y: in-place correction for GS-type smoothers)
    template <class VT, class T, bool DOT>
    struct op_prolong
    {
        using val_t                   = VT;
        using acc_t                   = T;
        static constexpr bool kFma    = true;
        static constexpr bool kReduce = DOT;
        const T* __restrict__ e;
        const T* x;
        T*       y;
        const T* __restrict__ dv;
        __device__ __forceinline__ T gather(int c) const
        {
            return __ldg(e + c);
        }
        __device__ __forceinline__ double finish(int i, T s) const
        {
            T yi = x[i] + s;
            y[i] = yi;
            return DOT ? (double)yi * (double)dv[i] : 0.0;
        }
        // (x may alias y, but only row i itself writes y_i, after this load)
        struct pre_t
        {
            T x, dv;
        };
        __device__ __forceinline__ pre_t pre(int i) const
        {
            return {x[i], DOT ? __ldg(dv + i) : T(0)};
        }
        __device__ __forceinline__ double finish(int i, T s, const pre_t& p) const
        {
            T yi = p.x + s;
            y[i] = yi;
            return DOT ? (double)yi * (double)p.dv : 0.0;
        }
    };

    // y = R r; with x0 set, also x0 = omega D_c^-1 y: the coarse level's first
    // Jacobi sweep from zero, the value op_pre0 would compute there, so the coarse
    // pre-smoothing pass gathers one vector instead of two.
    template <class VT, class T>
    struct op_restrict
    {
        using val_t                   = VT;
        using acc_t                   = T;
        static constexpr bool kFma    = true;
        static constexpr bool kReduce = false;
        const T* __restrict__ r;
        T* __restrict__ y;
        const T* __restrict__ invd_c = nullptr;
        T omega                      = T(0);
        T* __restrict__ x0           = nullptr;
        __device__ __forceinline__ T gather(int c) const
        {
            return __ldg(r + c);
        }
        __device__ __forceinline__ double finish(int i, T s) const
        {
            y[i] = s;
            if(x0)
                x0[i] = omega * (__ldg(invd_c + i) * s);
            return 0.0;
        }
        using pre_t = T; // D_c^-1 of row i (when x0 is written)
        __device__ __forceinline__ T pre(int i) const
        {
            return x0 ? __ldg(invd_c + i) : T(0);
        }
        __device__ __forceinline__ double finish(int i, T s, T di) const
        {
            y[i] = s;
            if(x0)
                x0[i] = omega * (di * s);
            return 0.0;
        }
    };

    // ================================================================ small kernels
    template <class T>
    __global__ void k_zero(T* x, int64_t n, const int* skip)
    {
        if(skip && *skip)
            return;
        for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
            i += (int64_t)gridDim.x * blockDim.x)
            x[i] = T(0);
    }

    template <class T>
    __global__ void k_copy(T* __restrict__ y, const T* __restrict__ x, int64_t n, const int* skip)
    {
        if(skip && *skip)
            return;
        for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
            i += (int64_t)gridDim.x * blockDim.x)
            y[i] = x[i];
    }

    __global__ void k_copy_d(double* __restrict__ y, const double* __restrict__ x, int64_t n,
                             const int* skip)
    {
        if(skip && *skip)
            return;
        for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
            i += (int64_t)gridDim.x * blockDim.x)
            y[i] = x[i];
    }

    __global__ void k_d2f(const double* __restrict__ x, float* __restrict__ y, int64_t n,
                          const int* skip)
    {
        if(skip && *skip)
            return;
        for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
            i += (int64_t)gridDim.x * blockDim.x)
            y[i] = (float)x[i];
    }

    // k_d2f that also writes x0 = omega D^-1 b (FP32): the level-0 pre-smoothing
    // pass then gathers x0 once per entry instead of recomputing it from b and
    // D^-1 at every gather (the same FP32 products op_pre0 forms, so the cycle's
    // result is unchanged; the reduced-precision passes are issue-bound).
    __global__ void k_d2f_x0(const double* __restrict__ r, float* __restrict__ b,
                             const float* __restrict__ invd, float omega, float* __restrict__ x0,
                             int64_t n, const int* skip)
    {
        if(skip && *skip)
            return;
        for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
            i += (int64_t)gridDim.x * blockDim.x)
        {
            const float bi = (float)r[i];
            b[i]           = bi;
            x0[i]          = omega * (invd[i] * bi);
        }
    }

    // z = (double) x with (z, r) accumulated for the PCG beta.
    __global__ void __launch_bounds__(256)
        k_f2d_dot(const float* __restrict__ x, const double* __restrict__ r, double* __restrict__ z,
                  int64_t n, double* partial, unsigned int* counter, double* out, const int* skip)
    {
        if(skip && *skip)
            return;
        double acc = 0.0;
        for(int64_t i = blockIdx.x * 256ll + threadIdx.x; i < n; i += (int64_t)gridDim.x * 256)
        {
            double zi = (double)x[i];
            z[i]      = zi;
            acc += zi * r[i];
        }
        if(out)
            reduce_finish_sum<256>(acc, partial, counter, out);
    }

    // (z, r) and (z, q) with z = (double) x, each summed as k_f2d_dot and
    // k_red_dev<0> sum theirs (the flexible-PCG step of the reduced-precision
    // preconditioner; z itself is never written).
    __global__ void __launch_bounds__(256)
        k_f2d_dot2(const float* __restrict__ x, const double* __restrict__ r,
                   const double* __restrict__ q, int64_t n, red_buf zr, red_buf zq)
    {
        if(zr.skip && *zr.skip)
            return;
        double a1 = 0.0, a2 = 0.0;
        for(int64_t i = blockIdx.x * 256ll + threadIdx.x; i < n; i += (int64_t)gridDim.x * 256)
        {
            double zi = (double)x[i];
            a1 += zi * r[i];
            a2 = a2 + zi * q[i];
        }
        reduce_finish_sum<256>(a1, zr.partial, zr.counter, zr.out);
        reduce_finish_sum<256>(a2, zq.partial, zq.counter, zq.out);
    }

    // x += (double) e
    __global__ void k_add_f2d(const float* __restrict__ e, double* __restrict__ x, int64_t n)
    {
        for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
            i += (int64_t)gridDim.x * blockDim.x)
            x[i] += (double)e[i];
    }

    // Coarsest 1x1 level: x = b / a (amg.cpp:211-216).
    template <class T>
    __global__ void k_coarse1(const double* a, const T* b, T* x, const int* skip)
    {
        if(skip && *skip)
            return;
        x[0] = (T)__ddiv_rn((double)b[0], a[0]);
    }

    // x = Ainv b with the FP64 dense inverse (one warp per row, FP64 accumulation).
    template <class T>
    __global__ void k_coarse_dense(const double* __restrict__ Ainv, const T* __restrict__ b,
                                   T* __restrict__ x, int n, const int* skip)
    {
        if(skip && *skip)
            return;
        int row  = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
        int lane = threadIdx.x & 31;
        if(row >= n)
            return;
        double s = 0.0;
        for(int k = lane; k < n; k += 32)
            s = fma(Ainv[(size_t)row * n + k], (double)b[k], s);
        s = warp_sum(s);
        if(lane == 0)
            x[row] = (T)s;
    }

    // The reference's coarsest solve: `sweeps` lexicographic Gauss-Seidel sweeps
    // (amg.cpp:238-264, 362-388, 485-511), one thread, same operation order.
    template <class T>
    __global__ void k_coarse_gs(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                const double* __restrict__ v, int n, const T* __restrict__ b,
                                T* __restrict__ x, int sweeps, const int* skip)
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
                        sigma = __dadd_rn(sigma, __dmul_rn(v[k], (double)x[c]));
                    else
                        ajj = v[k];
                }
                x[j] = (T)__ddiv_rn(__dsub_rn((double)b[j], sigma), ajj);
            }
    }

    // Dense inverse of the coarsest operator by Gauss-Jordan with partial pivoting
    // (n <= kCoarseDenseMax), the whole GPU per pivot column: k_gj_pivot (one CTA)
    // picks the pivot -- the first row of the largest |M[r][c]|, r >= c, as a
    // sequential scan with a strict comparison picks it (a NaN never wins; a NaN on
    // the diagonal is kept) -- swaps, scales the pivot row and saves column c;
    // k_gj_elim then subtracts f_r x (pivot row) from every other row of M and I
    // with f_r from the saved column.  Columns of M left of c are exact zeros in
    // rows c and p and never reach I, so their updates are skipped; every entry of
    // I gets the same operations in the same order as a one-CTA sweep.
    constexpr int kCoarseDenseMax = 4096;

    __global__ void k_gj_init(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                              const double* __restrict__ v, int n, double* M, double* I)
    {
        const size_t nn = (size_t)n * n;
        for(size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < nn;
            k += (size_t)gridDim.x * blockDim.x)
        {
            M[k] = 0.0;
            I[k] = (k / n == k % n) ? 1.0 : 0.0;
        }
    }

    __global__ void k_gj_scatter(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                 const double* __restrict__ v, int n, double* M)
    {
        const int i = blockIdx.x * blockDim.x + threadIdx.x;
        if(i < n)
            for(int j = rp[i]; j < rp[i + 1]; j++)
                M[(size_t)i * n + ci[j]] += v[j];
    }

    // Pivot step of column c by one CTA (1024 threads): pivot choice, row swap,
    // scaling of the pivot row, column c saved to fcol.  Returns false (uniformly)
    // when the column has no nonzero pivot (*singular set).
    __device__ bool gj_pivot_step(double* M, double* I, int n, int c, double* fcol,
                                  int* singular)
    {
        __shared__ double s_v[32];
        __shared__ int    s_r[32];
        __shared__ int    s_piv;
        __shared__ double s_pv;
        const int         t = threadIdx.x, lane = t & 31, wid = t >> 5;
        double            bv = -1.0; // below every |x|; NaN never replaces it
        int               br = n;
        for(int r = c + t; r < n; r += blockDim.x)
        {
            const double a = fabs(M[(size_t)r * n + c]);
            if(a > bv)
            {
                bv = a;
                br = r;
            }
        }
        // largest value, lowest row among equal values
#pragma unroll
        for(int o = 16; o > 0; o >>= 1)
        {
            const double ov  = __shfl_xor_sync(0xffffffffu, bv, o);
            const int    orw = __shfl_xor_sync(0xffffffffu, br, o);
            if(ov > bv || (ov == bv && orw < br))
            {
                bv = ov;
                br = orw;
            }
        }
        if(lane == 0)
        {
            s_v[wid] = bv;
            s_r[wid] = br;
        }
        __syncthreads();
        if(t == 0)
        {
            for(int w = 1; w < (int)(blockDim.x >> 5); w++)
                if(s_v[w] > bv || (s_v[w] == bv && s_r[w] < br))
                {
                    bv = s_v[w];
                    br = s_r[w];
                }
            const double ac = fabs(M[(size_t)c * n + c]);
            s_piv = isnan(ac) ? c : br;
            s_pv  = isnan(ac) ? ac : bv;
            if(s_pv == 0.0)
                *singular = 1;
        }
        __syncthreads();
        if(s_pv == 0.0)
            return false;
        const int p = s_piv;
        if(p != c)
        {
            for(int k = c + t; k < n; k += blockDim.x)
            {
                const double a       = M[(size_t)c * n + k];
                M[(size_t)c * n + k] = M[(size_t)p * n + k];
                M[(size_t)p * n + k] = a;
            }
            for(int k = t; k < n; k += blockDim.x)
            {
                const double a       = I[(size_t)c * n + k];
                I[(size_t)c * n + k] = I[(size_t)p * n + k];
                I[(size_t)p * n + k] = a;
            }
        }
        __syncthreads();
        const double inv = 1.0 / M[(size_t)c * n + c];
        __syncthreads();
        for(int k = c + t; k < n; k += blockDim.x)
            M[(size_t)c * n + k] *= inv;
        for(int k = t; k < n; k += blockDim.x)
            I[(size_t)c * n + k] *= inv;
        for(int r = t; r < n; r += blockDim.x)
            if(r != c) // row c is being scaled; the elimination skips it
                fcol[r] = M[(size_t)r * n + c];
        return true;
    }

    // Entry (r, k), r != c, of the elimination of column c (f = the saved M[r][c]).
    __device__ __forceinline__ void gj_elim_entry(double* M, double* I, int n, int c, int r,
                                                  int k, double f)
    {
        if(k == c)
        {
            I[(size_t)r * n + c] -= f * I[(size_t)c * n + c];
            M[(size_t)r * n + c] = 0.0;
            return;
        }
        if(k > c)
            M[(size_t)r * n + k] -= f * M[(size_t)c * n + k];
        I[(size_t)r * n + k] -= f * I[(size_t)c * n + k];
    }

    __global__ void __launch_bounds__(1024)
        k_gj_pivot(double* M, double* I, int n, int c, double* fcol, int* singular)
    {
        if(*singular)
            return;
        gj_pivot_step(M, I, n, c, fcol, singular);
    }

    // grid (ceil(n / 256), n): row blockIdx.y, columns blockIdx.x * 256 + threadIdx.x
    __global__ void __launch_bounds__(256)
        k_gj_elim(double* M, double* I, int n, int c, const double* __restrict__ fcol,
                  const int* singular)
    {
        const int r = blockIdx.y;
        const int k = blockIdx.x * 256 + threadIdx.x;
        if(*singular || r == c || k >= n)
            return;
        gj_elim_entry(M, I, n, c, r, k, fcol[r]);
    }

    // The same steps in one CTA for small coarsest levels (n <= kCoarseDenseOneCta),
    // where a pair of launches per column would cost more than the work.
    constexpr int kCoarseDenseOneCta = 256;
    __global__ void __launch_bounds__(1024)
        k_gj_small(double* M, double* I, int n, double* fcol, int* singular)
    {
        for(int c = 0; c < n; c++)
        {
            if(!gj_pivot_step(M, I, n, c, fcol, singular))
                return;
            __syncthreads();
            for(int q = threadIdx.x; q < n * n; q += blockDim.x)
            {
                const int r = q / n, k = q % n;
                if(r != c)
                    gj_elim_entry(M, I, n, c, r, k, fcol[r]);
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
    // beats every uncoloured neighbour in the symmetrised pattern.
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

    // One colour of a GS / SOR sweep: x_i += omega (b_i - (A x)_i) / a_ii for the
    // rows of that colour (mutually independent, so updated in place).
    template <int LANES, class VT, class T>
    __global__ void k_gs_colour(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                const VT* __restrict__ v, const T* __restrict__ invd,
                                const int32_t* __restrict__ rows, int nrows,
                                const T* __restrict__ b, T* x, T omega, const int* skip)
    {
        if(skip && *skip)
            return;
        int64_t t    = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
        int64_t q    = t / LANES;
        int     lane = (int)(t % LANES);
        int     i    = q < nrows ? rows[q] : -1;
        T       s    = T(0);
        if(i >= 0)
            for(int j = rp[i] + lane; j < rp[i + 1]; j += LANES)
                s = acc_step<true>(to_acc(v[j], T(0)), x[ci[j]], s);
#pragma unroll
        for(int o = LANES / 2; o > 0; o >>= 1)
            s += __shfl_xor_sync(0xffffffffu, s, o, LANES);
        if(i >= 0 && lane == 0)
            x[i] = x[i] + omega * (invd[i] * (b[i] - s));
    }

    // ================================================================ precision plumbing
    __global__ void k_vals_f32(const double* __restrict__ v, int64_t n, float* __restrict__ f)
    {
        for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
            i += (int64_t)gridDim.x * blockDim.x)
            f[i] = (float)v[i];
    }

    __global__ void k_vals_bf16(const double* __restrict__ v, int64_t n,
                                __nv_bfloat16* __restrict__ f)
    {
        for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
            i += (int64_t)gridDim.x * blockDim.x)
            f[i] = __double2bfloat16(v[i]);
    }

    // FP32 (or BF16) value copies of a matrix and its FP32 inverse diagonal.
    // 1 in *wide when some column offset col - row leaves the int16 range.
    __global__ void k_dcol_check(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                 int64_t m, int* wide)
    {
        for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m;
            i += (int64_t)gridDim.x * blockDim.x)
            for(int j = rp[i]; j < rp[i + 1]; j++)
            {
                const int64_t d = (int64_t)ci[j] - i;
                if(d < INT16_MIN || d > INT16_MAX)
                {
                    atomicOr(wide, 1);
                    break;
                }
            }
    }

    __global__ void k_dcol_fill(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                int64_t m, int16_t* __restrict__ dcol)
    {
        for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m;
            i += (int64_t)gridDim.x * blockDim.x)
            for(int j = rp[i]; j < rp[i + 1]; j++)
                dcol[j] = (int16_t)(ci[j] - (int)i);
    }

    lab_status csr_ensure_lowp(lab_csr_impl* A, int precision, int use_bf16, cudaStream_t s)
    {
        if(precision == LAB_PREC_FP64)
            return LAB_OK;
        const int64_t nz = std::max<int64_t>(A->nnz, 1);
        unsigned      g  = grid_for(A->nnz);
        if(use_bf16 && !A->lp.bf16)
        {
            LAB_TRY(dalloc(&A->lp.bf16, (size_t)nz, s));
            if(A->nnz)
                LAB_LAUNCH(k_vals_bf16, g, 256, 0, s, (const double*)A->val, A->nnz, A->lp.bf16);
        }
        if(!use_bf16 && !A->lp.f32)
        {
            LAB_TRY(dalloc(&A->lp.f32, (size_t)nz, s));
            if(A->nnz)
                LAB_LAUNCH(k_vals_f32, g, 256, 0, s, (const double*)A->val, A->nnz, A->lp.f32);
        }
        if(A->lp.dcol_state == 0 && A->m > 0 && A->nnz > 0)
        {
            // compact 16-bit column offsets when every |col - row| fits
            dbuf<int> wide;
            LAB_TRY(wide.alloc(1, s));
            LAB_CUDA(cudaMemsetAsync(wide.get(), 0, sizeof(int), s));
            LAB_LAUNCH(k_dcol_check, grid_for(A->m), 256, 0, s, A->row_ptr, A->col_ind, A->m,
                       wide.get());
            int h = 1;
            LAB_TRY(copy_d2h_sync(&h, wide.get(), sizeof(int), s));
            if(h)
                A->lp.dcol_state = -1;
            else
            {
                LAB_TRY(dalloc(&A->lp.dcol, (size_t)A->nnz, s));
                LAB_LAUNCH(k_dcol_fill, grid_for(A->m), 256, 0, s, A->row_ptr, A->col_ind, A->m,
                           A->lp.dcol);
                A->lp.dcol_state = 1;
            }
        }
        if(A->m == A->n && !A->lp.invd32)
        {
            LAB_TRY(csr_ensure_invdiag(A, s));
            LAB_TRY(dalloc(&A->lp.invd32, (size_t)A->m + 1, s));
            if(A->m)
                LAB_LAUNCH(k_vals_f32, grid_for(A->m), 256, 0, s, (const double*)A->invdiag, A->m,
                           A->lp.invd32);
        }
        return LAB_OK;
    }

    unsigned grid_for(int64_t n)
    {
        return (unsigned)std::max<int64_t>(1, std::min<int64_t>(ceil_div<int64_t>(n, 256),
                                                                (int64_t)num_sms() * 8));
    }

    unsigned red_grid(int64_t n)
    {
        return (unsigned)std::max<int64_t>(1, std::min<int64_t>(kRedBlocks, ceil_div<int64_t>(n, 256)));
    }

    // Per-precision views of a level's vectors and operator data.
    template <class T>
    struct lv;
    template <>
    struct lv<double>
    {
        static double* x(level_ws& w) { return w.x; }
        static double* b(level_ws& w) { return w.b; }
        static double* r(level_ws& w) { return w.r; }
        static double* t(level_ws& w) { return w.t; }
        static const double* invd(const lab_csr_impl* A) { return A->invdiag; }
    };
    template <>
    struct lv<float>
    {
        static float* x(level_ws& w) { return w.xf; }
        static float* b(level_ws& w) { return w.bf; }
        static float* r(level_ws& w) { return w.rf; }
        static float* t(level_ws& w) { return w.tf; }
        static const float* invd(const lab_csr_impl* A) { return A->lp.invd32; }
    };

    // BF16 value storage on the two finest levels (LAB_PREC_FP32_BF16).
    static inline bool level_bf16(const lab_amg_options* o, int l)
    {
        return o->precision == LAB_PREC_FP32_BF16 && l < 2;
    }

    // Call f(values) with the value array the cycle of precision T reads.
    template <class T, class F>
    static lab_status with_vals(const lab_csr_impl* M, bool bf16, F&& f)
    {
        if constexpr(std::is_same<T, double>::value)
            return f(static_cast<const double*>(M->val));
        else
        {
            if(bf16)
                return f(static_cast<const __nv_bfloat16*>(M->lp.bf16));
            return f(static_cast<const float*>(M->lp.f32));
        }
    }

    template <class P>
    using vt_of = typename std::remove_const<typename std::remove_pointer<P>::type>::type;

    // ================================================================ setup of the cycle
    static lab_status build_colouring(lab_csr_impl* A, level_ws& w, cudaStream_t s)
    {
        if(w.colour)
            return LAB_OK;
        const int64_t m = A->m;
        lab_csr_impl* T = nullptr;
        LAB_TRY(transpose(A, &T, s));
        lab_csr_impl* G  = nullptr;
        lab_status    st = spgeam(1.0, A, 1.0, T, &G, s); // symmetrised pattern A + A^T
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
            // every round colours at least the highest-priority uncoloured row
            for(int64_t c = 0; c <= m; c++)
            {
                cudaMemsetAsync(rem.get(), 0, sizeof(int), s);
                k_jpl_round<<<(unsigned)ceil_div<int64_t>(m, 256), 256, 0, s>>>(
                    G->row_ptr, G->col_ind, m, colour.get(), (int)c, rem.get());
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
        if(n > kCoarseDenseMax)
        {
            h->coarse_singular = 2; // too large for the dense path: GS sweeps are used
            return LAB_OK;
        }
        dbuf<double> M, fcol;
        dbuf<int>    sing;
        LAB_TRY(M.alloc((size_t)n * n, s));
        LAB_TRY(fcol.alloc((size_t)n, s));
        LAB_TRY(sing.alloc(1, s));
        LAB_TRY(dalloc(&h->coarse_inv, (size_t)n * n, s));
        LAB_CUDA(cudaMemsetAsync(sing.get(), 0, sizeof(int), s));
        const unsigned ginit = (unsigned)std::min<int64_t>(
            ceil_div<int64_t>((int64_t)n * n, 256), (int64_t)num_sms() * 8);
        LAB_LAUNCH(k_gj_init, ginit, 256, 0, s, A->row_ptr, A->col_ind, A->val, n, M.get(),
                   h->coarse_inv);
        LAB_LAUNCH(k_gj_scatter, (unsigned)ceil_div(n, 256), 256, 0, s, A->row_ptr, A->col_ind,
                   A->val, n, M.get());
        if(n <= kCoarseDenseOneCta)
            LAB_LAUNCH(k_gj_small, 1, 1024, 0, s, M.get(), h->coarse_inv, n, fcol.get(),
                       sing.get());
        else
        {
            const dim3 gel((unsigned)ceil_div(n, 256), (unsigned)n);
            for(int c = 0; c < n; c++)
            {
                LAB_LAUNCH(k_gj_pivot, 1, 1024, 0, s, M.get(), h->coarse_inv, n, c,
                           fcol.get(), sing.get());
                LAB_LAUNCH(k_gj_elim, gel, 256, 0, s, M.get(), h->coarse_inv, n, c,
                           (const double*)fcol.get(), (const int*)sing.get());
            }
        }
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

    lab_status cycle_prepare(hierarchy_impl* h, const lab_amg_options* o, cudaStream_t s)
    {
        const int  L     = h->levels;
        const bool lowp  = o->precision != LAB_PREC_FP64;
        {
            // the SpMV plans of every operator, prolongation and restriction with one
            // host round trip (the per-level calls below then find them analysed)
            std::vector<lab_csr_impl*> all;
            for(int l = 0; l <= L; l++)
            {
                all.push_back(h->A[l]);
                if(l < L)
                {
                    all.push_back(h->P[l]);
                    all.push_back(h->R[l]);
                }
            }
            LAB_TRY(spmv_analyse_batch(all.data(), (int)all.size(), s));
        }
        for(int l = 0; l <= L; l++)
        {
            lab_csr_impl* A = h->A[l];
            level_ws&     w = h->ws[l];
            const size_t  m = (size_t)A->m + 1;
            LAB_TRY(spmv_analyse(A, s));
            LAB_TRY(csr_ensure_invdiag(A, s));
            if(l < L)
            {
                LAB_TRY(spmv_analyse(h->P[l], s));
                LAB_TRY(spmv_analyse(h->R[l], s));
            }
            if(!w.x)
            {
                LAB_TRY(dalloc(&w.x, m, s));
                LAB_TRY(dalloc(&w.b, m, s));
                LAB_TRY(dalloc(&w.r, m, s));
                LAB_TRY(dalloc(&w.t, m, s));
            }
            if(lowp)
            {
                const bool bf = level_bf16(o, l);
                LAB_TRY(csr_ensure_lowp(A, o->precision, bf, s));
                if(l < L)
                {
                    LAB_TRY(csr_ensure_lowp(h->P[l], o->precision, bf, s));
                    LAB_TRY(csr_ensure_lowp(h->R[l], o->precision, bf, s));
                }
                if(!w.xf)
                {
                    LAB_TRY(dalloc(&w.xf, m, s));
                    LAB_TRY(dalloc(&w.bf, m, s));
                    LAB_TRY(dalloc(&w.rf, m, s));
                    LAB_TRY(dalloc(&w.tf, m, s));
                }
            }
            if(o->smoother != LAB_SMOOTH_JACOBI && l < L)
                LAB_TRY(build_colouring(A, w, s));
        }
        LAB_TRY(build_coarse(h, o->coarse, s));
        h->ws_ready = 1;
        return LAB_OK;
    }

    // ================================================================ reductions
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

    lab_status dot_device(int64_t n, const double* x, const double* y, red_buf r, cudaStream_t s)
    {
        LAB_LAUNCH(k_red_dev<0>, red_grid(n), 256, 0, s, n, x, y, r.partial, r.counter, r.out,
                   r.skip);
        return LAB_OK;
    }

    lab_status norm_inf_device(int64_t n, const double* x, red_buf r, cudaStream_t s)
    {
        LAB_LAUNCH(k_red_dev<1>, red_grid(n), 256, 0, s, n, x, (const double*)nullptr, r.partial,
                   r.counter, r.out, r.skip);
        return LAB_OK;
    }

    // ================================================================ smoothing
    // One sweep reading xin; the new iterate is written to xout (Jacobi) or
    // xin in place (GS family); *result tells which.
    template <class T>
    static lab_status smooth(const lab_csr_impl* A, int l, level_ws& w, const T* b, T* xin, T* xout,
                             T** result, const cyc_ctx& c, red_buf dot = red_buf(),
                             const T* dv = nullptr)
    {
        const lab_amg_options* o = c.o;
        red_buf                rb;
        rb.skip       = c.skip;
        dot.skip      = c.skip;
        const T* invd = lv<T>::invd(A);
        const bool bf = level_bf16(o, l);
        if(o->smoother == LAB_SMOOTH_JACOBI)
        {
            *result = xout;
            return with_vals<T>(A, bf, [&](auto* vals) -> lab_status {
                using VT = vt_of<decltype(vals)>;
                if(dv)
                {
                    op_jacobi<VT, T, true> op{xin, b, invd, (T)o->omega, xout, dv};
                    return launch_rowop(A, vals, op, c.s, dot);
                }
                op_jacobi<VT, T, false> op{xin, b, invd, (T)o->omega, xout, nullptr};
                return launch_rowop(A, vals, op, c.s, rb);
            });
        }
        if(!w.colour_ptr_h)
        {
            set_error("multicolour smoother without a colouring of level %d", l);
            return LAB_BAD_ARG;
        }
        // GS family.  The reference maps SGS to plain GS (amg.cpp:130-132) and uses
        // omega 0.5 for SOR / SSOR (amg.cpp:133-137); SSOR sweeps forward then back.
        const T    omega = (o->smoother == LAB_SMOOTH_SOR || o->smoother == LAB_SMOOTH_SSOR)
                               ? (T)o->omega_sor
                               : T(1);
        const bool sym   = o->smoother == LAB_SMOOTH_SSOR;
        const int  lanes = A->plan.alg == LAB_SPMV_VECTOR ? std::min(A->plan.lanes, 32)
                           : (A->plan.max_row <= 32 ? 1 : A->plan.vlanes);
        auto pass = [&](int col) -> lab_status {
            return with_vals<T>(A, bf, [&](auto* vals) -> lab_status {
                using VT = vt_of<decltype(vals)>;
                int r0 = w.colour_ptr_h[col], r1 = w.colour_ptr_h[col + 1];
                int nr = r1 - r0;
                if(nr == 0)
                    return LAB_OK;
                unsigned g = (unsigned)ceil_div<int64_t>((int64_t)nr * lanes, 256);
#define LAB_GS(LN)                                                                              \
    LAB_LAUNCH((k_gs_colour<LN, VT, T>), g, 256, 0, c.s, A->row_ptr, A->col_ind, vals, invd,    \
               (const int32_t*)(w.colour + r0), nr, b, xin, omega, c.skip)
                switch(lanes)
                {
                case 1:
                    LAB_GS(1);
                    break;
                case 2:
                    LAB_GS(2);
                    break;
                case 4:
                    LAB_GS(4);
                    break;
                case 8:
                    LAB_GS(8);
                    break;
                case 16:
                    LAB_GS(16);
                    break;
                default:
                    LAB_GS(32);
                    break;
                }
#undef LAB_GS
                return LAB_OK;
            });
        };
        for(int col = 0; col < w.ncolours; col++)
            LAB_TRY(pass(col));
        if(sym)
            for(int col = w.ncolours - 1; col >= 0; col--)
                LAB_TRY(pass(col));
        *result = xin;
        if(dv)
        {
            if constexpr(std::is_same<T, double>::value)
                LAB_TRY(dot_device(A->m, xin, dv, dot, c.s));
        }
        return LAB_OK;
    }

    // ================================================================ coarsest level
    template <class T>
    static lab_status coarse_solve(hierarchy_impl* h, const T* b, T* x, bool zero_guess,
                                   int sweeps, const cyc_ctx& c)
    {
        lab_csr_impl* A = h->A[h->levels];
        const int     n = (int)A->m;
        if(n == 0)
            return LAB_OK;
        if(n == 1)
        {
            LAB_LAUNCH(k_coarse1<T>, 1, 1, 0, c.s, (const double*)A->val, b, x, c.skip);
            return LAB_OK;
        }
        if(c.o->coarse == LAB_COARSE_DIRECT && h->coarse_inv)
        {
            unsigned g = (unsigned)ceil_div(n, 8);
            LAB_LAUNCH(k_coarse_dense<T>, g, 256, 0, c.s, (const double*)h->coarse_inv, b, x, n,
                       c.skip);
            return LAB_OK;
        }
        if(zero_guess)
            LAB_LAUNCH(k_zero<T>, grid_for(n), 256, 0, c.s, x, (int64_t)n, c.skip);
        LAB_LAUNCH(k_coarse_gs<T>, 1, 1, 0, c.s, A->row_ptr, A->col_ind, A->val, n, b, x, sweeps,
                   c.skip);
        return LAB_OK;
    }

    // ================================================================ fused tail
    // The last levels of a V-cycle with Jacobi smoothing from a zero guess hold a
    // few hundred rows each, so their passes (restriction, residual, smoothing,
    // prolongation, the coarsest solve) cost launch and round-trip latency, not
    // bandwidth.  One CTA runs them all, from the restriction out of the entry
    // level p to the prolongation back into it, passes separated by block
    // barriers.  Each row is summed in its operator's schedule order (CSR order
    // for the one-thread-per-row plan, k_vector's lane order and xor tree for W
    // lanes), with the ops' own epilogue arithmetic, so the result equals the
    // per-pass launches bit for bit.  Vectors written inside the kernel are read
    // with plain (coherent) loads.
    constexpr int kTailMax = 8;
    constexpr int kTailNT  = 1024;

    struct tail_mat
    {
        const int32_t* rp;
        const int32_t* ci;
        const int16_t* dc; // col - row (reduced precision), or null
        const void*    v;
        int            m;
        int            W; // 1: CSR order; else lanes per row
    };
    struct tail_lvl
    {
        tail_mat    A, R, P; // R, P: to / from the next level
        const void* invd;
        void *      x, *t, *b, *r;
    };
    struct tail_args
    {
        tail_mat      Rp, Pp;
        const void*   wr;  // level-p residual
        const void*   cur; // level-p iterate
        void*         dst; // level-p corrected iterate
        tail_lvl      lv[kTailMax];
        int           nl; // levels p+1 .. L; lv[nl - 1] is the coarsest
        int           n1, n2;
        double        omega;
        const double* a11;  // coarsest 1x1: its value
        const double* ainv; // coarsest n x n: dense inverse
        int           nc;
        const int*    skip;
    };

    template <class T>
    __device__ __forceinline__ T tail_row(const tail_mat& M, int row, int lane, const T* x,
                                          bool valid)
    {
        T s = T(0);
        if(valid)
        {
            const int a = __ldg(M.rp + row), b = __ldg(M.rp + row + 1);
            const T*  v = static_cast<const T*>(M.v);
            if(M.W == 1)
            {
                for(int j = a; j < b; j++)
                {
                    const int c = M.dc ? col_of<int16_t>(__ldg(M.dc + j), row) : __ldg(M.ci + j);
                    s           = acc_step<true>(__ldg(v + j), x[c], s);
                }
            }
            else if constexpr(sizeof(T) == 8)
            {
                for(int j = a + lane; j < b; j += M.W)
                    s = acc_step<true>(__ldg(v + j), x[__ldg(M.ci + j)], s);
            }
            else
            {
                for(int q = (a & ~3) + 4 * lane; q < b; q += 4 * M.W)
                {
                    T   v4[4];
                    int c4[4];
                    ld4(v + q, v4);
                    if(M.dc)
                    {
                        int16_t d4[4];
                        ld4(M.dc + q, d4);
#pragma unroll
                        for(int t = 0; t < 4; t++)
                            c4[t] = col_of<int16_t>(d4[t], row);
                    }
                    else
                        ld4(M.ci + q, c4);
                    T xg[4];
#pragma unroll
                    for(int t = 0; t < 4; t++)
                        if(q + t >= a && q + t < b)
                            xg[t] = x[c4[t]];
#pragma unroll
                    for(int t = 0; t < 4; t++)
                        if(q + t >= a && q + t < b)
                            s = acc_step<true>(v4[t], xg[t], s);
                }
            }
        }
        if(M.W > 1)
            for(int o = M.W / 2; o > 0; o >>= 1)
                s += __shfl_xor_sync(0xffffffffu, s, o, M.W);
        return s;
    }

    // One pass of M over x: fin(row, s) for every row, then a block barrier.
    template <class T, class F>
    __device__ __forceinline__ void tail_pass(const tail_mat& M, const T* x, F&& fin)
    {
        const int W = M.W, per = kTailNT / W;
        for(int base = 0; base < M.m; base += per) // same trip count in every thread
        {
            const int  row   = base + (int)threadIdx.x / W;
            const int  lane  = (int)threadIdx.x & (W - 1);
            const bool valid = row < M.m;
            const T    sum   = tail_row<T>(M, row, lane, x, valid);
            if(valid && lane == 0)
                fin(row, sum);
        }
        __syncthreads();
    }

    template <class T>
    __global__ void __launch_bounds__(kTailNT) k_tail(tail_args a)
    {
        if(a.skip && *a.skip)
            return;
        const T om = (T)a.omega;
        T*      cur[kTailMax];
        T*      oth[kTailMax];
        // weighted Jacobi sweep y = x + omega D^-1 (b - A x) (op_jacobi)
        auto jacobi = [&](const tail_lvl& L, const T* x, T* y) {
            const T* invd = static_cast<const T*>(L.invd);
            const T* b    = static_cast<const T*>(L.b);
            tail_pass<T>(L.A, x, [&](int i, T s) {
                T yi = x[i] + om * (__ldg(invd + i) * (b[i] - s));
                y[i] = yi;
            });
        };
        // b_{k} = R r; x_{k} = omega D_k^-1 b_{k} when level k is not the coarsest
        // (op_restrict with the fused first sweep)
        auto restrict_into = [&](const tail_mat& R, const T* r, int k) {
            const tail_lvl& C    = a.lv[k];
            T*              b    = static_cast<T*>(C.b);
            T*              x0   = k < a.nl - 1 ? static_cast<T*>(C.x) : nullptr;
            const T*        invd = static_cast<const T*>(C.invd);
            tail_pass<T>(R, r, [&](int i, T s) {
                b[i] = s;
                if(x0)
                    x0[i] = om * (__ldg(invd + i) * s);
            });
        };

        restrict_into(a.Rp, static_cast<const T*>(a.wr), 0);
        for(int k = 0; k < a.nl - 1; k++)
        {
            const tail_lvl& L = a.lv[k];
            cur[k]            = static_cast<T*>(L.x);
            oth[k]            = static_cast<T*>(L.t);
            for(int it = 1; it < a.n1; it++)
            {
                jacobi(L, cur[k], oth[k]);
                T* tmp = cur[k];
                cur[k] = oth[k];
                oth[k] = tmp;
            }
            {
                const T* b = static_cast<const T*>(L.b);
                T*       r = static_cast<T*>(L.r);
                tail_pass<T>(L.A, cur[k], [&](int i, T s) { r[i] = b[i] - s; });
            }
            restrict_into(L.R, static_cast<const T*>(L.r), k + 1);
        }
        {
            // coarsest level: x = b / a (1x1) or x = Ainv b (k_coarse1, k_coarse_dense)
            const tail_lvl& C = a.lv[a.nl - 1];
            const T*        b = static_cast<const T*>(C.b);
            T*              x = static_cast<T*>(C.x);
            if(a.nc == 1)
            {
                if(threadIdx.x == 0)
                    x[0] = (T)__ddiv_rn((double)b[0], a.a11[0]);
            }
            else
            {
                const int lane = threadIdx.x & 31;
                for(int row = threadIdx.x >> 5; row < a.nc; row += kTailNT / 32)
                {
                    double s = 0.0;
                    for(int k = lane; k < a.nc; k += 32)
                        s = fma(__ldg(a.ainv + (size_t)row * a.nc + k), (double)b[k], s);
                    s = warp_sum(s);
                    if(lane == 0)
                        x[row] = (T)s;
                }
            }
            __syncthreads();
            cur[a.nl - 1] = x;
        }
        for(int k = a.nl - 2; k >= 0; k--)
        {
            const tail_lvl& L = a.lv[k];
            {
                // x <- x + P e (op_prolong), into the other buffer
                const T* x = cur[k];
                T*       y = oth[k];
                tail_pass<T>(L.P, cur[k + 1], [&](int i, T s) {
                    T yi = x[i] + s;
                    y[i] = yi;
                });
                oth[k] = cur[k];
                cur[k] = y;
            }
            for(int it = 0; it < a.n2; it++)
            {
                jacobi(L, cur[k], oth[k]);
                T* tmp = cur[k];
                cur[k] = oth[k];
                oth[k] = tmp;
            }
        }
        {
            const T* x = static_cast<const T*>(a.cur);
            T*       y = static_cast<T*>(a.dst);
            tail_pass<T>(a.Pp, cur[0], [&](int i, T s) {
                T yi = x[i] + s;
                y[i] = yi;
            });
        }
    }

    template <class T>
    static tail_mat tail_mat_of(const lab_csr_impl* M)
    {
        tail_mat t;
        t.rp = M->row_ptr;
        t.ci = M->col_ind;
        t.m  = (int)M->m;
        // the W of launch_rowop's VECTOR dispatch (2, 4, 8, 16, else 32)
        const int ln = M->plan.lanes;
        t.W = M->plan.alg != LAB_SPMV_VECTOR ? 1 : (ln == 2 || ln == 4 || ln == 8 || ln == 16) ? ln : 32;
        if constexpr(std::is_same<T, double>::value)
        {
            t.dc = nullptr;
            t.v  = M->val;
        }
        else
        {
            t.dc = M->lp.dcol;
            t.v  = M->lp.f32;
        }
        return t;
    }

    // Levels l+1 .. L form a fused tail when the cycle is a V-cycle with Jacobi
    // smoothing (n1 >= 1) from a zero guess, level l's operators are not BF16,
    // every operator below l is small (A: <= 1024 rows; A, R, P: <= 16384 entries,
    // <= 4096 rows) and the coarsest level is solved by a 1x1 division or the
    // dense inverse.
    static bool tail_ok(const hierarchy_impl* h, const lab_amg_options* o, int l)
    {
        const int L = h->levels;
        if(o->cycle != LAB_CYCLE_V || o->smoother != LAB_SMOOTH_JACOBI || o->n1 < 1 || l < 1 ||
           l >= L || L - l > kTailMax || level_bf16(o, l))
            return false;
        auto small = [](const lab_csr_impl* M, int64_t rows) {
            return M && M->m <= rows && M->nnz <= 16384 && M->plan.analysed;
        };
        for(int k = l; k < L; k++)
            if(!small(h->R[k], 4096) || !small(h->P[k], 4096) || !small(h->A[k + 1], 1024))
                return false;
        const int64_t nc = h->A[L]->m;
        return nc == 1 || (nc > 1 && o->coarse == LAB_COARSE_DIRECT && h->coarse_inv);
    }

    template <class T>
    static lab_status tail_launch(hierarchy_impl* h, int l, const T* wr, const T* cur, T* dst,
                                  const cyc_ctx& c)
    {
        const lab_amg_options* o = c.o;
        tail_args              a{};
        a.Rp  = tail_mat_of<T>(h->R[l]);
        a.Pp  = tail_mat_of<T>(h->P[l]);
        a.wr  = wr;
        a.cur = cur;
        a.dst = dst;
        a.nl  = h->levels - l;
        for(int k = 0; k < a.nl; k++)
        {
            const int  lk = l + 1 + k;
            tail_lvl&  t  = a.lv[k];
            level_ws&  w  = h->ws[lk];
            t.A           = tail_mat_of<T>(h->A[lk]);
            if(lk < h->levels)
            {
                t.R = tail_mat_of<T>(h->R[lk]);
                t.P = tail_mat_of<T>(h->P[lk]);
            }
            t.invd = lv<T>::invd(h->A[lk]);
            t.x    = lv<T>::x(w);
            t.t    = lv<T>::t(w);
            t.b    = lv<T>::b(w);
            t.r    = lv<T>::r(w);
        }
        a.n1    = o->n1;
        a.n2    = o->n2;
        a.omega = o->omega;
        a.nc    = (int)h->A[h->levels]->m;
        a.a11   = (const double*)h->A[h->levels]->val;
        a.ainv  = (const double*)h->coarse_inv;
        a.skip  = c.skip;
        LAB_LAUNCH(k_tail<T>, 1, kTailNT, 0, c.s, a);
        return LAB_OK;
    }

    // ================================================================ the recursion
    // cycle(l): x <- cycle(x; b) on level l.  kind 0 = V (amg.cpp:144-267),
    // 1 = W (269-390), 2 = F (392-513).  zero_guess: x enters as 0 (not read).
    // With `dv` (level 0 of the FP64 preconditioner) the kernel writing the final
    // x also accumulates (x, dv) into dot.out.
    // The buffer a zero-guess Jacobi cycle on level l starts in: x, or the level's
    // scratch vector when the number of Jacobi writes is odd, so the last write
    // lands in x.
    template <class T>
    static T* cycle_start(hierarchy_impl* h, int l, int kind, T* x, const lab_amg_options* o)
    {
        const int visits = kind == 0 ? 1 : 2;
        const int flips  = (o->n1 >= 1) ? (o->n1 - 1) + visits * (1 + o->n2)
                                        : o->n1 + visits * (1 + o->n2);
        return (flips & 1) ? lv<T>::t(h->ws[l]) : x;
    }

    // x0_ready: the caller's restriction already wrote omega D^-1 b into the
    // buffer cycle_start() names (zero guess, Jacobi, n1 >= 1 only).
    template <class T>
    static lab_status cycle(hierarchy_impl* h, int l, int kind, T* x, const T* b, bool zero_guess,
                            const cyc_ctx& c, red_buf dot = red_buf(), const T* dv = nullptr,
                            bool x0_ready = false)
    {
        const lab_amg_options* o = c.o;
        red_buf                rb;
        rb.skip  = c.skip;
        dot.skip = c.skip;
        if(l == h->levels)
        {
            LAB_TRY(coarse_solve<T>(h, b, x, zero_guess, kind == 0 ? 1000 : 100, c));
            if constexpr(std::is_same<T, double>::value)
                if(dv)
                    LAB_TRY(dot_device(h->A[l]->m, x, dv, dot, c.s));
            return LAB_OK;
        }
        lab_csr_impl* A   = h->A[l];
        lab_csr_impl* P   = h->P[l];
        lab_csr_impl* R   = h->R[l];
        level_ws&     w   = h->ws[l];
        level_ws&     wc  = h->ws[l + 1];
        const int64_t m   = A->m;
        const int     n1  = o->n1, n2 = o->n2;
        const bool    jac = o->smoother == LAB_SMOOTH_JACOBI;
        const bool    bf  = level_bf16(o, l);
        T*            wr  = lv<T>::r(w);
        T*            cx  = lv<T>::x(wc);
        T*            cb  = lv<T>::b(wc);
        const T*      invd = lv<T>::invd(A);

        // Jacobi alternates between x and the level's scratch vector; start in the
        // buffer that makes the last write land in x (GS sweeps and the correction
        // work in place).
        T*        cur    = x;
        T*        oth    = lv<T>::t(w);
        const int visits = kind == 0 ? 1 : 2;
        if(jac)
        {
            int flips = (zero_guess && n1 >= 1) ? (n1 - 1) + visits * (1 + n2)
                                                : n1 + visits * (1 + n2);
            if(zero_guess && (flips & 1))
            {
                cur = lv<T>::t(w);
                oth = x;
            }
        }
        auto flip = [&](T* res) {
            if(res != cur)
            {
                oth = cur;
                cur = res;
            }
        };
        auto residual = [&]() -> lab_status {
            return with_vals<T>(A, bf, [&](auto* vals) -> lab_status {
                op_res<vt_of<decltype(vals)>, T> op{cur, b, wr};
                return launch_rowop(A, vals, op, c.s, rb);
            });
        };

        // ---- pre-smoothing + residual
        if(zero_guess && n1 >= 1 && jac)
        {
            if(x0_ready)
                LAB_TRY(residual()); // cur = omega D^-1 b already
            else
                LAB_TRY(with_vals<T>(A, bf, [&](auto* vals) -> lab_status {
                    op_pre0<vt_of<decltype(vals)>, T> op{b, invd, (T)o->omega, cur, wr};
                    return launch_rowop(A, vals, op, c.s, rb);
                }));
            for(int k = 1; k < n1; k++)
            {
                T* res = nullptr;
                LAB_TRY(smooth<T>(A, l, w, b, cur, oth, &res, c));
                flip(res);
            }
            if(n1 > 1)
                LAB_TRY(residual());
        }
        else
        {
            if(zero_guess)
                LAB_LAUNCH(k_zero<T>, grid_for(m), 256, 0, c.s, cur, m, c.skip);
            for(int k = 0; k < n1; k++)
            {
                T* res = nullptr;
                LAB_TRY(smooth<T>(A, l, w, b, cur, oth, &res, c));
                flip(res);
            }
            LAB_TRY(residual());
        }

        // ---- restrict, recurse, correct
        auto coarse_correct = [&](bool cz, int ckind, bool last) -> lab_status {
            if(cz && kind == 0 && ckind == 0 && !(last && dv) && tail_ok(h, o, l))
            {
                // restriction, levels l+1 .. L and the prolongation in one launch
                T* dst = jac ? oth : cur;
                LAB_TRY(tail_launch<T>(h, l, (const T*)wr, (const T*)cur, dst, c));
                flip(dst);
                return LAB_OK;
            }
            // fuse the coarse level's first sweep from zero into the restriction
            const bool fuse_x0 = cz && jac && n1 >= 1 && l + 1 < h->levels;
            T*         x0      = fuse_x0 ? cycle_start<T>(h, l + 1, ckind, cx, o) : nullptr;
            LAB_TRY(with_vals<T>(R, bf, [&](auto* vals) -> lab_status {
                op_restrict<vt_of<decltype(vals)>, T> op{wr, cb, lv<T>::invd(h->A[l + 1]),
                                                         (T)o->omega, x0};
                return launch_rowop(R, vals, op, c.s, rb);
            }));
            LAB_TRY(cycle<T>(h, l + 1, ckind, cx, cb, cz, c, red_buf(), nullptr, fuse_x0));
            const bool fuse = last && dv && n2 == 0 && kind == 0;
            T*         dst  = jac ? oth : cur;
            LAB_TRY(with_vals<T>(P, bf, [&](auto* vals) -> lab_status {
                using VT = vt_of<decltype(vals)>;
                if(fuse)
                {
                    op_prolong<VT, T, true> op{cx, cur, dst, dv};
                    return launch_rowop(P, vals, op, c.s, dot);
                }
                op_prolong<VT, T, false> op{cx, cur, dst, nullptr};
                return launch_rowop(P, vals, op, c.s, rb);
            }));
            flip(dst);
            return LAB_OK;
        };
        auto post = [&](int sweeps, bool last) -> lab_status {
            for(int k = 0; k < sweeps; k++)
            {
                T*   res      = nullptr;
                bool fuse_dot = last && dv && k == sweeps - 1;
                LAB_TRY(smooth<T>(A, l, w, b, cur, oth, &res, c, fuse_dot ? dot : red_buf(),
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
            LAB_TRY(residual());
            LAB_TRY(coarse_correct(false, kind == 1 ? 1 : 0, false));
            LAB_TRY(post(n2, true)); // n3 = n2 (amg.cpp:537)
            if constexpr(std::is_same<T, double>::value)
                if(dv && n2 == 0)
                    LAB_TRY(dot_device(m, cur, dv, dot, c.s));
        }
        if(cur != x)
            LAB_LAUNCH(k_copy<T>, grid_for(m), 256, 0, c.s, x, (const T*)cur, m, c.skip);
        return LAB_OK;
    }

    // ================================================================ entry points
    // The reduced-precision cycle on r: x (FP32, the level-0 workspace) = cycle(0; fp32(r)).
    static lab_status cycle_lowp(hierarchy_impl* h, const cyc_ctx& c, const double* r)
    {
        level_ws&              w = h->ws[0];
        const int64_t          m = h->A[0]->m;
        const lab_amg_options* o = c.o;
        if(h->levels > 0 && o->smoother == LAB_SMOOTH_JACOBI && o->n1 >= 1)
        {
            float* x0 = cycle_start<float>(h, 0, o->cycle, w.xf, o);
            LAB_LAUNCH(k_d2f_x0, grid_for(m), 256, 0, c.s, r, w.bf, lv<float>::invd(h->A[0]),
                       (float)o->omega, x0, m, c.skip);
            return cycle<float>(h, 0, o->cycle, w.xf, (const float*)w.bf, true, c, red_buf(),
                                nullptr, true);
        }
        LAB_LAUNCH(k_d2f, grid_for(m), 256, 0, c.s, r, w.bf, m, c.skip);
        return cycle<float>(h, 0, o->cycle, w.xf, (const float*)w.bf, true, c);
    }

    lab_status cycle_precond(hierarchy_impl* h, const cyc_ctx& c, const double* r, double* z,
                             red_buf dot)
    {
        if(c.o->precision == LAB_PREC_FP64)
        {
            if(dot.out)
                return cycle<double>(h, 0, c.o->cycle, z, r, true, c, dot, r);
            return cycle<double>(h, 0, c.o->cycle, z, r, true, c);
        }
        // Reduced precision: r -> fp32, FP32 cycle, z = fp64(x) with (z, r) fused.
        LAB_TRY(cycle_lowp(h, c, r));
        const int64_t m = h->A[0]->m;
        LAB_LAUNCH(k_f2d_dot, red_grid(m), 256, 0, c.s, (const float*)h->ws[0].xf, r, z, m,
                   dot.partial, dot.counter, dot.out, c.skip);
        return LAB_OK;
    }

    lab_status cycle_precond_flex(hierarchy_impl* h, const cyc_ctx& c, const double* r,
                                  const double* q, red_buf zr, red_buf zq, const float** z32)
    {
        LAB_TRY(cycle_lowp(h, c, r));
        const int64_t m = h->A[0]->m;
        zr.skip         = c.skip;
        LAB_LAUNCH(k_f2d_dot2, red_grid(m), 256, 0, c.s, (const float*)h->ws[0].xf, r, q, m, zr,
                   zq);
        *z32 = h->ws[0].xf;
        return LAB_OK;
    }

    lab_status cycle_iterate(hierarchy_impl* h, const cyc_ctx& c, const double* b, double* x)
    {
        if(c.o->precision == LAB_PREC_FP64)
            return cycle<double>(h, 0, c.o->cycle, x, b, false, c);
        // correction form: x += cycle(0; b - A x) with the FP64 residual
        level_ws&     w = h->ws[0];
        lab_csr_impl* A = h->A[0];
        const int64_t m = A->m;
        op_residual   opr{x, b, w.r};
        LAB_TRY(launch_rowop(A, A->val, opr, c.s));
        LAB_LAUNCH(k_d2f, grid_for(m), 256, 0, c.s, (const double*)w.r, w.bf, m, c.skip);
        LAB_TRY(cycle<float>(h, 0, c.o->cycle, w.xf, (const float*)w.bf, true, c));
        LAB_LAUNCH(k_add_f2d, grid_for(m), 256, 0, c.s, (const float*)w.xf, x, m);
        return LAB_OK;
    }
}
