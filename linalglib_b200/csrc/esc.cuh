// Expand-sort-compress (ESC) engine for row-wise sparse constructions whose
// floating-point results must equal a sequential reference bit for bit.
//
// For one output row, an expansion functor emits its items in the reference's
// canonical order (item t = t-th contribution the reference would accumulate).
// Each item becomes a 64-bit key (column << 32 | t) with its value stored at
// vals[t].  A bitonic sort of the keys groups equal columns while keeping them
// in canonical order, and each group is summed left to right with one rounding
// per addition -- exactly the reference's "first contribution sets the entry,
// later ones add" loop.  Output columns come out ascending.
//
// Tiers by the row's item count n (the upper bound on its nonzeros):
//   W  n <= 256    one warp per row, keys/values in shared memory
//   B  n <= 4096   one 512-thread CTA per row, shared memory
//   G  n >  4096   one 1024-thread CTA per row, keys/values in global scratch
#pragma once

#include "internal.cuh"

#include <functional>

namespace lab
{
    constexpr int kEscLaneCap = 32;
    constexpr int kEscWarpCap = 256;
    constexpr int kEscCtaCap  = 4096;
    constexpr int kEscCtaNT   = 512;
    constexpr int kEscBigNT   = 1024;
    constexpr int kEscWarpsPerCta = 8;

    struct grp_warp
    {
        static constexpr int size = 32;
        __device__ static int rank()
        {
            return threadIdx.x & 31;
        }
        __device__ static void sync()
        {
            __syncwarp();
        }
    };

    template <int NT>
    struct grp_cta
    {
        static constexpr int size = NT;
        __device__ static int rank()
        {
            return threadIdx.x;
        }
        __device__ static void sync()
        {
            __syncthreads();
        }
    };

    __host__ __device__ inline int pow2_ceil(int n)
    {
        int p = 1;
        while(p < n)
            p <<= 1;
        return p;
    }

    __device__ __forceinline__ int key_col(uint64_t k)
    {
        return (int)(k >> 32);
    }
    __device__ __forceinline__ int key_pos(uint64_t k)
    {
        return (int)(k & 0xffffffffu);
    }
    __device__ __forceinline__ uint64_t make_key(int col, int pos)
    {
        return ((uint64_t)(uint32_t)col << 32) | (uint32_t)pos;
    }

    template <class G>
    __device__ void bitonic_sort(uint64_t* keys, int n)
    {
        const int np = pow2_ceil(n);
        for(int i = n + G::rank(); i < np; i += G::size)
            keys[i] = ~0ull;
        G::sync();
        for(int k = 2; k <= np; k <<= 1)
        {
            for(int j = k >> 1; j > 0; j >>= 1)
            {
                for(int i = G::rank(); i < np; i += G::size)
                {
                    int ixj = i ^ j;
                    if(ixj > i)
                    {
                        uint64_t a  = keys[i];
                        uint64_t b  = keys[ixj];
                        bool     up = (i & k) == 0;
                        if((a > b) == up)
                        {
                            keys[i]   = b;
                            keys[ixj] = a;
                        }
                    }
                }
                G::sync();
            }
        }
    }

    // Exclusive prefix count of `flag` across the group for one chunk of
    // G::size items; returns the exclusive position and adds the chunk total
    // to *running (shared by the group).
    template <class G>
    __device__ int group_prefix(bool flag, int* s_tmp, int& total)
    {
        if(G::size == 32)
        {
            unsigned b    = __ballot_sync(0xffffffffu, flag);
            int      lane = threadIdx.x & 31;
            total         = __popc(b);
            return __popc(b & ((1u << lane) - 1u));
        }
        else
        {
            int      lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
            unsigned b    = __ballot_sync(0xffffffffu, flag);
            if(lane == 0)
                s_tmp[wid] = __popc(b);
            __syncthreads();
            int before = 0, tot = 0;
            for(int w = 0; w < G::size / 32; w++)
            {
                int c = s_tmp[w];
                if(w < wid)
                    before += c;
                tot += c;
            }
            __syncthreads();
            total = tot;
            return before + __popc(b & ((1u << lane) - 1u));
        }
    }

    // Symbolic: number of distinct columns among the n sorted keys.
    template <class G>
    __device__ int esc_count_unique(const uint64_t* keys, int n, int* s_tmp)
    {
        int total = 0;
        for(int base = 0; base < n; base += G::size)
        {
            int  i    = base + G::rank();
            bool head = i < n && (i == 0 || key_col(keys[i]) != key_col(keys[i - 1]));
            int  t;
            group_prefix<G>(head, s_tmp, t);
            total += t;
        }
        return total;
    }

    // Numeric: groups summed in canonical order, written ascending to out.
    template <class G>
    __device__ void esc_write(const uint64_t* keys, const double* vals, int n, int* s_tmp,
                              int32_t* out_col, double* out_val)
    {
        int running = 0;
        for(int base = 0; base < n; base += G::size)
        {
            int  i    = base + G::rank();
            bool head = i < n && (i == 0 || key_col(keys[i]) != key_col(keys[i - 1]));
            int  t;
            int  pos = running + group_prefix<G>(head, s_tmp, t);
            if(head)
            {
                int    c = key_col(keys[i]);
                double s = vals[key_pos(keys[i])];
                for(int j = i + 1; j < n && key_col(keys[j]) == c; j++)
                    s = __dadd_rn(s, vals[key_pos(keys[j])]);
                out_col[pos] = c;
                if(out_val)
                    out_val[pos] = s;
            }
            running += t;
        }
    }

    // ------------------------------------------------------------------ lane tier
    // Rows with at most kEscLaneCap items: one lane per row.  The lane keeps the
    // row's distinct columns as a sorted list in shared memory (entry e of lane l
    // at [e][l], bank-conflict free) and applies the items one at a time in
    // canonical order: a new column is inserted with its value, a repeated one
    // is added to (rounded once per addition) -- the reference's accumulation.
    // Exp::emit_seq(row, f) calls f(col, val) for the row's items in order.
    constexpr int kEscLaneWarps = 4;

    template <class Exp, int MODE>
    __global__ void __launch_bounds__(32 * kEscLaneWarps)
        k_esc_lane(Exp e, const int32_t* __restrict__ rows, int nrows, int32_t* counts,
                   int32_t* out_col, double* out_val)
    {
        __shared__ int    skey[kEscLaneWarps][kEscLaneCap][32];
        __shared__ double sval[MODE == 1 ? kEscLaneWarps : 1][MODE == 1 ? kEscLaneCap : 1][32];
        const int         w = threadIdx.x >> 5, lane = threadIdx.x & 31;
        for(int r = blockIdx.x * blockDim.x + threadIdx.x; r < nrows; r += gridDim.x * blockDim.x)
        {
            const int row = rows[r];
            int       len = 0;
            e.template emit_seq<MODE == 1>(row, [&](int c, double v) {
                int pos = 0;
                while(pos < len && skey[w][pos][lane] < c)
                    pos++;
                if(pos < len && skey[w][pos][lane] == c)
                {
                    if(MODE == 1)
                        sval[w][pos][lane] = __dadd_rn(sval[w][pos][lane], v);
                    return;
                }
                for(int q = len; q > pos; q--)
                {
                    skey[w][q][lane] = skey[w][q - 1][lane];
                    if(MODE == 1)
                        sval[w][q][lane] = sval[w][q - 1][lane];
                }
                skey[w][pos][lane] = c;
                if(MODE == 1)
                    sval[w][pos][lane] = v;
                len++;
            });
            if(MODE == 0)
                counts[row] = len;
            else
            {
                const int32_t o = e.out_start(row);
                for(int q = 0; q < len; q++)
                {
                    out_col[o + q] = skey[w][q][lane];
                    if(out_val)
                        out_val[o + q] = sval[MODE == 1 ? w : 0][MODE == 1 ? q : 0][lane];
                }
            }
        }
    }

    // ------------------------------------------------------------------ kernels
    // Exp interface:
    //   __device__ int  upper(int row) const        item count (computed before)
    //   template <class G> __device__ int expand(int row, uint64_t* keys, double* vals) const
    //        writes the row's items in canonical order, ends with G::sync(), returns n
    //   __device__ int32_t out_start(int row) const  (numeric pass)
    // MODE 0 = symbolic (counts[row] = distinct columns), 1 = numeric.
    template <class Exp, int MODE>
    __global__ void __launch_bounds__(32 * kEscWarpsPerCta)
        k_esc_warp(Exp e, const int32_t* __restrict__ rows, int nrows, int32_t* counts,
                   int32_t* out_col, double* out_val)
    {
        __shared__ uint64_t s_keys[kEscWarpsPerCta][kEscWarpCap];
        __shared__ double   s_vals[kEscWarpsPerCta][kEscWarpCap];
        const int           wid   = threadIdx.x >> 5;
        const int           gwarp = blockIdx.x * kEscWarpsPerCta + wid;
        const int           nwarp = gridDim.x * kEscWarpsPerCta;
        for(int r = gwarp; r < nrows; r += nwarp)
        {
            int row = rows ? rows[r] : r;
            int n   = e.template expand<grp_warp>(row, s_keys[wid], s_vals[wid]);
            bitonic_sort<grp_warp>(s_keys[wid], n);
            if(MODE == 0)
            {
                int c = esc_count_unique<grp_warp>(s_keys[wid], n, nullptr);
                if((threadIdx.x & 31) == 0)
                    counts[row] = c;
            }
            else
            {
                int32_t o = e.out_start(row);
                esc_write<grp_warp>(s_keys[wid], s_vals[wid], n, nullptr, out_col + o,
                                    out_val ? out_val + o : nullptr);
            }
            __syncwarp();
        }
    }

    template <class Exp, int MODE>
    __global__ void __launch_bounds__(kEscCtaNT)
        k_esc_cta(Exp e, const int32_t* __restrict__ rows, int nrows, int32_t* counts,
                  int32_t* out_col, double* out_val)
    {
        extern __shared__ __align__(16) unsigned char esc_smem[];
        uint64_t*      keys = reinterpret_cast<uint64_t*>(esc_smem);
        double*        vals = reinterpret_cast<double*>(esc_smem + sizeof(uint64_t) * kEscCtaCap);
        __shared__ int s_tmp[32];
        for(int r = blockIdx.x; r < nrows; r += gridDim.x)
        {
            int row = rows[r];
            int n   = e.template expand<grp_cta<kEscCtaNT>>(row, keys, vals);
            bitonic_sort<grp_cta<kEscCtaNT>>(keys, n);
            if(MODE == 0)
            {
                int c = esc_count_unique<grp_cta<kEscCtaNT>>(keys, n, s_tmp);
                if(threadIdx.x == 0)
                    counts[row] = c;
            }
            else
            {
                int32_t o = e.out_start(row);
                esc_write<grp_cta<kEscCtaNT>>(keys, vals, n, s_tmp, out_col + o,
                                              out_val ? out_val + o : nullptr);
            }
            __syncthreads();
        }
    }

    template <class Exp, int MODE>
    __global__ void __launch_bounds__(kEscBigNT)
        k_esc_big(Exp e, const int32_t* __restrict__ rows, int nrows, const int64_t* offsets,
                  uint64_t* g_keys, double* g_vals, int32_t* counts, int32_t* out_col,
                  double* out_val)
    {
        __shared__ int s_tmp[32];
        for(int r = blockIdx.x; r < nrows; r += gridDim.x)
        {
            int       row  = rows[r];
            uint64_t* keys = g_keys + offsets[r];
            double*   vals = g_vals + offsets[r];
            int       n    = e.template expand<grp_cta<kEscBigNT>>(row, keys, vals);
            bitonic_sort<grp_cta<kEscBigNT>>(keys, n);
            if(MODE == 0)
            {
                int c = esc_count_unique<grp_cta<kEscBigNT>>(keys, n, s_tmp);
                if(threadIdx.x == 0)
                    counts[row] = c;
            }
            else
            {
                int32_t o = e.out_start(row);
                esc_write<grp_cta<kEscBigNT>>(keys, vals, n, s_tmp, out_col + o,
                                              out_val ? out_val + o : nullptr);
            }
            __syncthreads();
        }
    }

    // Row classification by item count: tier lists (unordered within a tier).
    struct esc_tiers
    {
        dbuf<int32_t> rows; // [m] : lane rows, then W rows, then B rows, then G rows
        int           nl = 0, nw = 0, nb = 0, ng = 0;
        dbuf<int64_t> g_offsets;  // [ng] scratch offsets of G rows
        int64_t       g_total = 0;
        dbuf<uint64_t> g_keys;
        dbuf<double>   g_vals;
    };

    lab_status esc_classify(const int32_t* upper, int64_t m, esc_tiers& t, cudaStream_t s);

    template <class Exp, int MODE>
    lab_status esc_run(const Exp& e, int64_t m, esc_tiers& t, int32_t* counts, int32_t* out_col,
                       double* out_val, cudaStream_t s)
    {
        stream_fork f(s, m); // the tiers are disjoint row sets: they run side by side
        if(t.nl > 0)
        {
            unsigned grid = (unsigned)std::min<int64_t>(
                ceil_div<int64_t>(t.nl, 32 * kEscLaneWarps), (int64_t)num_sms() * 16);
            LAB_LAUNCH((k_esc_lane<Exp, MODE>), grid, 32 * kEscLaneWarps, 0, f.next(), e, t.rows.get(),
                       t.nl, counts, out_col, out_val);
        }
        const int32_t* wrows = t.rows.get() + t.nl;
        if(t.nw > 0)
        {
            unsigned grid = (unsigned)std::min<int64_t>(
                ceil_div<int64_t>(t.nw, kEscWarpsPerCta), (int64_t)num_sms() * 8);
            LAB_LAUNCH((k_esc_warp<Exp, MODE>), grid, 32 * kEscWarpsPerCta, 0, f.next(), e, wrows, t.nw,
                       counts, out_col, out_val);
        }
        if(t.nb > 0)
        {
            size_t smem = (sizeof(uint64_t) + sizeof(double)) * kEscCtaCap;
            static const cudaError_t attr = cudaFuncSetAttribute(
                k_esc_cta<Exp, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            LAB_CUDA(attr);
            unsigned grid = (unsigned)std::min<int64_t>(t.nb, (int64_t)num_sms() * 3);
            LAB_LAUNCH((k_esc_cta<Exp, MODE>), grid, kEscCtaNT, smem, f.next(), e, wrows + t.nw, t.nb,
                       counts, out_col, out_val);
        }
        if(t.ng > 0)
        {
            unsigned grid = (unsigned)std::min<int64_t>(t.ng, (int64_t)num_sms() * 2);
            LAB_LAUNCH((k_esc_big<Exp, MODE>), grid, kEscBigNT, 0, f.next(), e, wrows + t.nw + t.nb,
                       t.ng, t.g_offsets.get(), t.g_keys.get(), t.g_vals.get(), counts, out_col,
                       out_val);
        }
        return LAB_OK;
    }

    // Full two-pass construction of a CSR matrix (m x n) from an expansion:
    // item counts -> tiers -> symbolic counts -> row_ptr -> numeric fill.
    // n_late: when given, the column count is n_late() evaluated after the first
    // synchronisation here (for a value the caller copies to pinned memory
    // asynchronously, so it needs no round trip of its own).
    template <class Exp>
    lab_status esc_build(const Exp& e, const int32_t* upper, int64_t m, int64_t n,
                         lab_csr_impl** out, cudaStream_t s,
                         const std::function<int64_t()>& n_late = {})
    {
        esc_tiers t;
        LAB_TRY(esc_classify(upper, m, t, s));
        if(n_late)
            n = n_late();
        lab_csr_impl* C = nullptr;
        dbuf<int32_t> counts;
        LAB_TRY(counts.alloc((size_t)m + 1, s));
        if(m > 0)
            LAB_CUDA(cudaMemsetAsync(counts.get(), 0, sizeof(int32_t) * m, s));
        LAB_TRY((esc_run<Exp, 0>(e, m, t, counts.get(), nullptr, nullptr, s)));
        // allocate C with the exact nnz
        dbuf<int32_t> rp;
        LAB_TRY(rp.alloc((size_t)m + 1, s));
        int64_t nnz = 0;
        LAB_TRY(counts_to_rowptr(counts.get(), rp.get(), m, &nnz, s));
        LAB_TRY(csr_alloc(&C, m, n, nnz, s));
        cudaError_t ce = cudaMemcpyAsync(C->row_ptr, rp.get(), sizeof(int32_t) * (m + 1),
                                         cudaMemcpyDeviceToDevice, s);
        if(ce != cudaSuccess)
        {
            csr_release(C);
            return cuda_status(ce, "esc_build row_ptr", __FILE__, __LINE__);
        }
        Exp e2       = e;
        e2.out_rp    = C->row_ptr;
        lab_status st = esc_run<Exp, 1>(e2, m, t, nullptr, C->col_ind, C->val, s);
        if(st != LAB_OK)
        {
            csr_release(C);
            return st;
        }
        *out = C;
        return LAB_OK;
    }
}
