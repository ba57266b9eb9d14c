// SpGEMM, SpGEAM and transpose on the ESC engine (esc.cuh), plus the tier
// classification shared with the AMG prolongation builders.
#include "amg.cuh"
#include "esc.cuh"

namespace lab
{
    // ------------------------------------------------------------ tiers
    // 0: lane tier, 1: warp tier, 2: CTA tier, 3: global tier
    __device__ __forceinline__ int tier_of(int u)
    {
        return u <= kEscLaneCap ? 0 : (u <= kEscWarpCap ? 1 : (u <= kEscCtaCap ? 2 : 3));
    }

    __global__ void k_tier_count(const int32_t* __restrict__ upper, int64_t m, int* cnt)
    {
        __shared__ int s[4];
        if(threadIdx.x < 4)
            s[threadIdx.x] = 0;
        __syncthreads();
        for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m;
            i += (int64_t)gridDim.x * blockDim.x)
            atomicAdd(&s[tier_of(upper[i])], 1);
        __syncthreads();
        if(threadIdx.x < 4 && s[threadIdx.x])
            atomicAdd(&cnt[threadIdx.x], s[threadIdx.x]);
    }

    // Append row i to list `t`: one atomic per warp and list (warp-aggregated), so
    // millions of rows do not serialise on a single counter.  Must be called by
    // every lane of the warp (inactive lanes pass t < 0).
    __device__ __forceinline__ int warp_append(int* cursor, int t, int ntiers)
    {
        const int lane = threadIdx.x & 31;
        int       pos  = -1;
        for(int tt = 0; tt < ntiers; tt++)
        {
            unsigned bal = __ballot_sync(0xffffffffu, t == tt);
            if(!bal)
                continue;
            int leader = __ffs(bal) - 1;
            int base   = 0;
            if(lane == leader)
                base = atomicAdd(&cursor[tt], __popc(bal));
            base = __shfl_sync(0xffffffffu, base, leader);
            if(t == tt)
                pos = base + __popc(bal & ((1u << lane) - 1u));
        }
        return pos;
    }

    __global__ void k_tier_fill(const int32_t* __restrict__ upper, int64_t m, int* cursor,
                                int32_t* rows, int64_t* gsize)
    {
        // warp-uniform trip count: whole warps step together
        for(int64_t base = blockIdx.x * (int64_t)blockDim.x; base < m;
            base += (int64_t)gridDim.x * blockDim.x)
        {
            const int64_t i = base + threadIdx.x;
            int           u = i < m ? upper[i] : 0;
            int           t = i < m ? tier_of(u) : -1;
            int           p = warp_append(cursor, t, 4);
            if(t >= 0)
            {
                rows[p] = (int32_t)i;
                if(t == 3)
                    gsize[p - cursor[5]] = pow2_ceil(u);
            }
        }
    }

    lab_status esc_classify(const int32_t* upper, int64_t m, esc_tiers& t, cudaStream_t s)
    {
        t.nl = t.nw = t.nb = t.ng = 0;
        if(m == 0)
            return LAB_OK;
        dbuf<int> cnt;
        LAB_TRY(cnt.alloc(8, s));
        LAB_CUDA(cudaMemsetAsync(cnt.get(), 0, sizeof(int) * 8, s));
        unsigned grid = (unsigned)std::min<int64_t>(ceil_div<int64_t>(m, 256), 4096);
        LAB_LAUNCH(k_tier_count, grid, 256, 0, s, upper, m, cnt.get());
        int h[4];
        LAB_TRY(copy_d2h_sync(h, cnt.get(), sizeof(int) * 4, s));
        t.nl = h[0];
        t.nw = h[1];
        t.nb = h[2];
        t.ng = h[3];
        // cursors: [0..3] = start of each tier's run in rows[], [5] = G start (gsize index)
        const int gs = t.nl + t.nw + t.nb;
        int cur[8] = {0, t.nl, t.nl + t.nw, gs, 0, gs, 0, 0};
        LAB_CUDA(cudaMemcpyAsync(cnt.get(), cur, sizeof(cur), cudaMemcpyHostToDevice, s));
        LAB_TRY(t.rows.alloc((size_t)m, s));
        LAB_TRY(t.g_offsets.alloc((size_t)std::max(t.ng, 1) + 1, s));
        // (cur[] may leave scope at once: a copy from pageable host memory is staged
        // before cudaMemcpyAsync returns)
        LAB_LAUNCH(k_tier_fill, grid, 256, 0, s, upper, m, cnt.get(), t.rows.get(),
                   t.g_offsets.get());
        if(t.ng > 0)
        {
            // scratch offsets: exclusive scan of padded sizes
            LAB_CUDA(cudaMemsetAsync(t.g_offsets.get() + t.ng, 0, sizeof(int64_t), s));
            LAB_TRY(scan_i64(t.g_offsets.get(), t.ng + 1, s));
            LAB_TRY(copy_d2h_sync(&t.g_total, t.g_offsets.get() + t.ng, sizeof(int64_t), s));
            LAB_TRY(t.g_keys.alloc((size_t)t.g_total, s));
            LAB_TRY(t.g_vals.alloc((size_t)t.g_total, s));
        }
        return LAB_OK;
    }

    // ------------------------------------------------------------ expansions
    struct csr_ref
    {
        const int32_t* rp;
        const int32_t* ci;
        const double*  v;
    };

    // C = A*B: items in A-row order, then B-row order (host_csrgemm.cpp:119-139).
    struct exp_gemm
    {
        csr_ref        A, B;
        const int32_t* out_rp = nullptr;
        template <class G>
        __device__ int expand(int row, uint64_t* keys, double* vals) const
        {
            int off = 0;
            for(int j = A.rp[row]; j < A.rp[row + 1]; j++)
            {
                const int    k  = A.ci[j];
                const double a  = A.v[j]; // alpha * a with alpha = 1 is exact
                const int    b0 = B.rp[k], b1 = B.rp[k + 1];
                for(int p = b0 + G::rank(); p < b1; p += G::size)
                {
                    int t   = off + (p - b0);
                    keys[t] = make_key(B.ci[p], t);
                    vals[t] = __dmul_rn(a, B.v[p]);
                }
                off += b1 - b0;
            }
            G::sync();
            return off;
        }
        template <bool VALS, class F>
        __device__ void emit_seq(int row, F&& f) const
        {
            // canonical order (A entry, then B entry); the loads of four A entries,
            // their B-row bounds and four B entries at a time are issued together
            const int a0 = A.rp[row], a1 = A.rp[row + 1];
            for(int j0 = a0; j0 < a1; j0 += 4)
            {
                int    kk[4], lo[4], hi[4];
                double av[4];
#pragma unroll
                for(int u = 0; u < 4; u++)
                {
                    const bool ok = j0 + u < a1;
                    kk[u]         = ok ? A.ci[j0 + u] : 0;
                    av[u]         = (VALS && ok) ? A.v[j0 + u] : 0.0;
                }
#pragma unroll
                for(int u = 0; u < 4; u++)
                {
                    const bool ok = j0 + u < a1;
                    lo[u]         = ok ? B.rp[kk[u]] : 0;
                    hi[u]         = ok ? B.rp[kk[u] + 1] : 0;
                }
#pragma unroll
                for(int u = 0; u < 4; u++)
                    for(int p0 = lo[u]; p0 < hi[u]; p0 += 4)
                    {
                        int    cc[4];
                        double bv[4];
#pragma unroll
                        for(int t = 0; t < 4; t++)
                        {
                            const bool ok = p0 + t < hi[u];
                            cc[t]         = ok ? B.ci[p0 + t] : 0;
                            bv[t]         = (VALS && ok) ? B.v[p0 + t] : 0.0;
                        }
#pragma unroll
                        for(int t = 0; t < 4; t++)
                            if(p0 + t < hi[u])
                                f(cc[t], VALS ? __dmul_rn(av[u], bv[t]) : 0.0);
                    }
            }
        }
        __device__ int32_t out_start(int row) const
        {
            return out_rp[row];
        }
    };

    __global__ void k_gemm_upper(csr_ref A, const int32_t* __restrict__ Brp, int64_t m,
                                 int32_t* upper, int* overflow)
    {
        int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
        if(i >= m)
            return;
        int64_t u = 0;
        for(int j = A.rp[i]; j < A.rp[i + 1]; j++)
        {
            int k = A.ci[j];
            u += Brp[k + 1] - Brp[k];
        }
        if(u > (1 << 30))
        {
            atomicOr(overflow, 1);
            u = 0;
        }
        upper[i] = (int32_t)u;
    }

    // Warp-per-row form for long A rows (coarse levels): the lanes take strided
    // entries and the 64-bit sum is reduced by shuffles (integer: exact).
    __global__ void k_gemm_upper_warp(csr_ref A, const int32_t* __restrict__ Brp, int64_t m,
                                      int32_t* upper, int* overflow)
    {
        const int64_t i    = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
        const int     lane = threadIdx.x & 31;
        if(i >= m)
            return;
        long long u = 0;
        for(int j = A.rp[i] + lane; j < A.rp[i + 1]; j += 32)
        {
            const int k = A.ci[j];
            u += Brp[k + 1] - Brp[k];
        }
#pragma unroll
        for(int o = 16; o > 0; o >>= 1)
            u += __shfl_xor_sync(0xffffffffu, u, o);
        if(lane != 0)
            return;
        if(u > (1 << 30))
        {
            atomicOr(overflow, 1);
            u = 0;
        }
        upper[i] = (int32_t)u;
    }

    // C = alpha*A + beta*B: A's entries then B's (host_csrgeam.cpp).
    struct exp_geam
    {
        csr_ref        A, B;
        double         alpha, beta;
        const int32_t* out_rp = nullptr;
        template <class G>
        __device__ int expand(int row, uint64_t* keys, double* vals) const
        {
            const int a0 = A.rp[row], a1 = A.rp[row + 1];
            const int b0 = B.rp[row], b1 = B.rp[row + 1];
            for(int p = a0 + G::rank(); p < a1; p += G::size)
            {
                int t   = p - a0;
                keys[t] = make_key(A.ci[p], t);
                vals[t] = __dmul_rn(alpha, A.v[p]);
            }
            for(int p = b0 + G::rank(); p < b1; p += G::size)
            {
                int t   = (a1 - a0) + (p - b0);
                keys[t] = make_key(B.ci[p], t);
                vals[t] = __dmul_rn(beta, B.v[p]);
            }
            G::sync();
            return (a1 - a0) + (b1 - b0);
        }
        template <bool VALS, class F>
        __device__ void emit_seq(int row, F&& f) const
        {
            for(int p = A.rp[row]; p < A.rp[row + 1]; p++)
                f(A.ci[p], VALS ? __dmul_rn(alpha, A.v[p]) : 0.0);
            for(int p = B.rp[row]; p < B.rp[row + 1]; p++)
                f(B.ci[p], VALS ? __dmul_rn(beta, B.v[p]) : 0.0);
        }
        __device__ int32_t out_start(int row) const
        {
            return out_rp[row];
        }
    };

    __global__ void k_geam_upper(const int32_t* __restrict__ Arp, const int32_t* __restrict__ Brp,
                                 int64_t m, int32_t* upper)
    {
        int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
        if(i < m)
            upper[i] = (Arp[i + 1] - Arp[i]) + (Brp[i + 1] - Brp[i]);
    }

    // Sort each row of an unsorted CSR (unique columns) by column.
    struct exp_rowsort
    {
        csr_ref        A;
        const int32_t* out_rp = nullptr;
        template <class G>
        __device__ int expand(int row, uint64_t* keys, double* vals) const
        {
            const int a0 = A.rp[row], a1 = A.rp[row + 1];
            for(int p = a0 + G::rank(); p < a1; p += G::size)
            {
                int t   = p - a0;
                keys[t] = make_key(A.ci[p], t);
                vals[t] = A.v[p];
            }
            G::sync();
            return a1 - a0;
        }
        template <bool VALS, class F>
        __device__ void emit_seq(int row, F&& f) const
        {
            for(int p = A.rp[row]; p < A.rp[row + 1]; p++)
                f(A.ci[p], VALS ? A.v[p] : 0.0);
        }
        __device__ int32_t out_start(int row) const
        {
            return out_rp[row];
        }
    };

    __global__ void k_row_lengths(const int32_t* __restrict__ rp, int64_t m, int32_t* len)
    {
        int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
        if(i < m)
            len[i] = rp[i + 1] - rp[i];
    }

    lab_status row_lengths(const int32_t* rp, int64_t m, int32_t* len, cudaStream_t s)
    {
        if(m > 0)
            LAB_LAUNCH(k_row_lengths, (unsigned)ceil_div<int64_t>(m, 256), 256, 0, s, rp, m, len);
        return LAB_OK;
    }

    // ------------------------------------------------------------ transpose
    __global__ void k_col_count(const int32_t* __restrict__ ci, int64_t nnz, int32_t* cnt)
    {
        for(int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < nnz;
            j += (int64_t)gridDim.x * blockDim.x)
            atomicAdd(&cnt[ci[j]], 1);
    }

    __global__ void k_transpose_scatter(csr_ref A, int64_t m, int32_t* cursor, int32_t* tci,
                                        double* tv)
    {
        int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
        if(i >= m)
            return;
        for(int j = A.rp[i]; j < A.rp[i + 1]; j++)
        {
            int p  = atomicAdd(&cursor[A.ci[j]], 1);
            tci[p] = (int32_t)i;
            tv[p]  = A.v[j];
        }
    }

    // T = A^T with rows listing source rows ascending (host_csr2csc.cpp:30-75).
    lab_status transpose(const lab_csr_impl* A, lab_csr_impl** out, cudaStream_t s)
    {
        const int64_t m = A->m, n = A->n, nnz = A->nnz;
        dbuf<int32_t> cnt, cursor, tci;
        dbuf<double>  tv;
        LAB_TRY(cnt.alloc((size_t)n + 1, s));
        LAB_CUDA(cudaMemsetAsync(cnt.get(), 0, sizeof(int32_t) * (n + 1), s));
        if(nnz > 0)
        {
            unsigned g = (unsigned)std::min<int64_t>(ceil_div<int64_t>(nnz, 256), 8192);
            LAB_LAUNCH(k_col_count, g, 256, 0, s, A->col_ind, nnz, cnt.get());
        }
        lab_csr_impl* T = nullptr;
        LAB_TRY(csr_alloc(&T, n, m, nnz, s));
        lab_status st = counts_to_rowptr(cnt.get(), T->row_ptr, n, nullptr, s);
        if(st == LAB_OK && nnz > 0)
        {
            st = cursor.alloc((size_t)n + 1, s);
            if(st == LAB_OK)
                st = tci.alloc((size_t)nnz, s);
            if(st == LAB_OK)
                st = tv.alloc((size_t)nnz, s);
            if(st == LAB_OK)
            {
                cudaMemcpyAsync(cursor.get(), T->row_ptr, sizeof(int32_t) * (n + 1),
                                cudaMemcpyDeviceToDevice, s);
                k_transpose_scatter<<<(unsigned)ceil_div<int64_t>(m, 256), 256, 0, s>>>(
                    csr_ref{A->row_ptr, A->col_ind, A->val}, m, cursor.get(), tci.get(), tv.get());
                g_launches.fetch_add(1);
                st = LAB_OK;
                if(cudaGetLastError() != cudaSuccess)
                    st = LAB_CUDA_ERROR;
            }
            if(st == LAB_OK)
            {
                // sort each row of T by source row
                dbuf<int32_t> upper;
                st = upper.alloc((size_t)n + 1, s);
                if(st == LAB_OK)
                    st = row_lengths(T->row_ptr, n, upper.get(), s);
                esc_tiers t;
                if(st == LAB_OK)
                    st = esc_classify(upper.get(), n, t, s);
                exp_rowsort e{csr_ref{T->row_ptr, tci.get(), tv.get()}, T->row_ptr};
                if(st == LAB_OK)
                    st = esc_run<exp_rowsort, 1>(e, n, t, nullptr, T->col_ind, T->val, s);
            }
        }
        if(st != LAB_OK)
        {
            csr_release(T);
            return st;
        }
        *out = T;
        return LAB_OK;
    }

    // ------------------------------------------------------------ hash-accumulator SpGEMM
    // Rows with more than 32 products (A*P and the Galerkin R*(A*P) on every level)
    // go to a warp-per-row hash accumulator whose table lives in shared memory and
    // is sized per row class (2x the row's product bound in the symbolic pass, 2x
    // its exact column count in the numeric pass), so small rows run at high
    // occupancy.  The row's products are enumerated flat: the A entries of the row
    // are staged with their B-row bounds and a prefix of the B-row lengths, then
    // each lane fetches kHashU products 32 apart (independent loads in flight) and
    // the warp applies them 32 at a time in canonical order.  Lanes holding the
    // same column in one chunk form a group (match.any) whose lowest lane adds the
    // members' products one by one, in lane order, to that column's slot; the first
    // product of a column is assigned.  That is the accumulation order of
    // host_csrgemm.cpp:119-139 (A-row order, then B-row order, rounded once per
    // addition).  The filled slots are then sorted by column and written.
    constexpr int kHashACap    = 64; // A entries staged per piece
    constexpr int kHashU       = 4;  // products in flight per lane
    constexpr int kHashClasses = 8;
    static_assert(kHashU == 4, "the chunk's slot map is one int4 per lane");

    template <int MODE, int HS>
    struct alignas(16) hash_smem
    {
        int      jmap[32 * kHashU]; // A entry of each product slot of the current chunk
        int      key[HS];
        double   val[MODE == 1 ? HS : 1];
        uint64_t sk[MODE == 1 ? HS : 1]; // the filled slots (<= 3/4 of HS) padded to a power of 2
        double   aa[MODE == 1 ? kHashACap : 1];
        double   sp[MODE == 1 ? 32 : 1];
        int      ab0[kHashACap];
        int      aoff[kHashACap];
        int      claims;
    };

    __device__ __forceinline__ unsigned hash_slot(int c, unsigned mask)
    {
        return ((unsigned)c * 2654435761u >> 7) & mask;
    }

    __device__ __forceinline__ int warp_inclusive_sum(int v)
    {
        const int lane = threadIdx.x & 31;
#pragma unroll
        for(int o = 1; o < 32; o <<= 1)
        {
            int t = __shfl_up_sync(0xffffffffu, v, o);
            if(lane >= o)
                v += t;
        }
        return v;
    }

    // Claims col's slot (linear probing); returns the slot, *isnew if it was empty.
    template <int HS>
    __device__ __forceinline__ unsigned hash_claim(int* key, int col, bool* isnew)
    {
        constexpr unsigned mask = HS - 1;
        unsigned           slot = hash_slot(col, mask);
        *isnew                  = false;
        for(unsigned probe = 0; probe < HS; probe++)
        {
            int old = atomicCAS(&key[slot], -1, col);
            if(old == -1)
            {
                *isnew = true;
                break;
            }
            if(old == col)
                break;
            slot = (slot + 1) & mask;
        }
        return slot;
    }

    // MODE 0: symbolic (counts[row], or the row goes to the overflow list when more
    // than 3/4 of the table fills up); MODE 1: numeric into out_rp / out_ci / out_v.
    template <int MODE, int HS, int WARPS>
    __global__ void __launch_bounds__(32 * WARPS)
        k_hash_gemm(csr_ref A, csr_ref B, const int32_t* __restrict__ rows, int nrows,
                    int32_t* counts, const int32_t* __restrict__ out_rp, int32_t* out_ci,
                    double* out_v, int32_t* ovf_rows, int* n_ovf, const int* nrows_dev)
    {
        if(nrows_dev) // the list's length is known on the device only (nrows: its capacity)
            nrows = min(nrows, *nrows_dev);
        using S = hash_smem<MODE, HS>;
        extern __shared__ __align__(16) unsigned char hsm[];
        const int      wid  = threadIdx.x >> 5;
        const int      lane = threadIdx.x & 31;
        S&             sm   = reinterpret_cast<S*>(hsm)[wid];
        const unsigned full = 0xffffffffu;

        for(int r = blockIdx.x * WARPS + wid; r < nrows; r += gridDim.x * WARPS)
        {
            const int row = rows[r];
            for(int q = lane; q < HS; q += 32)
                sm.key[q] = -1;
            if(lane == 0)
                sm.claims = 0;
            __syncwarp();
            bool      ovf   = false;
            const int a_end = A.rp[row + 1];
            for(int ps = A.rp[row]; ps < a_end && !ovf; ps += kHashACap)
            {
                const int nA = min(kHashACap, a_end - ps);
                int       len[2];
#pragma unroll
                for(int h = 0; h < 2; h++)
                {
                    const int q = lane + 32 * h;
                    len[h]      = 0;
                    if(q < nA)
                    {
                        const int k  = A.ci[ps + q];
                        const int b0 = B.rp[k];
                        len[h]       = B.rp[k + 1] - b0;
                        sm.ab0[q]    = b0;
                        if(MODE == 1)
                            sm.aa[q] = A.v[ps + q];
                    }
                }
                const int inc0 = warp_inclusive_sum(len[0]);
                const int inc1 = warp_inclusive_sum(len[1]);
                const int tot0 = __shfl_sync(full, inc0, 31);
                const int T    = tot0 + __shfl_sync(full, inc1, 31);
                sm.aoff[lane]      = inc0 - len[0];
                sm.aoff[lane + 32] = tot0 + inc1 - len[1];
                __syncwarp();
                int jcarry = 0; // A entry of the product just before the chunk
                for(int t0 = 0; t0 < T && !ovf; t0 += 32 * kHashU)
                {
                    // Map the chunk's product slots t0 .. t0 + 127 to their A entries
                    // (the largest j with aoff[j] <= t): each non-empty A entry marks the
                    // slot where its products start, then an inclusive max-scan over the
                    // slots (lane k owns slots 4k .. 4k + 3) fills the rest.
                    reinterpret_cast<int4*>(sm.jmap)[lane] = make_int4(-1, -1, -1, -1);
                    __syncwarp();
#pragma unroll
                    for(int h = 0; h < 2; h++)
                    {
                        const int j = lane + 32 * h;
                        if(j < nA)
                        {
                            const int o   = sm.aoff[j];
                            const int nxt = j + 1 < nA ? sm.aoff[j + 1] : T;
                            if(nxt > o && o >= t0 && o < t0 + 32 * kHashU)
                                sm.jmap[o - t0] = j;
                        }
                    }
                    __syncwarp();
                    int4 q4 = reinterpret_cast<const int4*>(sm.jmap)[lane];
                    q4.y    = max(q4.x, q4.y);
                    q4.z    = max(q4.y, q4.z);
                    q4.w    = max(q4.z, q4.w);
                    int run = q4.w;
#pragma unroll
                    for(int o = 1; o < 32; o <<= 1)
                    {
                        const int t = __shfl_up_sync(full, run, o);
                        if(lane >= o)
                            run = max(run, t);
                    }
                    int before = __shfl_up_sync(full, run, 1);
                    before     = lane == 0 ? jcarry : max(jcarry, before);
                    q4.x       = max(before, q4.x);
                    q4.y       = max(before, q4.y);
                    q4.z       = max(before, q4.z);
                    q4.w       = max(before, q4.w);
                    reinterpret_cast<int4*>(sm.jmap)[lane] = q4;
                    jcarry = __shfl_sync(full, q4.w, 31);
                    __syncwarp();
                    int    c[kHashU];
                    int    jj[kHashU];
                    double bv[kHashU];
#pragma unroll
                    for(int u = 0; u < kHashU; u++)
                    {
                        const int t = t0 + 32 * u + lane;
                        c[u]        = -1;
                        jj[u]       = 0;
                        bv[u]       = 0.0;
                        if(t < T)
                        {
                            const int j = sm.jmap[32 * u + lane];
                            const int p = sm.ab0[j] + (t - sm.aoff[j]);
                            jj[u]       = j;
                            c[u]        = __ldg(B.ci + p);
                            if(MODE == 1)
                                bv[u] = __ldg(B.v + p);
                        }
                    }
#pragma unroll
                    for(int u = 0; u < kHashU; u++)
                    {
                        const int cc = c[u];
                        if(MODE == 0)
                        {
                            bool isnew = false;
                            if(cc >= 0)
                                hash_claim<HS>(sm.key, cc, &isnew);
                            const unsigned nb = __ballot_sync(full, isnew);
                            if(lane == 0)
                                sm.claims += __popc(nb);
                        }
                        else
                        {
                            const double   pr  = cc >= 0 ? __dmul_rn(sm.aa[jj[u]], bv[u]) : 0.0;
                            const unsigned grp = __match_any_sync(full, cc);
                            sm.sp[lane]        = pr;
                            __syncwarp();
                            if(cc >= 0 && (grp & ((1u << lane) - 1u)) == 0)
                            {
                                bool           isnew = false;
                                const unsigned slot  = hash_claim<HS>(sm.key, cc, &isnew);
                                unsigned       mm    = grp;
                                double         e;
                                if(isnew)
                                {
                                    e = pr;
                                    mm &= mm - 1u;
                                }
                                else
                                    e = sm.val[slot];
                                while(mm)
                                {
                                    e = __dadd_rn(e, sm.sp[__ffs(mm) - 1]);
                                    mm &= mm - 1u;
                                }
                                sm.val[slot] = e;
                            }
                        }
                        __syncwarp();
                    }
                    if(MODE == 0 && sm.claims > 3 * HS / 4)
                        ovf = true; // too many distinct columns for this table
                }
                __syncwarp();
            }
            if(MODE == 0)
            {
                if(lane == 0)
                {
                    if(ovf)
                        ovf_rows[atomicAdd(n_ovf, 1)] = row;
                    else
                        counts[row] = sm.claims;
                }
            }
            else
            {
                // compact the filled slots, sort by column, write
                int n = 0;
                for(int q0 = 0; q0 < HS; q0 += 32)
                {
                    const int      q    = q0 + lane;
                    const bool     fill = sm.key[q] >= 0;
                    const unsigned bal  = __ballot_sync(full, fill);
                    if(fill)
                        sm.sk[n + __popc(bal & ((1u << lane) - 1u))] = make_key(sm.key[q], q);
                    n += __popc(bal);
                }
                __syncwarp();
                bitonic_sort<grp_warp>(sm.sk, n);
                const int32_t o = out_rp[row];
                for(int i = lane; i < n; i += 32)
                {
                    out_ci[o + i] = key_col(sm.sk[i]);
                    out_v[o + i]  = sm.val[key_pos(sm.sk[i])];
                }
            }
            __syncwarp();
        }
    }

    // Row classes.  Symbolic (by the product bound ub): 0 = lane tier (ub <= 32),
    // 1..4 = hash tables of 128..1024 slots (ub <= slots / 2; class 4 takes every
    // larger row and checks for overflow, and its overflow rows get 4096 slots).  Numeric (by the exact column count of
    // rows with ub > 32): 1..6 = tables of 64..2048 slots (count <= 3/4 of the
    // slots), 7 = global sort tier.
    // Row class of a product row.  Phase 0 (symbolic, by the product bound ub): the
    // smallest table of 128..1024 slots with slots >= sym / 2 x ub (sym = 2 by
    // default; the bound is loose for Galerkin products, many products per column,
    // and rows that fill 3/4 of the 1024-slot table are retried with 4096 slots, then
    // the global sort tier).  Phase 1 (numeric, by the exact count): the smallest
    // table of 64..2048 slots filled to at most fill_num / fill_den (3/4 by default:
    // fewer slots to clear and compact, more tables per SM, a few more probes);
    // larger rows go to the sort tier.  The class only sizes the table: every class
    // accumulates in the same order, so results do not depend on the tuning.
    __device__ __forceinline__ int gemm_class(int phase, int ub, int cnt, gemm_tune t)
    {
        if(ub <= kEscLaneCap)
            return 0;
        if(phase == 0)
        {
            int c = 1, hs = 128;
            while(c < 4 && t.sym * ub > 2 * hs)
            {
                c++;
                hs <<= 1;
            }
            return c;
        }
        if(t.fill_den * cnt > t.fill_num * 2048)
            return 7;
        int c = 1, hs = 64;
        while(t.fill_den * cnt > t.fill_num * hs)
        {
            c++;
            hs <<= 1;
        }
        return c;
    }

    __global__ void k_gemm_class_count(int phase, const int32_t* __restrict__ upper,
                                       const int32_t* __restrict__ rp, int64_t m, int* hist,
                                       gemm_tune t)
    {
        __shared__ int sh[kHashClasses];
        if(threadIdx.x < kHashClasses)
            sh[threadIdx.x] = 0;
        __syncthreads();
        for(int64_t base = blockIdx.x * (int64_t)blockDim.x; base < m;
            base += (int64_t)gridDim.x * blockDim.x)
        {
            const int64_t i = base + threadIdx.x;
            int           c = -1;
            if(i < m)
                c = gemm_class(phase, upper[i], rp ? rp[i + 1] - rp[i] : 0, t);
            warp_append(sh, c, kHashClasses);
        }
        __syncthreads();
        if(threadIdx.x < kHashClasses && sh[threadIdx.x])
            atomicAdd(&hist[threadIdx.x], sh[threadIdx.x]);
    }

    __global__ void k_gemm_class_fill(int phase, const int32_t* __restrict__ upper,
                                      const int32_t* __restrict__ rp, int64_t m, int* cursor,
                                      int32_t* rows, gemm_tune t)
    {
        for(int64_t base = blockIdx.x * (int64_t)blockDim.x; base < m;
            base += (int64_t)gridDim.x * blockDim.x)
        {
            const int64_t i = base + threadIdx.x;
            int           c = -1;
            if(i < m)
                c = gemm_class(phase, upper[i], rp ? rp[i + 1] - rp[i] : 0, t);
            const int p = warp_append(cursor, c, kHashClasses);
            if(c >= 0)
                rows[p] = (int32_t)i;
        }
    }

    // Rows grouped by class: rows[start[c] .. start[c + 1]).
    struct gemm_classes
    {
        dbuf<int32_t> rows;
        int           start[kHashClasses + 1] = {};
        int           count(int c) const
        {
            return start[c + 1] - start[c];
        }
        const int32_t* of(int c) const
        {
            return rows.get() + start[c];
        }
    };

    // Classification in two halves around a synchronisation the caller makes
    // anyway: the count kernel and an asynchronous copy of the histogram into
    // pinned host memory, then (after the sync) the class starts and the fill.
    static lab_status gemm_class_count(int phase, const int32_t* upper, const int32_t* rp,
                                       int64_t m, int* dev_hist, int* host_hist, cudaStream_t s,
                                       gemm_tune t)
    {
        LAB_CUDA(cudaMemsetAsync(dev_hist, 0, sizeof(int) * kHashClasses, s));
        const unsigned grid = (unsigned)std::min<int64_t>(ceil_div<int64_t>(m, 256), 4096);
        LAB_LAUNCH(k_gemm_class_count, grid, 256, 0, s, phase, upper, rp, m, dev_hist, t);
        LAB_CUDA(cudaMemcpyAsync(host_hist, dev_hist, sizeof(int) * kHashClasses,
                                 cudaMemcpyDeviceToHost, s));
        return LAB_OK;
    }

    static lab_status gemm_class_fill(int phase, const int32_t* upper, const int32_t* rp,
                                      int64_t m, const int* host_hist, int* dev_start,
                                      gemm_classes& g, cudaStream_t s, gemm_tune t)
    {
        for(int c = 0; c < kHashClasses; c++)
            g.start[c + 1] = g.start[c] + host_hist[c];
        LAB_CUDA(cudaMemcpyAsync(dev_start, g.start, sizeof(int) * kHashClasses,
                                 cudaMemcpyHostToDevice, s));
        LAB_TRY(g.rows.alloc((size_t)m + 1, s));
        const unsigned grid = (unsigned)std::min<int64_t>(ceil_div<int64_t>(m, 256), 4096);
        LAB_LAUNCH(k_gemm_class_fill, grid, 256, 0, s, phase, upper, rp, m, dev_start,
                   g.rows.get(), t);
        return LAB_OK;
    }

    // Small pinned host buffer of this thread for the asynchronous copies above.
    static int* gemm_pinned()
    {
        static thread_local int* p = nullptr;
        if(!p && cudaMallocHost(&p, 64 * sizeof(int)) != cudaSuccess)
        {
            cudaGetLastError();
            p = nullptr;
        }
        return p;
    }

    template <int MODE, int HS, int WARPS>
    static lab_status launch_hash_cls(csr_ref Ar, csr_ref Br, const int32_t* rows, int n,
                                      int32_t* counts, const int32_t* out_rp, int32_t* out_ci,
                                      double* out_v, int32_t* ovf_rows, int* n_ovf, cudaStream_t s,
                                      const int* n_dev = nullptr)
    {
        if(n == 0)
            return LAB_OK;
        constexpr size_t smem = sizeof(hash_smem<MODE, HS>) * WARPS;
        static_assert(smem <= 227 * 1024, "hash table class exceeds shared memory");
        static const cudaError_t attr = cudaFuncSetAttribute(
            k_hash_gemm<MODE, HS, WARPS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        LAB_CUDA(attr);
        static int occ = -1;
        if(occ < 0)
        {
            int o = 0;
            LAB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                &o, k_hash_gemm<MODE, HS, WARPS>, 32 * WARPS, smem));
            occ = std::max(o, 1);
        }
        const unsigned grid = (unsigned)std::min<int64_t>(ceil_div<int64_t>(n, WARPS),
                                                          (int64_t)num_sms() * occ);
        LAB_LAUNCH((k_hash_gemm<MODE, HS, WARPS>), grid, 32 * WARPS, smem, s, Ar, Br, rows, n,
                   counts, out_rp, out_ci, out_v, ovf_rows, n_ovf, n_dev);
        return LAB_OK;
    }

    // One launch per non-empty hash class (1..6) of the phase.
    template <int MODE>
    static lab_status launch_hash_classes(const gemm_classes& g, csr_ref Ar, csr_ref Br,
                                          int32_t* counts, const int32_t* out_rp, int32_t* out_ci,
                                          double* out_v, int32_t* ovf_rows, int* n_ovf,
                                          stream_fork& f)
    {
        // the classes are independent row sets: they run side by side
#define LAB_HASH_CLS(C, HS, W)                                                                    \
    if(g.count(C))                                                                                \
        LAB_TRY((launch_hash_cls<MODE, HS, W>(Ar, Br, g.of(C), g.count(C), counts, out_rp, out_ci,\
                                              out_v, ovf_rows, n_ovf, f.next())))
        if constexpr(MODE == 0)
        {
            LAB_HASH_CLS(1, 128, 8);
            LAB_HASH_CLS(2, 256, 8);
            LAB_HASH_CLS(3, 512, 8);
            LAB_HASH_CLS(4, 1024, 8);
        }
        else
        {
            LAB_HASH_CLS(1, 64, 8);
            LAB_HASH_CLS(2, 128, 8);
            LAB_HASH_CLS(3, 256, 8);
            LAB_HASH_CLS(4, 512, 8);
            LAB_HASH_CLS(5, 1024, 4);
            LAB_HASH_CLS(6, 2048, 4);
        }
#undef LAB_HASH_CLS
        return LAB_OK;
    }

    __global__ void k_gsizes(const int32_t* __restrict__ rows, int n, const int32_t* __restrict__ upper,
                             int64_t* sizes)
    {
        int i = blockIdx.x * blockDim.x + threadIdx.x;
        if(i < n)
            sizes[i] = pow2_ceil(upper[rows[i]]);
        if(i == n)
            sizes[n] = 0;
    }

    // An explicit list of rows processed by the global-memory sort tier.
    static lab_status tiers_for_rows(const int32_t* rows, int n, const int32_t* upper,
                                     esc_tiers& t, cudaStream_t s)
    {
        t.nl = t.nw = t.nb = 0;
        t.ng = n;
        if(n == 0)
            return LAB_OK;
        LAB_TRY(t.rows.alloc((size_t)n, s));
        LAB_CUDA(cudaMemcpyAsync(t.rows.get(), rows, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, s));
        LAB_TRY(t.g_offsets.alloc((size_t)n + 1, s));
        LAB_LAUNCH(k_gsizes, (unsigned)ceil_div(n + 1, 256), 256, 0, s, (const int32_t*)t.rows.get(),
                   n, upper, t.g_offsets.get());
        LAB_TRY(scan_i64(t.g_offsets.get(), n + 1, s));
        LAB_TRY(copy_d2h_sync(&t.g_total, t.g_offsets.get() + n, sizeof(int64_t), s));
        LAB_TRY(t.g_keys.alloc((size_t)t.g_total, s));
        LAB_TRY(t.g_vals.alloc((size_t)t.g_total, s));
        return LAB_OK;
    }

    // Lane-tier rows as an ESC tier list.
    static lab_status lane_tiers(const gemm_classes& g, esc_tiers& t, cudaStream_t s)
    {
        t.nl = g.count(0);
        t.nw = t.nb = t.ng = 0;
        if(t.nl == 0)
            return LAB_OK;
        LAB_TRY(t.rows.alloc((size_t)t.nl, s));
        LAB_CUDA(cudaMemcpyAsync(t.rows.get(), g.of(0), sizeof(int32_t) * t.nl,
                                 cudaMemcpyDeviceToDevice, s));
        return LAB_OK;
    }

    lab_status spgemm(const lab_csr_impl* A, const lab_csr_impl* B, lab_csr_impl** C,
                      cudaStream_t s)
    {
        return spgemm_tuned(A, B, C, s, gemm_tune_lookup(A, B));
    }

    lab_status spgemm_tuned(const lab_csr_impl* A, const lab_csr_impl* B, lab_csr_impl** C,
                            cudaStream_t s, gemm_tune tune)
    {
        if(A->n != B->m)
        {
            set_error("spgemm: inner dimensions differ (%lld vs %lld)", (long long)A->n,
                      (long long)B->m);
            return LAB_BAD_ARG;
        }
        dbuf<int32_t> upper;
        dbuf<int>     ovf;
        LAB_TRY(upper.alloc((size_t)A->m + 1, s));
        LAB_TRY(ovf.alloc(1, s));
        LAB_CUDA(cudaMemsetAsync(ovf.get(), 0, sizeof(int), s));
        csr_ref Ar{A->row_ptr, A->col_ind, A->val}, Br{B->row_ptr, B->col_ind, B->val};
        if(A->m > 0 && A->nnz > 12 * A->m)
            LAB_LAUNCH(k_gemm_upper_warp, (unsigned)ceil_div<int64_t>(A->m * 32, 256), 256, 0, s,
                       Ar, B->row_ptr, A->m, upper.get(), ovf.get());
        else if(A->m > 0)
            LAB_LAUNCH(k_gemm_upper, (unsigned)ceil_div<int64_t>(A->m, 256), 256, 0, s, Ar,
                       B->row_ptr, A->m, upper.get(), ovf.get());
        exp_gemm      e{Ar, Br};
        const int64_t m  = A->m;
        int*          hp = gemm_pinned(); // [0] overflow, [1..] phase-0 classes, [16..] phase 1
        if(!hp)
            return LAB_OOM;
        dbuf<int> dh;
        LAB_TRY(dh.alloc(4 * kHashClasses, s));
        if(m > 0)
            LAB_TRY(gemm_class_count(0, upper.get(), nullptr, m, dh.get(), hp + 1, s, tune));
        LAB_CUDA(cudaMemcpyAsync(hp, ovf.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
        LAB_CUDA(cudaStreamSynchronize(s)); // the overflow flag and the class counts
        if(hp[0])
        {
            set_error("spgemm: a row has more than 2^30 intermediate products");
            return LAB_NOT_SUPPORTED;
        }
        if(m == 0)
            return esc_build(e, upper.get(), m, B->n, C, s);

        // ---- symbolic: lane tier (<= 32 products), hash classes, overflow -> global sort
        gemm_classes gs;
        LAB_TRY(gemm_class_fill(0, upper.get(), nullptr, m, hp + 1, dh.get() + kHashClasses, gs, s,
                                tune));
        dbuf<int32_t> counts, ovf_rows, ovf2_rows, rp;
        dbuf<int>     novf_d;
        LAB_TRY(counts.alloc((size_t)m + 1, s));
        LAB_TRY(ovf_rows.alloc((size_t)std::max(gs.count(4), 1), s));
        LAB_TRY(novf_d.alloc(2, s));
        LAB_CUDA(cudaMemsetAsync(novf_d.get(), 0, 2 * sizeof(int), s));
        LAB_CUDA(cudaMemsetAsync(counts.get(), 0, sizeof(int32_t) * (m + 1), s));
        esc_tiers tl;
        LAB_TRY(lane_tiers(gs, tl, s));
        {
            stream_fork f(s, m); // lane tier and hash classes side by side
            LAB_TRY((esc_run<exp_gemm, 0>(e, m, tl, counts.get(), nullptr, nullptr, f.next())));
            LAB_TRY(launch_hash_classes<0>(gs, Ar, Br, counts.get(), nullptr, nullptr, nullptr,
                                           ovf_rows.get(), novf_d.get(), f));
        }
        if(gs.count(4))
        {
            // rows that filled 3/4 of the 1024-slot table get 4096 slots; their number
            // is read on the device (a launch over the list's capacity), so no host
            // round trip.  Rows that fill that one too (rare) are found at the sync
            // below and go to the global sort tier.
            LAB_TRY(ovf2_rows.alloc((size_t)gs.count(4), s));
            LAB_TRY((launch_hash_cls<0, 4096, 4>(Ar, Br, ovf_rows.get(), gs.count(4), counts.get(),
                                                 nullptr, nullptr, nullptr, ovf2_rows.get(),
                                                 novf_d.get() + 1, s, novf_d.get())));
            LAB_CUDA(cudaMemcpyAsync(hp + 32, novf_d.get() + 1, sizeof(int), cudaMemcpyDeviceToHost,
                                     s));
        }
        else
            hp[32] = 0;

        // ---- row pointer and allocation
        LAB_TRY(rp.alloc((size_t)m + 1, s));
        int32_t nnz32 = 0;
        for(int pass = 0; pass < 2; pass++)
        {
            LAB_TRY(counts_to_rowptr(counts.get(), rp.get(), m, nullptr, s));
            // the numeric classes (by exact count) are counted before the one sync
            // that reads the nonzero total (and the 4096-slot overflow count)
            LAB_TRY(gemm_class_count(1, upper.get(), rp.get(), m, dh.get() + 2 * kHashClasses,
                                     hp + 16, s, tune));
            LAB_TRY(copy_d2h_sync(&nnz32, rp.get() + m, sizeof(int32_t), s));
            const int novf2 = hp[32];
            if(pass == 1 || novf2 == 0)
                break;
            // the global sort tier fills in the counts of the rows that overflowed,
            // then the scan runs again
            esc_tiers tg;
            LAB_TRY(tiers_for_rows(ovf2_rows.get(), novf2, upper.get(), tg, s));
            LAB_TRY((esc_run<exp_gemm, 0>(e, m, tg, counts.get(), nullptr, nullptr, s)));
        }
        if(nnz32 < 0)
        {
            set_error("nonzero count exceeds int32 range");
            return LAB_NOT_SUPPORTED;
        }
        const int64_t nnz = nnz32;
        lab_csr_impl* out = nullptr;
        LAB_TRY(csr_alloc(&out, m, B->n, nnz, s));
        lab_status st = LAB_OK;
        if(cudaMemcpyAsync(out->row_ptr, rp.get(), sizeof(int32_t) * (m + 1),
                           cudaMemcpyDeviceToDevice, s) != cudaSuccess)
            st = LAB_CUDA_ERROR;

        // ---- numeric: lane tier, hash classes by exact count, > 1024 columns -> sort
        exp_gemm e2 = e;
        e2.out_rp   = out->row_ptr;
        gemm_classes gn;
        if(st == LAB_OK)
            st = gemm_class_fill(1, upper.get(), rp.get(), m, hp + 16, dh.get() + 3 * kHashClasses,
                                 gn, s, tune);
        if(st == LAB_OK)
        {
            stream_fork f(s, m); // lane tier and hash classes side by side
            st = esc_run<exp_gemm, 1>(e2, m, tl, nullptr, out->col_ind, out->val, f.next());
            if(st == LAB_OK)
                st = launch_hash_classes<1>(gn, Ar, Br, nullptr, out->row_ptr, out->col_ind,
                                            out->val, nullptr, nullptr, f);
        }
        if(st == LAB_OK && gn.count(7))
        {
            esc_tiers tg;
            st = tiers_for_rows(gn.of(7), gn.count(7), upper.get(), tg, s);
            if(st == LAB_OK)
                st = esc_run<exp_gemm, 1>(e2, m, tg, nullptr, out->col_ind, out->val, s);
        }
        if(st != LAB_OK)
        {
            csr_release(out);
            return st;
        }
        *C = out;
        return LAB_OK;
    }

    lab_status spgeam(double alpha, const lab_csr_impl* A, double beta, const lab_csr_impl* B,
                      lab_csr_impl** C, cudaStream_t s)
    {
        if(A->m != B->m || A->n != B->n)
        {
            set_error("spgeam: shapes differ");
            return LAB_BAD_ARG;
        }
        dbuf<int32_t> upper;
        LAB_TRY(upper.alloc((size_t)A->m + 1, s));
        if(A->m > 0)
            LAB_LAUNCH(k_geam_upper, (unsigned)ceil_div<int64_t>(A->m, 256), 256, 0, s,
                       A->row_ptr, B->row_ptr, A->m, upper.get());
        exp_geam e{csr_ref{A->row_ptr, A->col_ind, A->val}, csr_ref{B->row_ptr, B->col_ind, B->val},
                   alpha, beta};
        return esc_build(e, upper.get(), A->m, A->n, C, s);
    }
}

using namespace lab;

extern "C" {

LAB_API lab_status lab_spgemm(lab_csr A, lab_csr B, lab_csr* C, lab_stream s)
{
    LAB_ARG(A && B && C, "null argument");
    LAB_TRY(ensure_init());
    lab_csr_impl* out = nullptr;
    LAB_TRY(spgemm(A, B, &out, to_stream(s)));
    *C = static_cast<lab_csr>(out);
    return LAB_OK;
}

LAB_API lab_status lab_spgeam(double alpha, lab_csr A, double beta, lab_csr B, lab_csr* C,
                              lab_stream s)
{
    LAB_ARG(A && B && C, "null argument");
    LAB_TRY(ensure_init());
    lab_csr_impl* out = nullptr;
    LAB_TRY(spgeam(alpha, A, beta, B, &out, to_stream(s)));
    *C = static_cast<lab_csr>(out);
    return LAB_OK;
}

LAB_API lab_status lab_transpose(lab_csr A, lab_csr* T, lab_stream s)
{
    LAB_ARG(A && T, "null argument");
    LAB_TRY(ensure_init());
    lab_csr_impl* out = nullptr;
    LAB_TRY(transpose(A, &out, to_stream(s)));
    *T = static_cast<lab_csr>(out);
    return LAB_OK;
}

} // extern "C"
