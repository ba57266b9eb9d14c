// SpGEMM, SpGEAM and transpose on the ESC engine (esc.cuh), plus the tier
// classification shared with the AMG prolongation builders.
#include "esc.cuh"

namespace lab
{
    // ------------------------------------------------------------ tiers
    __global__ void k_tier_count(const int32_t* __restrict__ upper, int64_t m, int* cnt)
    {
        __shared__ int s[3];
        if(threadIdx.x < 3)
            s[threadIdx.x] = 0;
        __syncthreads();
        for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m;
            i += (int64_t)gridDim.x * blockDim.x)
        {
            int u = upper[i];
            atomicAdd(&s[u <= kEscWarpCap ? 0 : (u <= kEscCtaCap ? 1 : 2)], 1);
        }
        __syncthreads();
        if(threadIdx.x < 3 && s[threadIdx.x])
            atomicAdd(&cnt[threadIdx.x], s[threadIdx.x]);
    }

    __global__ void k_tier_fill(const int32_t* __restrict__ upper, int64_t m, int* cursor,
                                int32_t* rows, int64_t* gsize)
    {
        for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m;
            i += (int64_t)gridDim.x * blockDim.x)
        {
            int u = upper[i];
            int t = u <= kEscWarpCap ? 0 : (u <= kEscCtaCap ? 1 : 2);
            int p = atomicAdd(&cursor[t], 1);
            rows[p] = (int32_t)i;
            if(t == 2)
                gsize[p - cursor[5]] = pow2_ceil(u);
        }
    }

    lab_status esc_classify(const int32_t* upper, int64_t m, esc_tiers& t, cudaStream_t s)
    {
        t.nw = t.nb = t.ng = 0;
        if(m == 0)
            return LAB_OK;
        dbuf<int> cnt;
        LAB_TRY(cnt.alloc(8, s));
        LAB_CUDA(cudaMemsetAsync(cnt.get(), 0, sizeof(int) * 8, s));
        unsigned grid = (unsigned)std::min<int64_t>(ceil_div<int64_t>(m, 256), 4096);
        LAB_LAUNCH(k_tier_count, grid, 256, 0, s, upper, m, cnt.get());
        int h[3];
        LAB_TRY(copy_d2h_sync(h, cnt.get(), sizeof(int) * 3, s));
        t.nw = h[0];
        t.nb = h[1];
        t.ng = h[2];
        // cursors: [0]=W start, [1]=B start, [2]=G start, [5]=G start (for gsize index)
        int cur[8] = {0, t.nw, t.nw + t.nb, 0, 0, t.nw + t.nb, 0, 0};
        LAB_CUDA(cudaMemcpyAsync(cnt.get(), cur, sizeof(cur), cudaMemcpyHostToDevice, s));
        LAB_TRY(t.rows.alloc((size_t)m, s));
        LAB_TRY(t.g_offsets.alloc((size_t)std::max(t.ng, 1) + 1, s));
        LAB_LAUNCH(k_tier_fill, grid, 256, 0, s, upper, m, cnt.get(), t.rows.get(),
                   t.g_offsets.get());
        LAB_CUDA(cudaStreamSynchronize(s)); // cur[] lives on the host stack
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
    // For rows with many products but few distinct columns (the Galerkin products
    // R*(A*P) and A*P on coarse levels: up to ~12k products, <= ~300 columns).
    // One warp per row.  The warp walks the A row in order; for each entry the
    // lanes take the distinct columns of the matching B row, so no two lanes ever
    // touch the same table key within a step, and a __syncwarp separates steps:
    // every column's contributions are added in A-row order, the first one
    // assigned, exactly as host_csrgemm.cpp:119-139.  Only the distinct columns
    // are then sorted.
    constexpr int kHashWarps = 4;
    constexpr int kHashSym   = 2048; // symbolic table slots per warp (keys only)
    constexpr int kHashNum   = 1024; // numeric table slots per warp
    constexpr int kHashNumMaxCnt = kHashNum / 2;

    __device__ __forceinline__ unsigned hash_slot(int c, unsigned mask)
    {
        return ((unsigned)c * 2654435761u >> 7) & mask;
    }

    // mode 0: symbolic (counts[row], or the row goes to the overflow list)
    template <int MODE>
    __global__ void __launch_bounds__(32 * kHashWarps)
        k_hash_gemm(csr_ref A, csr_ref B, const int32_t* __restrict__ rows, int nrows,
                    int32_t* counts, const int32_t* __restrict__ out_rp, int32_t* out_ci,
                    double* out_v, int32_t* ovf_rows, int* n_ovf)
    {
        extern __shared__ __align__(16) unsigned char hsm[];
        const int      wid  = threadIdx.x >> 5;
        const int      lane = threadIdx.x & 31;
        constexpr int  H    = MODE == 0 ? kHashSym : kHashNum;
        const size_t   per  = MODE == 0 ? (size_t)H * 4 : (size_t)H * 4 + (size_t)H * 8 + (size_t)(H / 2) * 8;
        unsigned char* base = hsm + per * wid;
        int*           skey = reinterpret_cast<int*>(base);
        double*        sval = reinterpret_cast<double*>(base + (size_t)H * 4);
        uint64_t*      sk   = reinterpret_cast<uint64_t*>(base + (size_t)H * 12);
        __shared__ int s_claims[kHashWarps];

        for(int r = blockIdx.x * kHashWarps + wid; r < nrows; r += gridDim.x * kHashWarps)
        {
            const int row = rows[r];
            int       cnt = 0;
            unsigned  Hr  = H;
            if(MODE == 1)
            {
                cnt = out_rp[row + 1] - out_rp[row];
                Hr  = (unsigned)max(32, pow2_ceil(2 * cnt));
            }
            const unsigned mask = Hr - 1;
            for(unsigned q = lane; q < Hr; q += 32)
                skey[q] = -1;
            if(lane == 0)
                s_claims[wid] = 0;
            __syncwarp();
            bool ovf = false;
            for(int j = A.rp[row]; j < A.rp[row + 1] && !ovf; j++)
            {
                const int    k  = A.ci[j];
                const double a  = A.v[j];
                const int    b0 = B.rp[k], b1 = B.rp[k + 1];
                for(int p = b0 + lane; p < b1; p += 32)
                {
                    const int c    = B.ci[p];
                    unsigned  slot = hash_slot(c, mask);
                    for(unsigned probe = 0; probe < Hr; probe++)
                    {
                        int old = atomicCAS(&skey[slot], -1, c);
                        if(old == -1)
                        {
                            if(MODE == 1)
                                sval[slot] = __dmul_rn(a, B.v[p]);
                            else
                                atomicAdd(&s_claims[wid], 1);
                            break;
                        }
                        if(old == c)
                        {
                            if(MODE == 1)
                                sval[slot] = __dadd_rn(sval[slot], __dmul_rn(a, B.v[p]));
                            break;
                        }
                        slot = (slot + 1) & mask;
                    }
                }
                __syncwarp();
                if(MODE == 0 && s_claims[wid] > (int)(3 * H / 4))
                    ovf = true; // too many distinct columns for this table
                __syncwarp();
            }
            if(MODE == 0)
            {
                if(lane == 0)
                {
                    if(ovf)
                        ovf_rows[atomicAdd(n_ovf, 1)] = row;
                    else
                        counts[row] = s_claims[wid];
                }
            }
            else
            {
                // compact the filled slots, sort by column, write
                int n = 0;
                for(unsigned q0 = 0; q0 < Hr; q0 += 32)
                {
                    unsigned q    = q0 + lane;
                    bool     full = skey[q] >= 0;
                    unsigned bal  = __ballot_sync(0xffffffffu, full);
                    if(full)
                        sk[n + __popc(bal & ((1u << lane) - 1u))] = make_key(skey[q], (int)q);
                    n += __popc(bal);
                }
                __syncwarp();
                bitonic_sort<grp_warp>(sk, n);
                const int32_t o = out_rp[row];
                for(int i = lane; i < n; i += 32)
                {
                    out_ci[o + i] = key_col(sk[i]);
                    out_v[o + i]  = sval[key_pos(sk[i])];
                }
            }
            __syncwarp();
        }
    }

    // Split row ids by item count: rows with ub <= 256 to `small`, others to `big`.
    __global__ void k_split_rows(const int32_t* __restrict__ upper, int64_t m, int32_t* small,
                                 int32_t* big, int* cnt)
    {
        for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m;
            i += (int64_t)gridDim.x * blockDim.x)
        {
            if(upper[i] <= kEscWarpCap)
                small[atomicAdd(&cnt[0], 1)] = (int32_t)i;
            else
                big[atomicAdd(&cnt[1], 1)] = (int32_t)i;
        }
    }

    // Numeric routing of the big rows: exact count <= kHashNumMaxCnt -> hash, else sort.
    __global__ void k_split_numeric(const int32_t* __restrict__ big, int nbig,
                                    const int32_t* __restrict__ rp, int32_t* hash_rows,
                                    int32_t* sort_rows, int* cnt)
    {
        for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < nbig; i += gridDim.x * blockDim.x)
        {
            int row = big[i];
            if(rp[row + 1] - rp[row] <= kHashNumMaxCnt)
                hash_rows[atomicAdd(&cnt[0], 1)] = row;
            else
                sort_rows[atomicAdd(&cnt[1], 1)] = row;
        }
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
        t.nw = t.nb = 0;
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

    template <int MODE>
    static lab_status launch_hash(csr_ref Ar, csr_ref Br, const int32_t* rows, int n,
                                  int32_t* counts, const int32_t* out_rp, int32_t* out_ci,
                                  double* out_v, int32_t* ovf_rows, int* n_ovf, cudaStream_t s)
    {
        if(n == 0)
            return LAB_OK;
        const size_t per  = MODE == 0 ? (size_t)kHashSym * 4
                                      : (size_t)kHashNum * 12 + (size_t)(kHashNum / 2) * 8;
        const size_t smem = per * kHashWarps;
        static const cudaError_t attr = cudaFuncSetAttribute(
            k_hash_gemm<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        LAB_CUDA(attr);
        unsigned grid = (unsigned)std::min<int64_t>(ceil_div<int64_t>(n, kHashWarps),
                                                    (int64_t)num_sms() * 8);
        LAB_LAUNCH(k_hash_gemm<MODE>, grid, 32 * kHashWarps, smem, s, Ar, Br, rows, n, counts,
                   out_rp, out_ci, out_v, ovf_rows, n_ovf);
        return LAB_OK;
    }

    lab_status spgemm(const lab_csr_impl* A, const lab_csr_impl* B, lab_csr_impl** C,
                      cudaStream_t s)
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
        if(A->m > 0)
            LAB_LAUNCH(k_gemm_upper, (unsigned)ceil_div<int64_t>(A->m, 256), 256, 0, s, Ar,
                       B->row_ptr, A->m, upper.get(), ovf.get());
        int h = 0;
        LAB_TRY(copy_d2h_sync(&h, ovf.get(), sizeof(int), s));
        if(h)
        {
            set_error("spgemm: a row has more than 2^30 intermediate products");
            return LAB_NOT_SUPPORTED;
        }
        exp_gemm      e{Ar, Br};
        const int64_t m = A->m;
        if(m == 0)
            return esc_build(e, upper.get(), m, B->n, C, s);

        // ---- tiers: <= 256 products: warp sort; more: warp hash; hash overflow: global sort
        dbuf<int32_t> small, big, counts, ovf_rows, rp;
        dbuf<int>     cnt;
        LAB_TRY(small.alloc((size_t)m, s));
        LAB_TRY(big.alloc((size_t)m, s));
        LAB_TRY(counts.alloc((size_t)m + 1, s));
        LAB_TRY(ovf_rows.alloc((size_t)m, s));
        LAB_TRY(cnt.alloc(8, s));
        LAB_CUDA(cudaMemsetAsync(cnt.get(), 0, sizeof(int) * 8, s));
        LAB_CUDA(cudaMemsetAsync(counts.get(), 0, sizeof(int32_t) * (m + 1), s));
        unsigned g = (unsigned)std::min<int64_t>(ceil_div<int64_t>(m, 256), 4096);
        LAB_LAUNCH(k_split_rows, g, 256, 0, s, (const int32_t*)upper.get(), m, small.get(),
                   big.get(), cnt.get());
        int hc[2];
        LAB_TRY(copy_d2h_sync(hc, cnt.get(), sizeof(int) * 2, s));
        const int nsmall = hc[0], nbig = hc[1];

        esc_tiers ts;
        ts.nw = nsmall;
        if(nsmall)
        {
            LAB_TRY(ts.rows.alloc((size_t)nsmall, s));
            LAB_CUDA(cudaMemcpyAsync(ts.rows.get(), small.get(), sizeof(int32_t) * nsmall,
                                     cudaMemcpyDeviceToDevice, s));
        }
        LAB_TRY((esc_run<exp_gemm, 0>(e, m, ts, counts.get(), nullptr, nullptr, s)));
        LAB_TRY(launch_hash<0>(Ar, Br, big.get(), nbig, counts.get(), nullptr, nullptr, nullptr,
                               ovf_rows.get(), cnt.get() + 2, s));
        int novf = 0;
        LAB_TRY(copy_d2h_sync(&novf, cnt.get() + 2, sizeof(int), s));
        if(novf)
        {
            esc_tiers tg;
            LAB_TRY(tiers_for_rows(ovf_rows.get(), novf, upper.get(), tg, s));
            LAB_TRY((esc_run<exp_gemm, 0>(e, m, tg, counts.get(), nullptr, nullptr, s)));
        }

        // ---- row pointer and allocation
        LAB_TRY(rp.alloc((size_t)m + 1, s));
        int64_t nnz = 0;
        LAB_TRY(counts_to_rowptr(counts.get(), rp.get(), m, &nnz, s));
        lab_csr_impl* out = nullptr;
        LAB_TRY(csr_alloc(&out, m, B->n, nnz, s));
        lab_status st = LAB_OK;
        if(cudaMemcpyAsync(out->row_ptr, rp.get(), sizeof(int32_t) * (m + 1),
                           cudaMemcpyDeviceToDevice, s) != cudaSuccess)
            st = LAB_CUDA_ERROR;

        // ---- numeric
        exp_gemm e2 = e;
        e2.out_rp   = out->row_ptr;
        if(st == LAB_OK)
            st = esc_run<exp_gemm, 1>(e2, m, ts, nullptr, out->col_ind, out->val, s);
        dbuf<int32_t> hrows, srows;
        if(st == LAB_OK && nbig)
        {
            st = hrows.alloc((size_t)nbig, s);
            if(st == LAB_OK)
                st = srows.alloc((size_t)nbig, s);
            if(st == LAB_OK)
            {
                cudaMemsetAsync(cnt.get() + 4, 0, sizeof(int) * 2, s);
                k_split_numeric<<<(unsigned)ceil_div(nbig, 256), 256, 0, s>>>(
                    big.get(), nbig, out->row_ptr, hrows.get(), srows.get(), cnt.get() + 4);
                g_launches.fetch_add(1);
                int hn[2] = {0, 0};
                st = copy_d2h_sync(hn, cnt.get() + 4, sizeof(int) * 2, s);
                if(st == LAB_OK)
                    st = launch_hash<1>(Ar, Br, hrows.get(), hn[0], nullptr, out->row_ptr,
                                        out->col_ind, out->val, nullptr, nullptr, s);
                if(st == LAB_OK && hn[1])
                {
                    esc_tiers tg;
                    st = tiers_for_rows(srows.get(), hn[1], upper.get(), tg, s);
                    if(st == LAB_OK)
                        st = esc_run<exp_gemm, 1>(e2, m, tg, nullptr, out->col_ind, out->val, s);
                }
            }
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
