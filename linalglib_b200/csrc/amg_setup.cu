// AMG setup on the device: strength of connection, PMIS aggregation, SA / UA
// prolongation, RS C/F splitting and direct interpolation, and the level loop.
// Integer outputs and every floating-point value of P and A_c are bit-identical
// to the reference host implementation (see the per-kernel citations).
#include "amg.cuh"
#include "esc.cuh"

#include <cfloat>
#include <chrono>

namespace lab
{
    // ------------------------------------------------------------ strength
    // host_amg_strength.cpp:33-70:
    //   conn[j] = (c != i) && |a_ij| >= eps * sqrt(|d_i| * |d_c|)
    template <int LANES>
    __global__ void k_strength(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                               const double* __restrict__ v, const double* __restrict__ d,
                               int64_t m, double eps, int32_t* __restrict__ conn)
    {
        int64_t t    = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
        int64_t i    = t / LANES;
        int     lane = (int)(t % LANES);
        if(i >= m)
            return;
        const double di = fabs(d[i]);
        for(int j = rp[i] + lane; j < rp[i + 1]; j += LANES)
        {
            const int    c   = ci[j];
            const double thr = __dmul_rn(eps, __dsqrt_rn(__dmul_rn(di, fabs(d[c]))));
            conn[j]          = (c != i) && (fabs(v[j]) >= thr);
        }
    }

    lab_status amg_strength(const lab_csr_impl* A, double eps, int32_t* conn, cudaStream_t s)
    {
        if(A->m == 0)
            return LAB_OK;
        dbuf<double> d;
        LAB_TRY(d.alloc((size_t)A->m, s));
        LAB_TRY(diag_into(A, d.get(), nullptr, s));
        double avg = (double)A->nnz / (double)A->m;
        if(avg <= 12.0)
            LAB_LAUNCH(k_strength<1>, (unsigned)ceil_div<int64_t>(A->m, 256), 256, 0, s,
                       A->row_ptr, A->col_ind, A->val, d.get(), A->m, eps, conn);
        else
            LAB_LAUNCH(k_strength<32>, (unsigned)ceil_div<int64_t>(A->m * 32, 256), 256, 0, s,
                       A->row_ptr, A->col_ind, A->val, d.get(), A->m, eps, conn);
        return LAB_OK;
    }

    // ------------------------------------------------------------ PMIS
    // host_amg_aggregation.cpp:32-38
    __device__ __forceinline__ unsigned int pmis_hash(unsigned int x)
    {
        x = ((x >> 16) ^ x) * 0x45d9f3bu;
        x = ((x >> 16) ^ x) * 0x45d9f3bu;
        x = (x >> 16) ^ x;
        return x / 2u;
    }

    // host_amg_aggregation.cpp:40-68
    __global__ void k_pmis_init(const int32_t* __restrict__ rp, const int32_t* __restrict__ conn,
                                int64_t m, int32_t* __restrict__ state, int32_t* __restrict__ hash,
                                int64_t* __restrict__ agg)
    {
        int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
        if(i >= m)
            return;
        int s = -2;
        for(int j = rp[i]; j < rp[i + 1]; j++)
            if(!conn || conn[j] == 1)
            {
                s = 0;
                break;
            }
        state[i] = s;
        hash[i]  = (int32_t)pmis_hash((unsigned int)i);
        agg[i]   = 0;
    }

    // k_pmis_init with a warp per row (long rows): any strong entry makes the
    // state 0 (the reference stops at the first one; the result is the same).
    __global__ void k_pmis_init_warp(const int32_t* __restrict__ rp,
                                     const int32_t* __restrict__ conn, int64_t m,
                                     int32_t* __restrict__ state, int32_t* __restrict__ hash,
                                     int64_t* __restrict__ agg)
    {
        const int64_t i    = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
        const int     lane = threadIdx.x & 31;
        if(i >= m)
            return;
        bool strong = false;
        for(int j = rp[i] + lane; j < rp[i + 1] && !strong; j += 32)
            strong = !conn || conn[j] == 1;
        strong = __any_sync(0xffffffffu, strong);
        if(lane != 0)
            return;
        state[i] = strong ? 0 : -2;
        hash[i]  = (int32_t)pmis_hash((unsigned int)i);
        agg[i]   = 0;
    }

    // One round of host_find_maximum_distance_two_node (host_amg_aggregation.cpp:95-180).
    // Reads the round's snapshot `st`, writes the row's new state to `out` (the
    // other buffer of a ping-pong pair; unchanged rows are copied through) and
    // agg for its own row only, so the parallel round equals the sequential one.
    // The lexicographic maximum replaces the running winner only on a strictly
    // larger (state, hash), so the CSR scan order decides ties exactly as in the
    // reference (lines 77-93).
    // Rounds after the first complete one return at once (amg_aggregation.cpp:154).
    __device__ __forceinline__ void pmis_round_row(int64_t i, const int32_t* __restrict__ rp,
                                                   const int32_t* __restrict__ ci,
                                                   const int32_t* __restrict__ conn,
                                                   const int32_t* __restrict__ st,
                                                   const int32_t* __restrict__ hash,
                                                   int32_t* __restrict__ out,
                                                   int64_t* __restrict__ agg, int32_t* flags,
                                                   int round)
    {
        if(st[i] != 0)
        {
            // decided rows keep their state; their scans would change nothing
            out[i] = st[i];
            return;
        }
        int bs = st[i], bh = hash[i], br = (int)i;
        for(int j = rp[i]; j < rp[i + 1]; j++)
        {
            if(conn && conn[j] != 1)
                continue;
            int c = ci[j], cs = st[c], chh = hash[c];
            if(cs > bs || (cs == bs && chh > bh))
            {
                bs = cs;
                bh = chh;
                br = c;
            }
        }
        const int r = br;
        for(int j = rp[r]; j < rp[r + 1]; j++)
        {
            if(conn && conn[j] != 1)
                continue;
            int c = ci[j], cs = st[c], chh = hash[c];
            if(cs > bs || (cs == bs && chh > bh))
            {
                bs = cs;
                bh = chh;
                br = c;
            }
        }
        int ns = st[i];
        if(ns == 0)
        {
            if(br == i)
            {
                ns     = 1;
                agg[i] = 1;
            }
            else if(bs == 1)
            {
                ns     = -1;
                agg[i] = 0;
            }
            else
                flags[round] = 1;
        }
        out[i] = ns;
    }

    // Persistent grid (grid-stride): the 20 round launches are made unconditionally
    // and the ones after convergence must cost next to nothing.
    __global__ void k_pmis_round(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                 const int32_t* __restrict__ conn, int64_t m,
                                 const int32_t* __restrict__ st, const int32_t* __restrict__ hash,
                                 int32_t* __restrict__ out, int64_t* __restrict__ agg,
                                 int32_t* flags, int round)
    {
        if(round > 0 && flags[round - 1] == 0)
            return;
        for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m;
            i += (int64_t)gridDim.x * blockDim.x)
            pmis_round_row(i, rp, ci, conn, st, hash, out, agg, flags, round);
    }

    // Warp-per-row form of k_pmis_round for long rows (coarse levels).  The
    // sequential scan keeps the first (state, hash) maximum it meets, so its result
    // is the lexicographic maximum of (state, hash, -scan position) over the start
    // value (position -1) and the strong neighbours; lanes take strided positions
    // and a shuffle reduction picks that maximum: the same winner as the scan.
    struct pmis_best
    {
        int s, h, pos, node;
    };
    __device__ __forceinline__ bool pmis_better(const pmis_best& a, const pmis_best& b)
    {
        if(a.s != b.s)
            return a.s > b.s;
        if(a.h != b.h)
            return a.h > b.h;
        return a.pos < b.pos;
    }
    __device__ __forceinline__ pmis_best pmis_warp_max(pmis_best v)
    {
#pragma unroll
        for(int o = 16; o > 0; o >>= 1)
        {
            pmis_best w;
            w.s    = __shfl_xor_sync(0xffffffffu, v.s, o);
            w.h    = __shfl_xor_sync(0xffffffffu, v.h, o);
            w.pos  = __shfl_xor_sync(0xffffffffu, v.pos, o);
            w.node = __shfl_xor_sync(0xffffffffu, v.node, o);
            if(pmis_better(w, v))
                v = w;
        }
        return v;
    }
    // best over {start} and the strong neighbours of row r (positions in CSR order)
    __device__ __forceinline__ pmis_best pmis_scan_warp(const int32_t* __restrict__ rp,
                                                        const int32_t* __restrict__ ci,
                                                        const int32_t* __restrict__ conn,
                                                        const int32_t* __restrict__ st,
                                                        const int32_t* __restrict__ hash, int r,
                                                        pmis_best start, int lane)
    {
        pmis_best v = start;
        const int a = rp[r], b = rp[r + 1];
        for(int j = a + lane; j < b; j += 32)
        {
            if(conn && conn[j] != 1)
                continue;
            const int c = ci[j];
            pmis_best w{st[c], hash[c], j - a, c};
            if(pmis_better(w, v))
                v = w;
        }
        return pmis_warp_max(v);
    }

    __device__ __forceinline__ void pmis_round_row_warp(
        int64_t i, int lane, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
        const int32_t* __restrict__ conn, const int32_t* __restrict__ st,
        const int32_t* __restrict__ hash, int32_t* __restrict__ out, int64_t* __restrict__ agg,
        int32_t* flags, int round)
    {
        if(st[i] != 0)
        {
            if(lane == 0)
                out[i] = st[i];
            return;
        }
        pmis_best v = pmis_scan_warp(rp, ci, conn, st, hash, (int)i,
                                     pmis_best{st[i], hash[i], -1, (int)i}, lane);
        // second scan over the winner's row, starting from the winner (position -1)
        v = pmis_scan_warp(rp, ci, conn, st, hash, v.node, pmis_best{v.s, v.h, -1, v.node}, lane);
        if(lane != 0)
            return;
        int ns = st[i];
        if(ns == 0)
        {
            if(v.node == i)
            {
                ns     = 1;
                agg[i] = 1;
            }
            else if(v.s == 1)
            {
                ns     = -1;
                agg[i] = 0;
            }
            else
                flags[round] = 1;
        }
        out[i] = ns;
    }

    __global__ void k_pmis_round_warp(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                      const int32_t* __restrict__ conn, int64_t m,
                                      const int32_t* __restrict__ st,
                                      const int32_t* __restrict__ hash, int32_t* __restrict__ out,
                                      int64_t* __restrict__ agg, int32_t* flags, int round)
    {
        if(round > 0 && flags[round - 1] == 0)
            return;
        const int lane = threadIdx.x & 31;
        for(int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < m;
            i += ((int64_t)gridDim.x * blockDim.x) >> 5)
            pmis_round_row_warp(i, lane, rp, ci, conn, st, hash, out, agg, flags, round);
    }

    // All rounds in one CTA for small levels (the per-round launches dominate
    // there): round r reads buffer r & 1 and writes the other, as the launches do,
    // and stops after the first round that left no row undecided.
    constexpr int kPmisSmallRows = 4096;

    __global__ void __launch_bounds__(1024)
        k_pmis_rounds_small(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                            const int32_t* __restrict__ conn, int64_t m, int32_t* b0, int32_t* b1,
                            const int32_t* __restrict__ hash, int64_t* __restrict__ agg,
                            int32_t* flags, int wide)
    {
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
        for(int r = 0; r < 20; r++)
        {
            if(r > 0 && flags[r - 1] == 0)
                break;
            const int32_t* st  = (r & 1) ? b1 : b0;
            int32_t*       out = (r & 1) ? b0 : b1;
            if(wide)
                for(int64_t i = wid; i < m; i += nw)
                    pmis_round_row_warp(i, lane, rp, ci, conn, st, hash, out, agg, flags, r);
            else
                for(int64_t i = threadIdx.x; i < m; i += blockDim.x)
                    pmis_round_row(i, rp, ci, conn, st, hash, out, agg, flags, r);
            __syncthreads();
        }
    }

    // Rounds that ran: round r runs iff r == 0 or round r-1 left a row undecided.
    __device__ __forceinline__ int pmis_rounds_run(const int32_t* flags)
    {
        int k = 1;
        while(k < 20 && flags[k - 1] != 0)
            k++;
        return k;
    }

    // host_add_unassigned_nodes_to_closest_aggregation (host_amg_aggregation.cpp:182-221),
    // pass k of 2.  The rounds left the state in buffer (K & 1) of the pair
    // {b0, b1} (K = rounds run); pass k reads buffer (K + k) & 1 and writes the other.
    __global__ void k_pmis_attach(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                  const int32_t* __restrict__ conn, int64_t m, int32_t* b0,
                                  int32_t* b1, const int32_t* __restrict__ flags, int k,
                                  int64_t* __restrict__ agg)
    {
        int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
        if(i >= m)
            return;
        const int      sel = (pmis_rounds_run(flags) + k) & 1;
        const int32_t* st  = sel ? b1 : b0;
        int32_t*       out = sel ? b0 : b1;
        int            s   = st[i];
        if(s == -1)
        {
            for(int j = rp[i]; j < rp[i + 1]; j++)
            {
                if((!conn || conn[j] == 1) && st[ci[j]] == 1)
                {
                    agg[i] = agg[ci[j]];
                    s      = 1;
                    break;
                }
            }
        }
        else if(s == -2)
            agg[i] = -2;
        out[i] = s;
    }

    // Warp-per-row form of k_pmis_attach for long rows: the first strong neighbour
    // in CSR order whose state is 1 (ballot per 32-entry chunk, lowest lane first).
    __global__ void k_pmis_attach_warp(const int32_t* __restrict__ rp,
                                       const int32_t* __restrict__ ci,
                                       const int32_t* __restrict__ conn, int64_t m, int32_t* b0,
                                       int32_t* b1, const int32_t* __restrict__ flags, int k,
                                       int64_t* __restrict__ agg)
    {
        const int64_t i    = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
        const int     lane = threadIdx.x & 31;
        if(i >= m)
            return;
        const int      sel = (pmis_rounds_run(flags) + k) & 1;
        const int32_t* st  = sel ? b1 : b0;
        int32_t*       out = sel ? b0 : b1;
        int            s   = st[i];
        if(s == -1)
        {
            const int a = rp[i], b = rp[i + 1];
            for(int base = a; base < b; base += 32)
            {
                const int      j   = base + lane;
                const bool     hit = j < b && (!conn || conn[j] == 1) && st[ci[j]] == 1;
                const unsigned bal = __ballot_sync(0xffffffffu, hit);
                if(bal)
                {
                    const int first = base + __ffs(bal) - 1;
                    if(lane == 0)
                        agg[i] = agg[ci[first]];
                    s = 1;
                    break;
                }
            }
        }
        else if(s == -2 && lane == 0)
            agg[i] = -2;
        if(lane == 0)
            out[i] = s;
    }

    __global__ void k_count_rounds(const int32_t* flags, int* out)
    {
        int r = 0;
        while(r < 20 && flags[r] != 0)
            r++;
        *out = r;
    }

    // amg_aggregation.cpp:168-177: roots are the nodes marked 1 before the scan
    __global__ void k_pmis_roots(const int64_t* __restrict__ agg, int64_t m, int64_t* roots)
    {
        int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
        if(i < m)
            roots[i] = agg[i] == 1 ? 1 : -1;
    }

    // Strong-neighbour lists of long rows (coarse SA levels keep only 10-20 % of
    // their entries strong): the PMIS passes then scan the strong columns alone,
    // in CSR order (the scans' tie rules depend on that order only).
    __global__ void k_strong_count(const int32_t* __restrict__ rp,
                                   const int32_t* __restrict__ conn, int64_t m,
                                   int32_t* __restrict__ cnt)
    {
        const int64_t i    = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
        const int     lane = threadIdx.x & 31;
        if(i >= m)
            return;
        int c = 0;
        for(int j = rp[i] + lane; j < rp[i + 1]; j += 32)
            c += conn[j] == 1;
#pragma unroll
        for(int o = 16; o > 0; o >>= 1)
            c += __shfl_xor_sync(0xffffffffu, c, o);
        if(lane == 0)
            cnt[i] = c;
    }

    __global__ void k_strong_fill(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                  const int32_t* __restrict__ conn, int64_t m,
                                  const int32_t* __restrict__ srp, int32_t* __restrict__ sci)
    {
        const int64_t i    = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
        const int     lane = threadIdx.x & 31;
        if(i >= m)
            return;
        int o = srp[i];
        for(int base = rp[i]; base < rp[i + 1]; base += 32)
        {
            const int      j   = base + lane;
            const bool     st  = j < rp[i + 1] && conn[j] == 1;
            const unsigned bal = __ballot_sync(0xffffffffu, st);
            if(st)
                sci[o + __popc(bal & ((1u << lane) - 1u))] = ci[j];
            o += __popc(bal);
        }
    }

    // compute_aggregates_using_pmis (amg_aggregation.cpp:106-215)
    lab_status amg_pmis(const lab_csr_impl* A, const int32_t* conn, int64_t* agg, int* rounds,
                        cudaStream_t s, int64_t* roots = nullptr)
    {
        const int64_t m = A->m;
        if(m == 0)
        {
            if(rounds)
                *rounds = 0;
            return LAB_OK;
        }
        // the passes read (prp, pci, pconn): A with its conn flags, or, for long
        // rows, the strong-neighbour lists (pconn = null: every entry strong)
        const int32_t* prp   = A->row_ptr;
        const int32_t* pci   = A->col_ind;
        const int32_t* pconn = conn;
        int64_t        pnnz  = A->nnz;
        dbuf<int32_t>  srp, sci;
        if(conn && A->nnz > 12 * m)
        {
            const unsigned gw = (unsigned)ceil_div<int64_t>(m * 32, 256);
            LAB_TRY(srp.alloc((size_t)m + 1, s));
            LAB_TRY(sci.alloc((size_t)std::max<int64_t>(A->nnz, 1), s));
            LAB_LAUNCH(k_strong_count, gw, 256, 0, s, A->row_ptr, conn, m, srp.get());
            LAB_TRY(counts_to_rowptr(srp.get(), srp.get(), m, &pnnz, s));
            LAB_LAUNCH(k_strong_fill, gw, 256, 0, s, A->row_ptr, A->col_ind, conn, m,
                       (const int32_t*)srp.get(), sci.get());
            prp   = srp.get();
            pci   = sci.get();
            pconn = nullptr;
        }
        dbuf<int32_t> state, snap, hash, flags;
        LAB_TRY(state.alloc((size_t)m, s));
        LAB_TRY(snap.alloc((size_t)m, s));
        LAB_TRY(hash.alloc((size_t)m, s));
        LAB_TRY(flags.alloc(24, s));
        LAB_CUDA(cudaMemsetAsync(flags.get(), 0, sizeof(int32_t) * 24, s));
        const unsigned g = (unsigned)ceil_div<int64_t>(m, 256);
        const bool     wide = pnnz > 12 * m;
        const unsigned gw   = (unsigned)ceil_div<int64_t>(m * 32, 256);
        if(wide)
            LAB_LAUNCH(k_pmis_init_warp, gw, 256, 0, s, prp, pconn, m, state.get(),
                       hash.get(), agg);
        else
            LAB_LAUNCH(k_pmis_init, g, 256, 0, s, prp, pconn, m, state.get(), hash.get(),
                       agg);
        // ping-pong: round r reads buffer r & 1 of {state, snap} and writes the other
        int32_t* buf[2] = {state.get(), snap.get()};
        // long rows (coarse levels): a warp per row
        if(m <= kPmisSmallRows)
            LAB_LAUNCH(k_pmis_rounds_small, 1, 1024, 0, s, prp, pci, pconn, m, buf[0], buf[1],
                       (const int32_t*)hash.get(), agg, flags.get(), (int)wide);
        else
        {
            for(int r = 0; r < 20; r++)
            {
                if(wide)
                    LAB_LAUNCH(k_pmis_round_warp, std::min<unsigned>(gw, num_sms() * 8), 256, 0,
                               s, prp, pci, pconn, m, (const int32_t*)buf[r & 1], hash.get(),
                               buf[(r + 1) & 1], agg, flags.get(), r);
                else
                    LAB_LAUNCH(k_pmis_round, std::min<unsigned>(g, num_sms() * 8), 256, 0, s, prp,
                               pci, pconn, m, (const int32_t*)buf[r & 1], hash.get(),
                               buf[(r + 1) & 1], agg, flags.get(), r);
            }
        }
        if(rounds)
        {
            dbuf<int> d;
            LAB_TRY(d.alloc(1, s));
            LAB_LAUNCH(k_count_rounds, 1, 1, 0, s, flags.get(), d.get());
            LAB_TRY(copy_d2h_sync(rounds, d.get(), sizeof(int), s));
        }
        if(roots)
            LAB_LAUNCH(k_pmis_roots, g, 256, 0, s, (const int64_t*)agg, m, roots);
        LAB_TRY(scan_i64(agg, m, s));
        for(int k = 0; k < 2; k++)
        {
            if(wide)
                LAB_LAUNCH(k_pmis_attach_warp, gw, 256, 0, s, prp, pci, pconn, m,
                           state.get(), snap.get(), (const int32_t*)flags.get(), k, agg);
            else
                LAB_LAUNCH(k_pmis_attach, g, 256, 0, s, prp, pci, pconn, m,
                           state.get(), snap.get(), (const int32_t*)flags.get(), k, agg);
        }
        return LAB_OK;
    }

    // ------------------------------------------------------------ SA prolongation
    // construct_prolongation_using_smoothed_aggregation (saamg.cpp:51-207).
    // Items of row i, in CSR order: every diagonal or strong entry whose column
    // has an aggregate >= 0, keyed by that aggregate, valued
    //   1 - relax                      (diagonal)
    //   (-relax * (1 / dtilde)) * a_ij  (strong), dtilde = a_ii - sum_weak a_ij
    // summed per aggregate in CSR order (std::map accumulation, lines 177-187).
    struct exp_sap
    {
        const int32_t* rp;
        const int32_t* ci;
        const double*  v;
        const int32_t* conn;
        const int64_t* agg;
        double         relax;
        const int32_t* out_rp = nullptr;

        template <class G>
        __device__ int expand(int row, uint64_t* keys, double* vals) const
        {
            __shared__ int s_pref[32];
            const int      a0 = rp[row], a1 = rp[row + 1];
            // saamg.cpp:145-163: the diagonal plus the weak entries' negated values,
            // summed in CSR order.  A warp loads 32 entries at once and every lane
            // runs the same ordered chain over the contributing ones (shuffles);
            // larger groups sum sequentially (every thread computes it).
            double dg = 0.0;
            if constexpr(G::size == 32)
            {
                const unsigned full = 0xffffffffu;
                const int      lane = G::rank();
                for(int base = a0; base < a1; base += 32)
                {
                    const int j    = base + lane;
                    double    t    = 0.0;
                    bool      add  = false, sub = false;
                    if(j < a1)
                    {
                        const int c = ci[j];
                        add         = c == row;
                        sub         = !add && conn[j] == 0;
                        if(add || sub)
                            t = v[j];
                    }
                    unsigned       mask = __ballot_sync(full, add || sub);
                    const unsigned subs = __ballot_sync(full, sub);
                    while(mask)
                    {
                        const int    l = __ffs(mask) - 1;
                        const double x = __shfl_sync(full, t, l);
                        dg             = ((subs >> l) & 1u) ? __dsub_rn(dg, x) : __dadd_rn(dg, x);
                        mask &= mask - 1u;
                    }
                }
            }
            else
            {
                for(int j = a0; j < a1; j++)
                {
                    if(ci[j] == row)
                        dg = __dadd_rn(dg, v[j]);
                    else if(conn[j] == 0)
                        dg = __dsub_rn(dg, v[j]);
                }
            }
            const double inv  = __ddiv_rn(1.0, dg);
            const double coef = __dmul_rn(-relax, inv);
            const double dval = __dsub_rn(1.0, relax);
            int          n    = 0;
            for(int base = a0; base < a1; base += G::size)
            {
                int  j  = base + G::rank();
                bool q  = false;
                int  c  = 0;
                int64_t ag = -1;
                if(j < a1)
                {
                    c = ci[j];
                    if(c == row || conn[j] == 1)
                    {
                        ag = agg[c];
                        q  = ag >= 0;
                    }
                }
                int tot;
                int pos = n + group_prefix<G>(q, s_pref, tot);
                if(q)
                {
                    keys[pos] = make_key((int)ag, pos);
                    vals[pos] = (c == row) ? dval : __dmul_rn(coef, v[j]);
                }
                n += tot;
            }
            G::sync();
            return n;
        }
        template <bool VALS, class F>
        __device__ void emit_seq(int row, F&& f) const
        {
            const int a0 = rp[row], a1 = rp[row + 1];
            double    coef = 0.0, dval = 0.0;
            if(VALS)
            {
                double dg = 0.0;
                for(int j = a0; j < a1; j++)
                {
                    if(ci[j] == row)
                        dg = __dadd_rn(dg, v[j]);
                    else if(conn[j] == 0)
                        dg = __dsub_rn(dg, v[j]);
                }
                coef = __dmul_rn(-relax, __ddiv_rn(1.0, dg));
                dval = __dsub_rn(1.0, relax);
            }
            for(int j = a0; j < a1; j++)
            {
                const int c = ci[j];
                if(c != row && conn[j] != 1)
                    continue;
                const int64_t ag = agg[c];
                if(ag >= 0)
                    f((int)ag, VALS ? ((c == row) ? dval : __dmul_rn(coef, v[j])) : 0.0);
            }
        }
        __device__ int32_t out_start(int row) const
        {
            return out_rp[row];
        }
    };

    // Long rows (coarse levels): one warp per row computes the row's diagonal-plus-
    // weak sum (saamg.cpp:145-163, in CSR order, as exp_sap::expand) and compacts
    // the candidate entries (the diagonal and the strong ones, in CSR order) to the
    // front of the row's slot range, so the expansion then walks ~10 candidates
    // instead of the whole row.
    __global__ void k_sap_prep(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                               const double* __restrict__ v, const int32_t* __restrict__ conn,
                               int64_t m, int32_t* __restrict__ sci, double* __restrict__ sv,
                               int32_t* __restrict__ cnt, double* __restrict__ dgs)
    {
        const int64_t  i    = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
        const int      lane = threadIdx.x & 31;
        const unsigned full = 0xffffffffu;
        if(i >= m)
            return;
        const int a0 = rp[i], a1 = rp[i + 1];
        double    dg = 0.0;
        int       o  = a0;
        for(int base = a0; base < a1; base += 32)
        {
            const int j    = base + lane;
            int       c    = -1, cn = 0;
            double    x    = 0.0;
            if(j < a1)
            {
                c  = ci[j];
                cn = conn[j];
                x  = v[j];
            }
            const bool     add  = j < a1 && c == i;
            const bool     sub  = j < a1 && !add && cn == 0;
            const bool     cand = j < a1 && (add || cn == 1);
            unsigned       mask = __ballot_sync(full, add || sub);
            const unsigned subs = __ballot_sync(full, sub);
            while(mask)
            {
                const int    l = __ffs(mask) - 1;
                const double t = __shfl_sync(full, x, l);
                dg             = ((subs >> l) & 1u) ? __dsub_rn(dg, t) : __dadd_rn(dg, t);
                mask &= mask - 1u;
            }
            const unsigned cb = __ballot_sync(full, cand);
            if(cand)
            {
                const int q = o + __popc(cb & ((1u << lane) - 1u));
                sci[q]      = c;
                sv[q]       = x;
            }
            o += __popc(cb);
        }
        if(lane == 0)
        {
            cnt[i] = o - a0;
            dgs[i] = dg;
        }
    }

    // exp_sap over the compacted candidates of k_sap_prep (row r: slots
    // rp[r] .. rp[r] + cnt[r]) with the precomputed diagonal sums.
    struct exp_sap_c
    {
        const int32_t* rp;
        const int32_t* cnt;
        const int32_t* ci;
        const double*  v;
        const double*  dgs;
        const int64_t* agg;
        double         relax;
        const int32_t* out_rp = nullptr;

        template <class G>
        __device__ int expand(int row, uint64_t* keys, double* vals) const
        {
            __shared__ int s_pref[32];
            const int      a0   = rp[row], a1 = a0 + cnt[row];
            const double   coef = __dmul_rn(-relax, __ddiv_rn(1.0, dgs[row]));
            const double   dval = __dsub_rn(1.0, relax);
            int            n    = 0;
            for(int base = a0; base < a1; base += G::size)
            {
                const int j  = base + G::rank();
                bool      q  = false;
                int       c  = 0;
                int64_t   ag = -1;
                if(j < a1)
                {
                    c  = ci[j];
                    ag = agg[c];
                    q  = ag >= 0;
                }
                int tot;
                int pos = n + group_prefix<G>(q, s_pref, tot);
                if(q)
                {
                    keys[pos] = make_key((int)ag, pos);
                    vals[pos] = (c == row) ? dval : __dmul_rn(coef, v[j]);
                }
                n += tot;
            }
            G::sync();
            return n;
        }
        template <bool VALS, class F>
        __device__ void emit_seq(int row, F&& f) const
        {
            const int    a0   = rp[row], a1 = a0 + cnt[row];
            const double coef = VALS ? __dmul_rn(-relax, __ddiv_rn(1.0, dgs[row])) : 0.0;
            const double dval = __dsub_rn(1.0, relax);
            for(int j = a0; j < a1; j++)
            {
                const int     c  = ci[j];
                const int64_t ag = agg[c];
                if(ag >= 0)
                    f((int)ag, VALS ? ((c == row) ? dval : __dmul_rn(coef, v[j])) : 0.0);
            }
        }
        __device__ int32_t out_start(int row) const
        {
            return out_rp[row];
        }
    };

    lab_status amg_sa_prolongation(const lab_csr_impl* A, const int32_t* conn, const int64_t* agg,
                                   double relax, lab_csr_impl** P, cudaStream_t s)
    {
        // n_c = max aggregate + 1 (saamg.cpp:68-76): the maximum travels to pinned
        // memory asynchronously and is read at esc_build's first synchronisation
        int64_t* hp = pinned_small();
        if(!hp)
            return LAB_OOM;
        hp[0] = -1;
        if(A->m > 0)
            LAB_TRY(max_i64_async(agg, A->m, hp, s));
        const std::function<int64_t()> nc_late = [hp] { return (hp[0] > -1 ? hp[0] : -1) + 1; };
        if(A->m > 0 && A->nnz > 12 * A->m)
        {
            dbuf<int32_t> cnt, sci;
            dbuf<double>  sv, dgs;
            LAB_TRY(cnt.alloc((size_t)A->m + 1, s));
            LAB_TRY(sci.alloc((size_t)A->nnz, s));
            LAB_TRY(sv.alloc((size_t)A->nnz, s));
            LAB_TRY(dgs.alloc((size_t)A->m, s));
            LAB_LAUNCH(k_sap_prep, (unsigned)ceil_div<int64_t>(A->m * 32, 256), 256, 0, s,
                       A->row_ptr, A->col_ind, (const double*)A->val, conn, A->m, sci.get(),
                       sv.get(), cnt.get(), dgs.get());
            exp_sap_c e{A->row_ptr, cnt.get(), sci.get(), sv.get(), dgs.get(), agg, relax};
            return esc_build(e, cnt.get(), A->m, 0, P, s, nc_late);
        }
        dbuf<int32_t> upper;
        LAB_TRY(upper.alloc((size_t)A->m + 1, s));
        LAB_TRY(row_lengths(A->row_ptr, A->m, upper.get(), s));
        exp_sap e{A->row_ptr, A->col_ind, A->val, conn, agg, relax};
        return esc_build(e, upper.get(), A->m, 0, P, s, nc_late);
    }

    // ------------------------------------------------------------ UA prolongation
    __global__ void k_ua_count(const int64_t* __restrict__ agg, int64_t m, int32_t* cnt)
    {
        int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
        if(i < m)
            cnt[i] = agg[i] >= 0 ? 1 : 0;
    }

    __global__ void k_ua_fill(const int64_t* __restrict__ agg, int64_t m,
                              const int32_t* __restrict__ rp, int32_t* ci, double* v)
    {
        int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
        if(i < m && agg[i] >= 0)
        {
            ci[rp[i]] = (int32_t)agg[i];
            v[rp[i]]  = 1.0;
        }
    }

    // construct_prolongation_using_unsmoothed_aggregation (uaamg.cpp:49-128)
    lab_status amg_ua_prolongation(const lab_csr_impl* A, const int64_t* agg, lab_csr_impl** P,
                                   cudaStream_t s)
    {
        const int64_t m  = A->m;
        int64_t       mx = -1;
        if(m > 0)
            LAB_TRY(max_i64(agg, m, &mx, s));
        int64_t       nc = (mx > -1 ? mx : -1) + 1;
        dbuf<int32_t> cnt, rp;
        LAB_TRY(cnt.alloc((size_t)m + 1, s));
        LAB_TRY(rp.alloc((size_t)m + 1, s));
        if(m > 0)
            LAB_LAUNCH(k_ua_count, (unsigned)ceil_div<int64_t>(m, 256), 256, 0, s, agg, m, cnt.get());
        int64_t nnz = 0;
        LAB_TRY(counts_to_rowptr(cnt.get(), rp.get(), m, &nnz, s));
        lab_csr_impl* out = nullptr;
        LAB_TRY(csr_alloc(&out, m, nc, nnz, s));
        LAB_CUDA(cudaMemcpyAsync(out->row_ptr, rp.get(), sizeof(int32_t) * (m + 1),
                                 cudaMemcpyDeviceToDevice, s));
        if(m > 0)
            LAB_LAUNCH(k_ua_fill, (unsigned)ceil_div<int64_t>(m, 256), 256, 0, s, agg, m,
                       out->row_ptr, out->col_ind, out->val);
        *P = out;
        return LAB_OK;
    }

    // ------------------------------------------------------------ RS strength
    // host_amg_strength.cpp:72-156
    __global__ void k_classical_strength(const int32_t* __restrict__ rp,
                                         const int32_t* __restrict__ ci,
                                         const double* __restrict__ v, int64_t m, double theta,
                                         int32_t* __restrict__ conn, int32_t* __restrict__ cnt)
    {
        int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
        if(i >= m)
            return;
        double mx = -DBL_MAX;
        for(int j = rp[i]; j < rp[i + 1]; j++)
            if(ci[j] != i)
                mx = (mx < -v[j]) ? -v[j] : mx; // std::max(mx, -a_ij)
        const double thr = __dmul_rn(theta, mx);
        int          c   = 0;
        for(int j = rp[i]; j < rp[i + 1]; j++)
        {
            int str = (-v[j] >= thr && ci[j] != i);
            conn[j] = str;
            c += str;
        }
        cnt[i] = c;
    }

    __global__ void k_fill_s(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                             const double* __restrict__ v, const int32_t* __restrict__ conn,
                             int64_t m, const int32_t* __restrict__ srp, int32_t* sci, double* sv)
    {
        int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
        if(i >= m)
            return;
        int p = srp[i];
        for(int j = rp[i]; j < rp[i + 1]; j++)
            if(conn[j] == 1)
            {
                sci[p] = ci[j];
                sv[p]  = v[j];
                p++;
            }
    }

    lab_status amg_classical_strength(const lab_csr_impl* A, double theta, int32_t* conn,
                                      lab_csr_impl** S, cudaStream_t s)
    {
        const int64_t m = A->m;
        dbuf<int32_t> cnt, rp;
        LAB_TRY(cnt.alloc((size_t)m + 1, s));
        LAB_TRY(rp.alloc((size_t)m + 1, s));
        if(m > 0)
            LAB_LAUNCH(k_classical_strength, (unsigned)ceil_div<int64_t>(m, 256), 256, 0, s,
                       A->row_ptr, A->col_ind, A->val, m, theta, conn, cnt.get());
        int64_t nnz = 0;
        LAB_TRY(counts_to_rowptr(cnt.get(), rp.get(), m, &nnz, s));
        lab_csr_impl* out = nullptr;
        LAB_TRY(csr_alloc(&out, m, A->n, nnz, s));
        LAB_CUDA(cudaMemcpyAsync(out->row_ptr, rp.get(), sizeof(int32_t) * (m + 1),
                                 cudaMemcpyDeviceToDevice, s));
        if(m > 0)
            LAB_LAUNCH(k_fill_s, (unsigned)ceil_div<int64_t>(m, 256), 256, 0, s, A->row_ptr,
                       A->col_ind, A->val, conn, m, out->row_ptr, out->col_ind, out->val);
        *S = out;
        return LAB_OK;
    }

    // ------------------------------------------------------------ RS C/F splitting
    // host_compute_cfpoint_first_pass / second_pass (host_amg_aggregation.cpp:228-519).
    // The greedy bucket algorithm is inherently sequential (each choice reorders
    // the buckets the next choice reads), so it runs as one device thread over
    // L2-resident arrays; it is bit-exact by construction.
    constexpr uint32_t kF = 0, kC = 1, kU = 2, kFF = 3;

    __global__ void k_cf_first_pass(const int32_t* __restrict__ srp, const int32_t* __restrict__ sci,
                                    const int32_t* __restrict__ trp, const int32_t* __restrict__ tci,
                                    int m, uint32_t* cf, int* lambda, int* ptr, int* count,
                                    int* i2n, int* n2i, int first, int second)
    {
        if(threadIdx.x != 0 || blockIdx.x != 0)
            return;
        if(!first)
            goto second_pass;
        for(int i = 0; i <= m; i++)
        {
            ptr[i]   = 0;
            count[i] = 0;
        }
        ptr[m + 1] = 0;
        for(int i = 0; i < m; i++)
        {
            cf[i]     = kU;
            lambda[i] = trp[i + 1] - trp[i];
        }
        for(int i = 0; i < m; i++)
            ptr[lambda[i] + 1]++;
        for(int i = 0; i < m; i++)
            ptr[i + 1] += ptr[i];
        for(int i = 0; i < m; i++)
        {
            int lam    = lambda[i];
            int idx    = ptr[lam] + count[lam];
            i2n[idx]   = i;
            n2i[i]     = idx;
            count[lam] = count[lam] + 1;
        }
        for(int i = m - 1; i >= 0; i--)
        {
            int node = i2n[i];
            if(lambda[node] <= 0)
                break;
            if(cf[node] != kU)
                continue;
            cf[node] = kC;
            for(int j = trp[node]; j < trp[node + 1]; j++)
                if(cf[tci[j]] == kU)
                    cf[tci[j]] = kFF;
            for(int j = trp[node]; j < trp[node + 1]; j++)
            {
                int f = tci[j];
                if(cf[f] != kFF)
                    continue;
                cf[f] = kF;
                for(int k = srp[f]; k < srp[f + 1]; k++)
                {
                    int u = sci[k];
                    if(cf[u] != kU)
                        continue;
                    int lu = lambda[u], op = n2i[u], np = ptr[lu] + count[lu] - 1;
                    n2i[i2n[op]] = np;
                    n2i[i2n[np]] = op;
                    int t        = i2n[op];
                    i2n[op]      = i2n[np];
                    i2n[np]      = t;
                    count[lu]--;
                    count[lu + 1]++;
                    ptr[lu + 1] = ptr[lu] + count[lu];
                    lambda[u]++;
                }
            }
            for(int j = srp[node]; j < srp[node + 1]; j++)
            {
                int u = sci[j];
                if(cf[u] != kU || lambda[u] <= 0)
                    continue;
                int lu = lambda[u], op = n2i[u], np = ptr[lu];
                n2i[i2n[op]] = np;
                n2i[i2n[np]] = op;
                int t        = i2n[op];
                i2n[op]      = i2n[np];
                i2n[np]      = t;
                count[lu]--;
                count[lu - 1]++;
                ptr[lu]++;
                lambda[u]--;
            }
        }
        for(int i = 0; i < m; i++)
            if(cf[i] == kU)
                cf[i] = kF;
    second_pass:
        if(!second)
            return;
        for(int i = 0; i < m; i++)
        {
            if(cf[i] != kF)
                continue;
            int s0 = srp[i], s1 = srp[i + 1], cand = -1;
            for(int j = s0; j < s1; j++)
            {
                int c = sci[j];
                if(cf[c] != kF)
                    continue;
                int  a = s0, b = srp[c], be = srp[c + 1];
                bool found = false;
                while(a < s1 && b < be)
                {
                    int c1 = sci[a], c2 = sci[b];
                    if(c1 < c2)
                        a++;
                    else if(c2 < c1)
                        b++;
                    else
                    {
                        a++;
                        b++;
                        if(cf[c1] == kC)
                        {
                            found = true;
                            break;
                        }
                    }
                }
                if(!found)
                {
                    if(cand >= 0)
                        cf[cand] = kF;
                    cand  = c;
                    cf[c] = kC;
                }
            }
        }
    }

    lab_status amg_cfpoints(const lab_csr_impl* S, uint32_t* cf, cudaStream_t s, int first,
                            int second)
    {
        const int64_t m = S->m;
        if(m == 0)
            return LAB_OK;
        lab_csr_impl* ST = nullptr;
        LAB_TRY(transpose(S, &ST, s));
        dbuf<int> lambda, ptr, count, i2n, n2i;
        lab_status st = lambda.alloc((size_t)m + 2, s);
        if(st == LAB_OK)
            st = ptr.alloc((size_t)m + 2, s);
        if(st == LAB_OK)
            st = count.alloc((size_t)m + 2, s);
        if(st == LAB_OK)
            st = i2n.alloc((size_t)m + 1, s);
        if(st == LAB_OK)
            st = n2i.alloc((size_t)m + 1, s);
        if(st == LAB_OK)
        {
            k_cf_first_pass<<<1, 1, 0, s>>>(S->row_ptr, S->col_ind, ST->row_ptr, ST->col_ind,
                                            (int)m, cf, lambda.get(), ptr.get(), count.get(),
                                            i2n.get(), n2i.get(), first, second);
            g_launches.fetch_add(1);
            cudaError_t e = cudaGetLastError();
            if(e != cudaSuccess)
                st = cuda_status(e, "k_cf_first_pass", __FILE__, __LINE__);
        }
        csr_release(ST);
        return st;
    }

    // ------------------------------------------------------------ RS direct interpolation
    __global__ void k_di_count(const int32_t* __restrict__ srp, const int32_t* __restrict__ sci,
                               const uint32_t* __restrict__ cf, int64_t m, int32_t* cnt,
                               int32_t* cflag)
    {
        int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
        if(i >= m)
            return;
        cflag[i] = (int32_t)cf[i];
        if(cf[i] == kC)
        {
            cnt[i] = 1;
            return;
        }
        int c = 0;
        for(int j = srp[i]; j < srp[i + 1]; j++)
            c += cf[sci[j]] == kC;
        cnt[i] = c;
    }

    // rsamg.cpp:765-865, including the index quirk at line 818 (A's column array
    // read at S positions).
    __global__ void k_di_fill(const int32_t* __restrict__ arp, const int32_t* __restrict__ aci,
                              const double* __restrict__ av, const int32_t* __restrict__ srp,
                              const int32_t* __restrict__ sci, const double* __restrict__ sv,
                              const uint32_t* __restrict__ cf, const int32_t* __restrict__ cidx,
                              int64_t m, const int32_t* __restrict__ prp, int32_t* pci, double* pv)
    {
        int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
        if(i >= m)
            return;
        int p = prp[i];
        if(cf[i] == kC)
        {
            pci[p] = cidx[i];
            pv[p]  = 1.0;
            return;
        }
        double dg = 0.0, pos = 0.0, neg = 0.0;
        for(int j = arp[i]; j < arp[i + 1]; j++)
        {
            if(aci[j] == i)
                dg = av[j];
            else if(av[j] < 0.0)
                neg = __dadd_rn(neg, av[j]);
            else
                pos = __dadd_rn(pos, av[j]);
        }
        double spos = 0.0, sneg = 0.0;
        for(int j = srp[i]; j < srp[i + 1]; j++)
        {
            if(cf[aci[j]] == kC)
            {
                if(sv[j] < 0.0)
                    sneg = __dadd_rn(sneg, sv[j]);
                else
                    spos = __dadd_rn(spos, sv[j]);
            }
        }
        const double alpha = __ddiv_rn(neg, sneg);
        const double beta  = __ddiv_rn(pos, spos);
        for(int j = srp[i]; j < srp[i + 1]; j++)
        {
            int c = sci[j];
            if(cf[c] != kC)
                continue;
            pci[p] = cidx[c];
            pv[p]  = sv[j] < 0.0 ? __ddiv_rn(__dmul_rn(-alpha, sv[j]), dg)
                                 : __ddiv_rn(__dmul_rn(-beta, sv[j]), dg);
            p++;
        }
    }

    lab_status amg_direct_interpolation(const lab_csr_impl* A, const lab_csr_impl* S,
                                        const uint32_t* cf, lab_csr_impl** P, cudaStream_t s)
    {
        const int64_t m = A->m;
        dbuf<int32_t> cnt, rp, cidx;
        LAB_TRY(cnt.alloc((size_t)m + 1, s));
        LAB_TRY(rp.alloc((size_t)m + 1, s));
        LAB_TRY(cidx.alloc((size_t)m + 1, s));
        if(m > 0)
            LAB_LAUNCH(k_di_count, (unsigned)ceil_div<int64_t>(m, 256), 256, 0, s, S->row_ptr,
                       S->col_ind, cf, m, cnt.get(), cidx.get());
        int64_t nc = 0;
        // cidx = exclusive scan of the C flags; total = number of C points
        LAB_TRY(counts_to_rowptr(cidx.get(), cidx.get(), m, &nc, s));
        int64_t nnz = 0;
        LAB_TRY(counts_to_rowptr(cnt.get(), rp.get(), m, &nnz, s));
        lab_csr_impl* out = nullptr;
        LAB_TRY(csr_alloc(&out, m, nc, nnz, s));
        LAB_CUDA(cudaMemcpyAsync(out->row_ptr, rp.get(), sizeof(int32_t) * (m + 1),
                                 cudaMemcpyDeviceToDevice, s));
        if(m > 0)
            LAB_LAUNCH(k_di_fill, (unsigned)ceil_div<int64_t>(m, 256), 256, 0, s, A->row_ptr,
                       A->col_ind, A->val, S->row_ptr, S->col_ind, S->val, cf, cidx.get(), m,
                       out->row_ptr, out->col_ind, out->val);
        *P = out;
        return LAB_OK;
    }

    // ------------------------------------------------------------ level loop
    lab_status hierarchy_release(hierarchy_impl* h)
    {
        if(!h)
            return LAB_OK;
        cudaDeviceSynchronize();
        solver_cache_forget(h);
        for(int l = 0; l <= kMaxLevels; l++)
        {
            if(h->A[l])
                csr_release(h->A[l]);
            level_ws& w = h->ws[l];
            void*     ptrs[] = {w.x,  w.b,  w.r,  w.t,  w.xf, w.bf, w.rf,
                                w.tf, w.xk, w.bk, w.rk, w.tk, w.colour};
            for(void* p : ptrs)
                if(p)
                    cudaFree(p);
            delete[] w.colour_ptr_h;
        }
        for(int l = 0; l < kMaxLevels; l++)
        {
            if(h->P[l])
                csr_release(h->P[l]);
            if(h->R[l])
                csr_release(h->R[l]);
        }
        if(h->coarse_inv)
            cudaFree(h->coarse_inv);
        if(h->coarse_inv32)
            cudaFree(h->coarse_inv32);
        delete static_cast<lab_hier_s*>(h);
        return LAB_OK;
    }

    // saamg_setup (saamg.cpp:210-282), uaamg_setup (uaamg.cpp:131-224),
    // rsamg_setup (rsamg.cpp:869-947)
    // Row schedules of the coarse levels.  Few rows leave little to spread over the
    // GPU, so small levels take more lanes per long row (the autotuner's choice on
    // the SA hierarchies measured), and the smallest ones the plain VECTOR kernel
    // instead of the staged one (whose tile set-up dominates there).  Level 0 keeps
    // the CSR-order schedule of the caller's matrix.  Built and loaded hierarchies
    // both get these plans, so they run identical cycles.
    lab_status hierarchy_plans(hierarchy_impl* h, cudaStream_t s)
    {
        // every level's statistics with one host round trip
        LAB_TRY(spmv_analyse_batch(h->A + 1, h->levels, s));
        for(int l = 1; l <= h->levels; l++)
        {
            lab_csr_impl* Al = h->A[l];
            spmv_plan&    p  = Al->plan;
            if(p.forced || Al->m == 0)
                continue;
            if(Al->m <= 16)
            {
                p.alg   = LAB_SPMV_VECTOR;
                p.lanes = p.max_row > 4 ? 32 : 4;
            }
            else if(Al->m < 1024 && p.alg == LAB_SPMV_VECTOR)
                p.lanes = std::min(32, 2 * p.vlanes);
        }
        return LAB_OK;
    }

    static lab_status amg_setup(int kind, const lab_csr_impl* A0, int max_level,
                                hierarchy_impl* h, cudaStream_t s)
    {
        max_level = std::min(max_level, kMaxLevels);
        h->kind   = kind;
        LAB_TRY(csr_alloc(&h->A[0], A0->m, A0->n, A0->nnz, s));
        LAB_CUDA(cudaMemcpyAsync(h->A[0]->row_ptr, A0->row_ptr, sizeof(int32_t) * (A0->m + 1),
                                 cudaMemcpyDeviceToDevice, s));
        if(A0->nnz)
        {
            LAB_CUDA(cudaMemcpyAsync(h->A[0]->col_ind, A0->col_ind, sizeof(int32_t) * A0->nnz,
                                     cudaMemcpyDeviceToDevice, s));
            LAB_CUDA(cudaMemcpyAsync(h->A[0]->val, A0->val, sizeof(double) * A0->nnz,
                                     cudaMemcpyDeviceToDevice, s));
        }
        double eps   = kind == LAB_AMG_UA ? 0.001 : 0.08;
        double relax = 2.0 / 3.0;
        double theta = 0.2;
        int    level = 0;
        while(level < max_level)
        {
            lab_csr_impl* Af = h->A[level];
            lab_csr_impl* P  = nullptr;
            dbuf<int32_t> conn;
            LAB_TRY(conn.alloc((size_t)std::max<int64_t>(Af->nnz, 1), s));
            if(Af->nnz)
                LAB_CUDA(cudaMemsetAsync(conn.get(), 0, sizeof(int32_t) * Af->nnz, s));
            if(kind == LAB_AMG_RS)
            {
                lab_csr_impl*  S = nullptr;
                dbuf<uint32_t> cf;
                LAB_TRY(cf.alloc((size_t)Af->m + 1, s));
                LAB_TRY(amg_classical_strength(Af, theta, conn.get(), &S, s));
                lab_status st = amg_cfpoints(S, cf.get(), s, 1, 1);
                if(st == LAB_OK)
                    st = amg_direct_interpolation(Af, S, cf.get(), &P, s);
                csr_release(S);
                LAB_TRY(st);
            }
            else
            {
                dbuf<int64_t> agg;
                LAB_TRY(agg.alloc((size_t)Af->m + 1, s));
                LAB_TRY(amg_strength(Af, eps, conn.get(), s));
                LAB_TRY(amg_pmis(Af, conn.get(), agg.get(), nullptr, s, nullptr));
                if(kind == LAB_AMG_SA)
                    LAB_TRY(amg_sa_prolongation(Af, conn.get(), agg.get(), relax, &P, s));
                else
                    LAB_TRY(amg_ua_prolongation(Af, agg.get(), &P, s));
            }
            if(P->n == 0)
            {
                csr_release(P);
                break;
            }
            h->P[level] = P;
            LAB_TRY(transpose(P, &h->R[level], s));
            lab_csr_impl* AP = nullptr;
            LAB_TRY(spgemm(Af, P, &AP, s));
            lab_status st = spgemm(h->R[level], AP, &h->A[level + 1], s);
            csr_release(AP);
            LAB_TRY(st);
            level++;
            eps *= 0.5;
        }
        h->levels = level;
        return hierarchy_plans(h, s);
    }
}

using namespace lab;

extern "C" {

LAB_API lab_status lab_strength(lab_csr A, double eps, int32_t* conn, lab_stream s)
{
    LAB_ARG(A && (conn || A->nnz == 0), "null argument");
    LAB_TRY(ensure_init());
    return amg_strength(A, eps, conn, to_stream(s));
}

LAB_API lab_status lab_classical_strength(lab_csr A, double theta, int32_t* conn, lab_csr* S,
                                          lab_stream s)
{
    LAB_ARG(A && S && (conn || A->nnz == 0), "null argument");
    LAB_TRY(ensure_init());
    lab_csr_impl* out = nullptr;
    LAB_TRY(amg_classical_strength(A, theta, conn, &out, to_stream(s)));
    *S = static_cast<lab_csr>(out);
    return LAB_OK;
}

LAB_API lab_status lab_pmis_aggregate(lab_csr A, const int32_t* conn, int64_t* aggregates,
                                      int* rounds, lab_stream s)
{
    LAB_ARG(A && (aggregates || A->m == 0), "null argument");
    LAB_TRY(ensure_init());
    return amg_pmis(A, conn, aggregates, rounds, to_stream(s), nullptr);
}

LAB_API lab_status lab_sa_prolongation(lab_csr A, const int32_t* conn, const int64_t* aggregates,
                                       double relax, lab_csr* P, lab_stream s)
{
    LAB_ARG(A && P, "null argument");
    LAB_TRY(ensure_init());
    lab_csr_impl* out = nullptr;
    LAB_TRY(amg_sa_prolongation(A, conn, aggregates, relax, &out, to_stream(s)));
    *P = static_cast<lab_csr>(out);
    return LAB_OK;
}

LAB_API lab_status lab_ua_prolongation(lab_csr A, const int64_t* aggregates, lab_csr* P,
                                       lab_stream s)
{
    LAB_ARG(A && P, "null argument");
    LAB_TRY(ensure_init());
    lab_csr_impl* out = nullptr;
    LAB_TRY(amg_ua_prolongation(A, aggregates, &out, to_stream(s)));
    *P = static_cast<lab_csr>(out);
    return LAB_OK;
}

LAB_API lab_status lab_cfpoints(lab_csr S, uint32_t* cf, lab_stream s)
{
    LAB_ARG(S && (cf || S->m == 0), "null argument");
    LAB_ARG(S->m == S->n, "S must be square");
    LAB_TRY(ensure_init());
    return amg_cfpoints(S, cf, to_stream(s), 1, 1);
}

LAB_API lab_status lab_cfpoints_passes(lab_csr S, uint32_t* cf, int first, int second,
                                       lab_stream s)
{
    LAB_ARG(S && (cf || S->m == 0), "null argument");
    LAB_ARG(S->m == S->n, "S must be square");
    LAB_TRY(ensure_init());
    return amg_cfpoints(S, cf, to_stream(s), first, second);
}

LAB_API lab_status lab_pmis_aggregate_roots(lab_csr A, const int32_t* conn, int64_t* aggregates,
                                            int64_t* root_nodes, int* rounds, lab_stream s)
{
    LAB_ARG(A && (aggregates || A->m == 0), "null argument");
    LAB_TRY(ensure_init());
    return amg_pmis(A, conn, aggregates, rounds, to_stream(s), root_nodes);
}

LAB_API lab_status lab_direct_interpolation(lab_csr A, lab_csr S, const uint32_t* cf,
                                            lab_csr* P, lab_stream s)
{
    LAB_ARG(A && S && P, "null argument");
    LAB_TRY(ensure_init());
    lab_csr_impl* out = nullptr;
    LAB_TRY(amg_direct_interpolation(A, S, cf, &out, to_stream(s)));
    *P = static_cast<lab_csr>(out);
    return LAB_OK;
}

LAB_API lab_status lab_amg_setup(lab_amg_kind kind, lab_csr A, int max_level, lab_hierarchy* out,
                                 lab_stream ls)
{
    LAB_ARG(A && out, "null argument");
    LAB_ARG(kind == LAB_AMG_SA || kind == LAB_AMG_UA || kind == LAB_AMG_RS, "unknown AMG kind");
    LAB_ARG(A->m == A->n, "AMG needs a square matrix");
    LAB_ARG(max_level >= 0, "negative max_level");
    LAB_TRY(ensure_init());
    cudaStream_t s = to_stream(ls);
    lab_hier_s*  h = new(std::nothrow) lab_hier_s();
    if(!h)
        return LAB_OOM;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
    lab_status st = amg_setup(kind, A, max_level, h, s);
    cudaEventRecord(e1, s);
    if(st == LAB_OK)
    {
        cudaError_t e = cudaEventSynchronize(e1);
        if(e != cudaSuccess)
            st = cuda_status(e, "lab_amg_setup", __FILE__, __LINE__);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        h->setup_ms = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if(st != LAB_OK)
    {
        hierarchy_release(h);
        return st;
    }
    *out = h;
    return LAB_OK;
}

LAB_API lab_status lab_hierarchy_destroy(lab_hierarchy h)
{
    return hierarchy_release(h);
}

LAB_API lab_status lab_hierarchy_levels(lab_hierarchy h, int* n)
{
    LAB_ARG(h && n, "null argument");
    *n = h->levels;
    return LAB_OK;
}

LAB_API lab_status lab_hierarchy_level(lab_hierarchy h, int l, lab_csr* A, lab_csr* P, lab_csr* R)
{
    LAB_ARG(h, "null hierarchy");
    LAB_ARG(l >= 0 && l <= h->levels, "level out of range");
    LAB_ARG(l < h->levels || (!P && !R), "no P/R on the coarsest level");
    if(A)
        *A = static_cast<lab_csr>(h->A[l]);
    if(P)
        *P = static_cast<lab_csr>(h->P[l]);
    if(R)
        *R = static_cast<lab_csr>(h->R[l]);
    return LAB_OK;
}

LAB_API lab_status lab_hierarchy_setup_ms(lab_hierarchy h, double* ms)
{
    LAB_ARG(h && ms, "null argument");
    *ms = h->setup_ms;
    return LAB_OK;
}

} // extern "C"
