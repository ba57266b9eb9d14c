// Row-operation engine: every CSR pass of the library (SpMV, residual, the
// fused smoother / restriction / prolongation kernels of the V-cycle, the
// SpMV+dot of PCG) is one instantiation of these kernels with a different Op.
//
//   Op::val_t                 stored matrix value type (double / float / bf16)
//   Op::acc_t                 accumulation type
//   Op::kFma                  true: s = fma(a, x, s); false: s = s + a*x (rounded twice)
//   Op::kReduce               true: finish() returns a contribution that is summed
//                             deterministically over the grid into red.out
//   acc_t gather(int col)     the x value for a column (may be computed on the fly)
//   double finish(int row, acc_t s)   epilogue with s = sum_j a_ij x_j in CSR order
//   Op::pre_t, pre_t pre(int row), double finish(int row, acc_t s, const pre_t&)
//                             (optional) the row's own epilogue operands (b_i,
//                             D^-1_i, x_i, ...) loaded before its entries, so their
//                             round trip overlaps the gathers instead of following
//                             the reduction; same arithmetic as finish(row, s)
//
// Two schedules, picked per matrix by lab_spmv_analysis:
//   ROWSEQ  one thread per row, CSR order (k_pipe): a persistent CTA streams
//           tiles of consecutive rows (row pointers, values, columns) through a
//           double-buffered shared-memory stage with 16-byte cp.async copies
//           (coalesced, L1 bypassed) and every thread walks its row from shared
//           memory.  With kFma this is bit-identical to the reference host SpMV
//           (host_matrix_vector.cpp:60-84).
//   VECTOR  W lanes per row (W = 2..32, k_vector), coalesced direct loads,
//           strided partial sums, xor-shuffle reduction.
#pragma once

#include "internal.cuh"

#include <map>
#include <mutex>
#include <type_traits>

#include "reduce.cuh"

namespace lab
{
    struct red_buf
    {
        double*       partial = nullptr; // >= grid blocks
        unsigned int* counter = nullptr;
        double*       out     = nullptr;
        const int*    skip    = nullptr; // kernel returns at once when *skip != 0
    };

    // CSR operand of a row kernel.  IT = int32_t: absolute column indices (the
    // stored layout); IT = int16_t: column minus row, the compact copy kept with
    // the reduced-precision values of a matrix whose offsets all fit in 16 bits.
    template <class VT, class IT = int32_t>
    struct csr_view
    {
        const int32_t* rp;
        const IT*      ci;
        const VT*      v;
        int32_t        m;
    };

    template <class IT>
    __device__ __forceinline__ int col_of(IT c, int row)
    {
        if constexpr(sizeof(IT) == 2)
        {
            // sign extension by integer arithmetic on the zero-extended bits (keeps
            // it off the conversion pipe)
            const int u = (int)(unsigned short)c;
            return row + ((u ^ 0x8000) - 0x8000);
        }
        else
            return (int)c;
    }

    __device__ __forceinline__ double to_acc(double v, double)
    {
        return v;
    }
    __device__ __forceinline__ float to_acc(float v, float)
    {
        return v;
    }
    __device__ __forceinline__ float to_acc(__nv_bfloat16 v, float)
    {
        return __bfloat162float(v);
    }
    __device__ __forceinline__ double to_acc(float v, double)
    {
        return (double)v;
    }

    struct no_pre
    {
    };
    template <class Op, class = void>
    struct op_pre
    {
        using type = no_pre;
    };
    template <class Op>
    struct op_pre<Op, std::void_t<typename Op::pre_t>>
    {
        using type = typename Op::pre_t;
    };
    template <class Op>
    using pre_of = typename op_pre<Op>::type;

    template <class Op>
    __device__ __forceinline__ pre_of<Op> pre_load(const Op& op, int row)
    {
        if constexpr(std::is_same<pre_of<Op>, no_pre>::value)
            return no_pre{};
        else
            return op.pre(row);
    }
    template <class Op>
    __device__ __forceinline__ double finish_with(const Op& op, int row, typename Op::acc_t s,
                                                  const pre_of<Op>& p)
    {
        if constexpr(std::is_same<pre_of<Op>, no_pre>::value)
            return op.finish(row, s);
        else
            return op.finish(row, s, p);
    }

    template <bool FMA>
    __device__ __forceinline__ double acc_step(double a, double x, double s)
    {
        return FMA ? fma(a, x, s) : __dadd_rn(s, __dmul_rn(a, x));
    }
    template <bool FMA>
    __device__ __forceinline__ float acc_step(float a, float x, float s)
    {
        return FMA ? fmaf(a, x, s) : __fadd_rn(s, __fmul_rn(a, x));
    }

    __device__ __forceinline__ void cp_async16(void* smem, const void* gmem)
    {
        unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem)
                     : "memory");
    }
    __device__ __forceinline__ void cp_async_wait_all()
    {
        asm volatile("cp.async.wait_all;\n" ::: "memory");
    }

    __device__ __forceinline__ void cp_async_commit()
    {
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    }
    template <int N>
    __device__ __forceinline__ void cp_async_wait_group()
    {
        asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
    }

    // ROWSEQ schedule: persistent, double-buffered tile pipeline.  A tile is NT
    // consecutive rows, one thread per row; each CTA walks tiles blockIdx.x,
    // blockIdx.x + gridDim.x, ... and prefetches tile k+1 (its row pointers, and
    // its contiguous value and column ranges) into the other shared-memory stage
    // with 16-byte cp.async copies while it computes tile k, so the DRAM stream
    // never waits for the gathers and the fma chains.  With MAXR > 0 every row
    // has at most MAXR entries: the row's gathers are issued (up to 16 at a time)
    // before their part of the accumulation chain.  Accumulation in CSR
    // order: with kFma bit-identical to the reference host SpMV
    // (host_matrix_vector.cpp:60-84).  A tile whose nnz exceeds the stage capacity
    // is read straight from global memory (same arithmetic).
    template <class VT, class IT = int32_t>
    __host__ __device__ constexpr size_t pipe_stage_bytes(int cap, int rt)
    {
        return ((size_t)(cap + 16) * sizeof(VT) + 15) / 16 * 16 +
               ((size_t)(cap + 16) * sizeof(IT) + 15) / 16 * 16 + ((size_t)(rt + 8) * 4 + 15) / 16 * 16;
    }

    template <class Op, int NT, int MAXR, class IT>
    __global__ void __launch_bounds__(NT)
        k_pipe(csr_view<typename Op::val_t, IT> A, Op op, int cap, red_buf red, int ntiles)
    {
        using VT = typename Op::val_t;
        using AT = typename Op::acc_t;
        constexpr int VPC = 16 / sizeof(VT);
        constexpr int CPC = 16 / sizeof(IT);
        static_assert(NT % 4 == 0, "tile rows must keep 16-byte row-pointer chunks");
        extern __shared__ __align__(16) unsigned char smem_raw[];
        const size_t sv_b    = ((size_t)(cap + 16) * sizeof(VT) + 15) / 16 * 16;
        const size_t sc_b    = ((size_t)(cap + 16) * sizeof(IT) + 15) / 16 * 16;
        const size_t stage_b = pipe_stage_bytes<VT, IT>(cap, NT);
        if(red.skip && *red.skip)
            return;

        auto issue = [&](int tile, int stage) {
            const int      r0   = tile * NT;
            const int      r1   = min(r0 + NT, A.m);
            const int      j0   = A.rp[r0];
            const int      j1   = A.rp[r1];
            const int      j0v  = j0 & ~(VPC - 1), j0c = j0 & ~(CPC - 1);
            unsigned char* base = smem_raw + stage * stage_b;
            int32_t*       sr   = reinterpret_cast<int32_t*>(base + sv_b + sc_b);
            const int      nr   = (r1 - r0 + 1 + 3) / 4; // rp[r0 .. r1], r0 % 4 == 0
            for(int k = threadIdx.x; k < nr; k += NT)
                cp_async16(sr + 4 * k, A.rp + r0 + 4 * k);
            if((j1 - j0v) <= cap + 8 && (j1 - j0c) <= cap + 8)
            {
                VT*       sv = reinterpret_cast<VT*>(base);
                IT*       sc = reinterpret_cast<IT*>(base + sv_b);
                const int nv = (j1 - j0v + VPC - 1) / VPC;
                const int nc = (j1 - j0c + CPC - 1) / CPC;
                for(int k = threadIdx.x; k < nv; k += NT)
                    cp_async16(sv + (size_t)k * VPC, A.v + j0v + (size_t)k * VPC);
                for(int k = threadIdx.x; k < nc; k += NT)
                    cp_async16(sc + (size_t)k * CPC, A.ci + j0c + (size_t)k * CPC);
            }
        };

        double contrib = 0.0;
        int    tile    = blockIdx.x;
        if(tile < ntiles)
            issue(tile, 0);
        cp_async_commit();
        for(int it = 0; tile < ntiles; it++, tile += gridDim.x)
        {
            const int nxt = tile + gridDim.x;
            if(nxt < ntiles)
                issue(nxt, (it + 1) & 1);
            cp_async_commit();
            cp_async_wait_group<1>(); // everything but the newest group has landed
            __syncthreads();
            const unsigned char* base   = smem_raw + (it & 1) * stage_b;
            const VT*            sv     = reinterpret_cast<const VT*>(base);
            const IT*            sc     = reinterpret_cast<const IT*>(base + sv_b);
            const int32_t*       sr     = reinterpret_cast<const int32_t*>(base + sv_b + sc_b);
            const int            r0     = tile * NT;
            const int            r1     = min(r0 + NT, A.m);
            const int            j0     = sr[0], j1 = sr[r1 - r0];
            const int            j0v    = j0 & ~(VPC - 1), j0c = j0 & ~(CPC - 1);
            const bool           staged = (j1 - j0v) <= cap + 8 && (j1 - j0c) <= cap + 8;
            const int            row    = r0 + threadIdx.x;
            if(row < r1)
            {
                const pre_of<Op> pr = pre_load(op, row);
                const int        a = sr[row - r0], b = sr[row - r0 + 1];
                AT               s = AT(0);
                if(MAXR > 0 && staged)
                {
                    // gathers issued 16 at a time before their part of the chain,
                    // the values re-read from shared memory
                    constexpr int CH = MAXR < 16 ? MAXR : 16;
#pragma unroll
                    for(int c0 = 0; c0 < MAXR; c0 += CH)
                    {
                        AT xv[CH > 0 ? CH : 1];
#pragma unroll
                        for(int q = 0; q < CH; q++)
                            if(a + c0 + q < b)
                                xv[q] = op.gather(col_of<IT>(sc[a + c0 + q - j0c], row));
#pragma unroll
                        for(int q = 0; q < CH; q++)
                            if(a + c0 + q < b)
                                s = acc_step<Op::kFma>(to_acc(sv[a + c0 + q - j0v], AT(0)), xv[q],
                                                       s);
                    }
                }
                else if(staged)
                {
                    for(int j = a; j < b; j++)
                        s = acc_step<Op::kFma>(to_acc(sv[j - j0v], AT(0)),
                                               op.gather(col_of<IT>(sc[j - j0c], row)), s);
                }
                else
                {
                    for(int j = a; j < b; j++)
                        s = acc_step<Op::kFma>(to_acc(A.v[j], AT(0)),
                                               op.gather(col_of<IT>(A.ci[j], row)), s);
                }
                contrib += finish_with(op, row, s, pr);
            }
            __syncthreads(); // this stage is refilled by the prefetch two tiles on
        }
        cp_async_wait_group<0>();
        if(Op::kReduce)
            reduce_finish_sum<NT>(contrib, red.partial, red.counter, red.out);
    }

    // ROWSEQ schedule for rows of 17..32 entries (27-point stencils): a warp owns a
    // tile of 32 consecutive rows, stages the tile's row pointers, values and
    // columns into its own shared-memory region with cp.async, and each lane
    // walks its row from there (CSR-order fma chain, bit-identical to k_pipe).
    // No block barrier: per-warp single buffering keeps the shared memory per
    // resident row small, so about 20 warps per SM stream tiles independently
    // (a CTA-wide double-buffered 256-row tile of 27-entry rows leaves one CTA,
    // 8 warps, per SM).  `cap` = 32 x the longest row; a larger tile is read from
    // global memory directly.
    constexpr int kWarpPipeWarps = 4;

    template <class VT, class IT = int32_t>
    __host__ __device__ constexpr size_t warp_stage_bytes(int cap)
    {
        return ((size_t)(cap + 16) * sizeof(VT) + 15) / 16 * 16 +
               ((size_t)(cap + 16) * sizeof(IT) + 15) / 16 * 16 + ((size_t)(32 + 8) * 4 + 15) / 16 * 16;
    }

    template <class Op, int MAXR, class IT>
    __global__ void __launch_bounds__(32 * kWarpPipeWarps)
        k_pipe_warp(csr_view<typename Op::val_t, IT> A, Op op, int cap, red_buf red, int ntiles)
    {
        using VT = typename Op::val_t;
        using AT = typename Op::acc_t;
        constexpr int VPC = 16 / sizeof(VT);
        constexpr int CPC = 16 / sizeof(IT);
        extern __shared__ __align__(16) unsigned char smem_raw[];
        const size_t   sv_b = ((size_t)(cap + 16) * sizeof(VT) + 15) / 16 * 16;
        const size_t   sc_b = ((size_t)(cap + 16) * sizeof(IT) + 15) / 16 * 16;
        const int      wid  = threadIdx.x >> 5, lane = threadIdx.x & 31;
        unsigned char* base = smem_raw + (size_t)wid * warp_stage_bytes<VT, IT>(cap);
        VT*            sv   = reinterpret_cast<VT*>(base);
        IT*            sc   = reinterpret_cast<IT*>(base + sv_b);
        int32_t*       sr   = reinterpret_cast<int32_t*>(base + sv_b + sc_b);
        if(red.skip && *red.skip)
            return;
        double contrib = 0.0;
        for(int tile = blockIdx.x * kWarpPipeWarps + wid; tile < ntiles;
            tile += gridDim.x * kWarpPipeWarps)
        {
            const int  r0     = tile * 32;
            const int  r1     = min(r0 + 32, A.m);
            const int  j0     = A.rp[r0];
            const int  j1     = A.rp[r1];
            const int  j0v    = j0 & ~(VPC - 1), j0c = j0 & ~(CPC - 1);
            const bool staged = (j1 - j0v) <= cap + 8 && (j1 - j0c) <= cap + 8;
            const int  nr     = (r1 - r0 + 1 + 3) / 4; // rp[r0 .. r1], r0 % 4 == 0
            for(int k = lane; k < nr; k += 32)
                cp_async16(sr + 4 * k, A.rp + r0 + 4 * k);
            if(staged)
            {
                const int nv = (j1 - j0v + VPC - 1) / VPC;
                const int nc = (j1 - j0c + CPC - 1) / CPC;
                for(int k = lane; k < nv; k += 32)
                    cp_async16(sv + (size_t)k * VPC, A.v + j0v + (size_t)k * VPC);
                for(int k = lane; k < nc; k += 32)
                    cp_async16(sc + (size_t)k * CPC, A.ci + j0c + (size_t)k * CPC);
            }
            cp_async_commit();
            cp_async_wait_group<0>();
            __syncwarp();
            const int row = r0 + lane;
            if(row < r1)
            {
                const pre_of<Op> pr = pre_load(op, row);
                const int        a = sr[lane], b = sr[lane + 1];
                AT               s = AT(0);
                if(staged)
                {
                    constexpr int CH = 16;
#pragma unroll
                    for(int c0 = 0; c0 < MAXR; c0 += CH)
                    {
                        AT xv[CH];
#pragma unroll
                        for(int q = 0; q < CH; q++)
                            if(a + c0 + q < b)
                                xv[q] = op.gather(col_of<IT>(sc[a + c0 + q - j0c], row));
#pragma unroll
                        for(int q = 0; q < CH; q++)
                            if(a + c0 + q < b)
                                s = acc_step<Op::kFma>(to_acc(sv[a + c0 + q - j0v], AT(0)), xv[q],
                                                       s);
                    }
                }
                else
                {
                    for(int j = a; j < b; j++)
                        s = acc_step<Op::kFma>(to_acc(A.v[j], AT(0)),
                                               op.gather(col_of<IT>(A.ci[j], row)), s);
                }
                contrib += finish_with(op, row, s, pr);
            }
            __syncwarp(); // the region is refilled by the warp's next tile
        }
        if(Op::kReduce)
            reduce_finish_sum<32 * kWarpPipeWarps>(contrib, red.partial, red.counter, red.out);
    }

    // ROWSEQ schedule for rows longer than 32 entries (coarse AMG levels): one
    // thread per row, the row walked in segments of SEG entries whose values,
    // columns and gathers are all issued before that segment's part of the
    // accumulation chain (CSR order, bit-identical to the reference host SpMV).
    // A lane's SEG consecutive entries share one or two L1 lines, so the strided
    // pattern across the warp costs L1 wavefronts, not DRAM traffic.
    constexpr int kSegLen = 8;

    template <class Op, int NT, class IT>
    __global__ void __launch_bounds__(NT)
        k_row_seg(csr_view<typename Op::val_t, IT> A, Op op, red_buf red)
    {
        using AT = typename Op::acc_t;
        if(red.skip && *red.skip)
            return;
        double    contrib = 0.0;
        const int row     = blockIdx.x * NT + threadIdx.x;
        if(row < A.m)
        {
            const pre_of<Op> pr = pre_load(op, row);
            const int        a = A.rp[row], b = A.rp[row + 1];
            AT               s = AT(0);
            for(int c0 = a; c0 < b; c0 += kSegLen)
            {
                AT vv[kSegLen], xv[kSegLen];
#pragma unroll
                for(int q = 0; q < kSegLen; q++)
                    if(c0 + q < b)
                    {
                        vv[q] = to_acc(A.v[c0 + q], AT(0));
                        xv[q] = op.gather(col_of<IT>(A.ci[c0 + q], row));
                    }
#pragma unroll
                for(int q = 0; q < kSegLen; q++)
                    if(c0 + q < b)
                        s = acc_step<Op::kFma>(vv[q], xv[q], s);
            }
            contrib = finish_with(op, row, s, pr);
        }
        if(Op::kReduce)
            reduce_finish_sum<NT>(contrib, red.partial, red.counter, red.out);
    }

    // Four consecutive entries from a 4-aligned position, as wide loads.
    __device__ __forceinline__ void ld4(const double* p, double (&o)[4])
    {
        const double2 u = __ldg(reinterpret_cast<const double2*>(p));
        const double2 w = __ldg(reinterpret_cast<const double2*>(p + 2));
        o[0] = u.x, o[1] = u.y, o[2] = w.x, o[3] = w.y;
    }
    __device__ __forceinline__ void ld4(const float* p, float (&o)[4])
    {
        const float4 u = __ldg(reinterpret_cast<const float4*>(p));
        o[0] = u.x, o[1] = u.y, o[2] = u.z, o[3] = u.w;
    }
    __device__ __forceinline__ void ld4(const __nv_bfloat16* p, __nv_bfloat16 (&o)[4])
    {
        const uint2           u = __ldg(reinterpret_cast<const uint2*>(p));
        const __nv_bfloat16* h = reinterpret_cast<const __nv_bfloat16*>(&u);
        o[0] = h[0], o[1] = h[1], o[2] = h[2], o[3] = h[3];
    }
    __device__ __forceinline__ void ld4(const int32_t* p, int32_t (&o)[4])
    {
        const int4 u = __ldg(reinterpret_cast<const int4*>(p));
        o[0] = u.x, o[1] = u.y, o[2] = u.z, o[3] = u.w;
    }
    __device__ __forceinline__ void ld4(const int16_t* p, int16_t (&o)[4])
    {
        const uint2    u = __ldg(reinterpret_cast<const uint2*>(p));
        const int16_t* h = reinterpret_cast<const int16_t*>(&u);
        o[0] = h[0], o[1] = h[1], o[2] = h[2], o[3] = h[3];
    }

    // VECTOR schedule (rows longer than 32 entries): W lanes per row and an
    // xor-shuffle reduction over the W lane sums.  FP64 values: lane-strided
    // single entries.  Reduced-precision values: each lane takes aligned quads of
    // entries with one wide load of values and one of columns (the row's first and
    // last quads masked to [a, b)) and its four gathers in flight together; loads
    // start at the row's aligned-down position and may run up to three entries
    // past the matrix end, inside the allocations' padding.
    template <class Op, int NT, int W, class IT>
    __global__ void __launch_bounds__(NT)
        k_vector(csr_view<typename Op::val_t, IT> A, Op op, red_buf red)
    {
        using VT = typename Op::val_t;
        using AT = typename Op::acc_t;
        if(red.skip && *red.skip)
            return;
        const int  lane = threadIdx.x & (W - 1);
        const int  row  = (int)(((int64_t)blockIdx.x * NT + threadIdx.x) / W);
        AT         s    = AT(0);
        pre_of<Op> pr{};
        if(row < A.m && lane == 0)
            pr = pre_load(op, row);
        if(row < A.m && sizeof(VT) == 8)
        {
            // FP64 values: one entry per lane step (a quad would need two loads anyway)
            const int a = A.rp[row], b = A.rp[row + 1];
#pragma unroll 4
            for(int j = a + lane; j < b; j += W)
                s = acc_step<Op::kFma>(to_acc(A.v[j], AT(0)), op.gather(col_of<IT>(A.ci[j], row)),
                                       s);
        }
        else if(row < A.m)
        {
            const int a = A.rp[row], b = A.rp[row + 1];
#pragma unroll 2
            for(int q = (a & ~3) + 4 * lane; q < b; q += 4 * W)
            {
                VT v4[4];
                IT c4[4];
                ld4(A.v + q, v4);
                ld4(A.ci + q, c4);
                AT xg[4];
#pragma unroll
                for(int t = 0; t < 4; t++)
                    if(q + t >= a && q + t < b)
                        xg[t] = op.gather(col_of<IT>(c4[t], row));
#pragma unroll
                for(int t = 0; t < 4; t++)
                    if(q + t >= a && q + t < b)
                        s = acc_step<Op::kFma>(to_acc(v4[t], AT(0)), xg[t], s);
            }
        }
#pragma unroll
        for(int o = W / 2; o > 0; o >>= 1)
            s += __shfl_xor_sync(0xffffffffu, s, o, W);
        double contrib = 0.0;
        if(row < A.m && lane == 0)
            contrib = finish_with(op, row, s, pr);
        if(Op::kReduce)
            reduce_finish_sum<NT>(contrib, red.partial, red.counter, red.out);
    }

    __device__ __forceinline__ void ld4(const uint16_t* p, uint16_t (&o)[4])
    {
        const uint2     u = __ldg(reinterpret_cast<const uint2*>(p));
        const uint16_t* h = reinterpret_cast<const uint16_t*>(&u);
        o[0] = h[0], o[1] = h[1], o[2] = h[2], o[3] = h[3];
    }

    template <class Op>
    using gather_t = std::decay_t<decltype(std::declval<const Op&>().gather(0))>;

    struct halo_view
    {
        const int32_t*  cnt;  // per chunk: staged distinct columns, -1 = direct reads
        const int32_t*  col;  // chunk c's distinct columns at c * slot, ascending
        const uint16_t* loc;  // per entry: its column's position in the chunk's list
        int             rows; // rows per chunk
        int             slot;
    };

    // VECTOR schedule with a per-chunk halo (long rows whose columns stay near the
    // diagonal: the coarse SA levels).  One CTA per chunk of consecutive rows first
    // stages x at the chunk's distinct columns in shared memory, one coalesced pass
    // over an ascending column list, then runs k_vector's per-row work -- the same
    // lanes, the same entries per lane in the same order, the same shuffle tree --
    // with every gather read from shared memory.  The distinct columns number about
    // a quarter of the entries on those levels, so most of the scattered gathers
    // that bound k_vector (one L1/TEX request per entry) disappear; the matrix
    // stream is unchanged (16-bit local positions in place of the 16-bit offsets).
    // Row results are bit-identical to k_vector.  Ops with a reduction keep
    // k_vector (a thread here sums several rows, which would regroup the sum).
    template <class Op, int NT, int W, class IT>
    __global__ void __launch_bounds__(NT)
        k_vhalo(csr_view<typename Op::val_t, IT> A, halo_view h, Op op, red_buf red)
    {
        using VT = typename Op::val_t;
        using AT = typename Op::acc_t;
        using GT = gather_t<Op>;
        static_assert(!Op::kReduce, "reductions keep k_vector");
        extern __shared__ __align__(16) unsigned char smem_raw[];
        GT* sx = reinterpret_cast<GT*>(smem_raw);
        if(red.skip && *red.skip)
            return;
        const int64_t r0  = (int64_t)blockIdx.x * h.rows;
        const int     r1  = (int)(r0 + h.rows < A.m ? r0 + h.rows : A.m);
        const int     cnt = h.cnt[blockIdx.x];
        if(cnt > 0)
        {
            // U list entries per thread in flight: U column loads, then U gathers
            // (ascending columns: neighbouring threads read neighbouring x)
            constexpr int  U  = 8;
            const int32_t* hc = h.col + (size_t)blockIdx.x * h.slot;
            for(int k0 = threadIdx.x; k0 < cnt; k0 += NT * U)
            {
                int c[U];
#pragma unroll
                for(int u = 0; u < U; u++)
                    c[u] = k0 + u * NT < cnt ? __ldg(hc + k0 + u * NT) : -1;
                GT g[U];
#pragma unroll
                for(int u = 0; u < U; u++)
                    if(c[u] >= 0)
                        g[u] = op.gather(c[u]);
#pragma unroll
                for(int u = 0; u < U; u++)
                    if(c[u] >= 0)
                        sx[k0 + u * NT] = g[u];
            }
        }
        __syncthreads();
        const bool staged = cnt >= 0;
        const int  lane   = threadIdx.x & (W - 1);
        for(int base = (int)r0; base < r1; base += NT / W)
        {
            const int  row = base + (int)threadIdx.x / W;
            AT         s   = AT(0);
            pre_of<Op> pr{};
            if(row < r1 && lane == 0)
                pr = pre_load(op, row);
            if(row < r1 && sizeof(VT) == 8)
            {
                const int a = A.rp[row], b = A.rp[row + 1];
                if(staged)
                {
#pragma unroll 4
                    for(int j = a + lane; j < b; j += W)
                        s = acc_step<Op::kFma>(to_acc(A.v[j], AT(0)), sx[h.loc[j]], s);
                }
                else
                {
#pragma unroll 4
                    for(int j = a + lane; j < b; j += W)
                        s = acc_step<Op::kFma>(to_acc(A.v[j], AT(0)),
                                               op.gather(col_of<IT>(A.ci[j], row)), s);
                }
            }
            else if(row < r1)
            {
                const int a = A.rp[row], b = A.rp[row + 1];
#pragma unroll 2
                for(int q = (a & ~3) + 4 * lane; q < b; q += 4 * W)
                {
                    VT v4[4];
                    ld4(A.v + q, v4);
                    AT xg[4];
                    if(staged)
                    {
                        uint16_t l4[4];
                        ld4(h.loc + q, l4);
#pragma unroll
                        for(int t = 0; t < 4; t++)
                            if(q + t >= a && q + t < b)
                                xg[t] = sx[l4[t]];
                    }
                    else
                    {
                        IT c4[4];
                        ld4(A.ci + q, c4);
#pragma unroll
                        for(int t = 0; t < 4; t++)
                            if(q + t >= a && q + t < b)
                                xg[t] = op.gather(col_of<IT>(c4[t], row));
                    }
#pragma unroll
                    for(int t = 0; t < 4; t++)
                        if(q + t >= a && q + t < b)
                            s = acc_step<Op::kFma>(to_acc(v4[t], AT(0)), xg[t], s);
                }
            }
#pragma unroll
            for(int o = W / 2; o > 0; o >>= 1)
                s += __shfl_xor_sync(0xffffffffu, s, o, W);
            if(row < r1 && lane == 0)
                finish_with(op, row, s, pr);
        }
    }

    constexpr int kRowseqNT = 256;
    constexpr int kVectorNT = 256;

    // Grid size a row op will use on this matrix (reduction partial buffers must
    // hold at least this many entries).
    inline int64_t rowop_grid(const lab_csr_impl* A)
    {
        if(A->m == 0)
            return 0;
        if(A->plan.alg == LAB_SPMV_ROWSEQ)
            return ceil_div<int64_t>(A->m, kRowseqNT);
        return ceil_div<int64_t>(A->m * (int64_t)A->plan.lanes, kVectorNT);
    }

    // Blocks per SM of one k_pipe instantiation at a given dynamic shared-memory
    // size (cached; the stage size differs per matrix).
    template <class Op, int MAXR, class IT>
    int pipe_occupancy(size_t smem)
    {
        const auto                   kernel = k_pipe<Op, kRowseqNT, MAXR, IT>;
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

    template <class Op, int MAXR, class IT>
    lab_status launch_pipe(const csr_view<typename Op::val_t, IT>& V, const Op& op, int cap,
                           cudaStream_t s, const red_buf& red)
    {
        using VT              = typename Op::val_t;
        const int      ntiles = (int)ceil_div<int64_t>(V.m, kRowseqNT);
        const size_t   smem   = 2 * pipe_stage_bytes<VT, IT>(cap, kRowseqNT);
        const int      occ    = pipe_occupancy<Op, MAXR, IT>(smem);
        const unsigned grid   = (unsigned)std::min<int64_t>(
            std::min<int64_t>(ntiles, (int64_t)num_sms() * occ), kRedBlocks);
        LAB_LAUNCH((k_pipe<Op, kRowseqNT, MAXR, IT>), grid, kRowseqNT, smem, s, V, op, cap, red,
                   ntiles);
        return LAB_OK;
    }

    template <class Op, int MAXR, class IT>
    lab_status launch_pipe_warp(const csr_view<typename Op::val_t, IT>& V, const Op& op, int cap,
                                cudaStream_t s, const red_buf& red)
    {
        using VT                    = typename Op::val_t;
        constexpr int  NT           = 32 * kWarpPipeWarps;
        const auto     kernel       = k_pipe_warp<Op, MAXR, IT>;
        const int      ntiles       = (int)ceil_div<int64_t>(V.m, 32);
        const size_t   smem         = kWarpPipeWarps * warp_stage_bytes<VT, IT>(cap);
        static std::mutex            mu;
        static std::map<size_t, int> cache;
        static const cudaError_t     attr = cudaFuncSetAttribute(
            kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        LAB_CUDA(attr);
        int occ = 1;
        {
            std::lock_guard<std::mutex> g(mu);
            auto                        it = cache.find(smem);
            if(it == cache.end())
            {
                int o = 0;
                if(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kernel, NT, smem) != cudaSuccess)
                {
                    cudaGetLastError();
                    o = 1;
                }
                it = cache.emplace(smem, std::max(o, 1)).first;
            }
            occ = it->second;
        }
        // persistent grid, at most kRedBlocks CTAs (the reduction partial buffers)
        const unsigned grid = (unsigned)std::min<int64_t>(
            std::min<int64_t>(ceil_div<int64_t>(ntiles, kWarpPipeWarps), (int64_t)num_sms() * occ),
            kRedBlocks);
        LAB_LAUNCH((k_pipe_warp<Op, MAXR, IT>), grid, NT, smem, s, V, op, cap, red, ntiles);
        return LAB_OK;
    }

    template <class Op, class IT>
    lab_status launch_row_seg(const csr_view<typename Op::val_t, IT>& V, const Op& op,
                              cudaStream_t s, const red_buf& red)
    {
        // one thread per row: ceil(m / 256) CTAs, the ROWSEQ partial-buffer size
        const unsigned grid = (unsigned)ceil_div<int64_t>(V.m, kRowseqNT);
        LAB_LAUNCH((k_row_seg<Op, kRowseqNT, IT>), grid, kRowseqNT, 0, s, V, op, red);
        return LAB_OK;
    }

    template <class Op, int W, class IT>
    lab_status launch_vector(const csr_view<typename Op::val_t, IT>& V, const Op& op,
                             unsigned grid, cudaStream_t s, const red_buf& red)
    {
        LAB_LAUNCH((k_vector<Op, kVectorNT, W, IT>), grid, kVectorNT, 0, s, V, op, red);
        return LAB_OK;
    }

    // The halo form when the matrix has one and the op has no reduction; returns
    // false (nothing launched) otherwise.
    template <class Op, int W, class IT>
    bool launch_vhalo(const lab_csr_impl* A, const csr_view<typename Op::val_t, IT>& V,
                      const Op& op, cudaStream_t s, const red_buf& red, lab_status* st)
    {
        const spmv_plan& p = A->plan;
        if constexpr(Op::kReduce)
            return false;
        else
        {
            if(p.halo_state != 1 || !p.halo_use || p.stream)
                return false;
            using GT          = gather_t<Op>;
            const auto kernel = k_vhalo<Op, kVectorNT, W, IT>;
            static const cudaError_t attr = cudaFuncSetAttribute(
                kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kHaloCap * (int)sizeof(GT));
            *st = LAB_OK;
            if(attr != cudaSuccess)
            {
                *st = cuda_status(attr, "cudaFuncSetAttribute(k_vhalo)", __FILE__, __LINE__);
                return true;
            }
            const halo_view h{p.hcnt, p.hcol, p.hloc, p.hrows, p.hslot};
            const size_t    smem = (size_t)std::max(p.hslot, 1) * sizeof(GT);
            *st                  = [&]() -> lab_status {
                LAB_LAUNCH(kernel, (unsigned)p.hchunks, kVectorNT, smem, s, V, h, op, red);
                return LAB_OK;
            }();
            return true;
        }
    }

}

#include "vstream.cuh"

namespace lab
{
    template <class Op, class IT>
    lab_status launch_rowop_view(const lab_csr_impl* A, const csr_view<typename Op::val_t, IT>& V,
                                 const Op& op, cudaStream_t s, const red_buf& red)
    {
        const spmv_plan& p = A->plan;
        if(p.alg == LAB_SPMV_ROWSEQ)
        {
            const int mr = std::max(1, p.max_row);
            if(mr <= 8)
                return launch_pipe<Op, 8, IT>(V, op, kRowseqNT * mr, s, red);
            if(mr <= 16)
                return launch_pipe<Op, 16, IT>(V, op, kRowseqNT * mr, s, red);
            if(mr <= 32)
                return launch_pipe_warp<Op, 32, IT>(V, op, 32 * mr, s, red);
            return launch_row_seg<Op, IT>(V, op, s, red);
        }
        const unsigned grid = (unsigned)rowop_grid(A);
        lab_status     st   = LAB_OK;
        switch(p.lanes)
        {
        case 2:
            if(launch_vstream<Op, 2, IT>(A, V, op, s, red, &st))
                return st;
            if(launch_vhalo<Op, 2, IT>(A, V, op, s, red, &st))
                return st;
            return launch_vector<Op, 2, IT>(V, op, grid, s, red);
        case 4:
            if(launch_vstream<Op, 4, IT>(A, V, op, s, red, &st))
                return st;
            if(launch_vhalo<Op, 4, IT>(A, V, op, s, red, &st))
                return st;
            return launch_vector<Op, 4, IT>(V, op, grid, s, red);
        case 8:
            if(launch_vstream<Op, 8, IT>(A, V, op, s, red, &st))
                return st;
            if(launch_vhalo<Op, 8, IT>(A, V, op, s, red, &st))
                return st;
            return launch_vector<Op, 8, IT>(V, op, grid, s, red);
        case 16:
            if(launch_vstream<Op, 16, IT>(A, V, op, s, red, &st))
                return st;
            if(launch_vhalo<Op, 16, IT>(A, V, op, s, red, &st))
                return st;
            return launch_vector<Op, 16, IT>(V, op, grid, s, red);
        default:
            if(launch_vstream<Op, 32, IT>(A, V, op, s, red, &st))
                return st;
            if(launch_vhalo<Op, 32, IT>(A, V, op, s, red, &st))
                return st;
            return launch_vector<Op, 32, IT>(V, op, grid, s, red);
        }
    }

    // One CSR pass of `op` over A with the given value array.  The matrix's 16-bit
    // column offsets are read in place of the int32 columns when it has them (every
    // offset fits: built with the SpMV plan), in every precision; the column each
    // entry names is the same, so results are unchanged.
    template <class Op>
    lab_status launch_rowop(const lab_csr_impl* A, const typename Op::val_t* vals, const Op& op,
                            cudaStream_t s, red_buf red = red_buf())
    {
        using VT = typename Op::val_t;
        if(A->m == 0)
            return LAB_OK;
        if(A->lp.dcol)
        {
            csr_view<VT, int16_t> V{A->row_ptr, A->lp.dcol, vals, (int32_t)A->m};
            return launch_rowop_view<Op, int16_t>(A, V, op, s, red);
        }
        csr_view<VT, int32_t> V{A->row_ptr, A->col_ind, vals, (int32_t)A->m};
        return launch_rowop_view<Op, int32_t>(A, V, op, s, red);
    }

    // ------------------------------------------------------------ basic ops
    struct op_spmv
    {
        using val_t                    = double;
        using acc_t                    = double;
        static constexpr bool kFma     = true;
        static constexpr bool kReduce  = false;
        const double* __restrict__ x;
        double* __restrict__ y;
        double alpha, beta;
        __device__ __forceinline__ double gather(int c) const
        {
            return __ldg(x + c);
        }
        // host_matrix_vector.cpp:82
        __device__ __forceinline__ double finish(int r, double s) const
        {
            y[r] = beta == 0.0 ? __dmul_rn(alpha, s) : fma(alpha, s, __dmul_rn(beta, y[r]));
            return 0.0;
        }
        using pre_t = double; // y_r (read only when beta != 0)
        __device__ __forceinline__ double pre(int r) const
        {
            return beta == 0.0 ? 0.0 : y[r];
        }
        __device__ __forceinline__ double finish(int r, double s, double yr) const
        {
            y[r] = beta == 0.0 ? __dmul_rn(alpha, s) : fma(alpha, s, __dmul_rn(beta, yr));
            return 0.0;
        }
    };

    struct op_residual
    {
        using val_t                   = double;
        using acc_t                   = double;
        static constexpr bool kFma    = false; // host_matrix_vector.cpp:53 uses s += a*x
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
            r[i] = __dsub_rn(b[i], s);
            return 0.0;
        }
        using pre_t = double; // b_i
        __device__ __forceinline__ double pre(int i) const
        {
            return __ldg(b + i);
        }
        __device__ __forceinline__ double finish(int i, double s, double bi) const
        {
            r[i] = __dsub_rn(bi, s);
            return 0.0;
        }
    };
}
