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
//
// Two schedules, picked per matrix by lab_spmv_analysis:
//   ROWSEQ  one thread per row.  The CTA's contiguous nnz range is staged into
//           shared memory with 16-byte cp.async copies (coalesced, L1 bypassed),
//           then every thread walks its row in CSR order.  With kFma this is
//           bit-identical to the reference host SpMV (host_matrix_vector.cpp:60-84).
//   VECTOR  W lanes per row (W = 2..32), strided loads, xor-shuffle reduction.
#pragma once

#include "internal.cuh"
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

    template <class VT>
    struct csr_view
    {
        const int32_t* rp;
        const int32_t* ci;
        const VT*      v;
        int32_t        m;
    };

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

    // Shared-memory bytes the ROWSEQ kernel needs for `cap` staged entries.
    template <class VT>
    __host__ __device__ constexpr size_t rowseq_smem(int cap)
    {
        return ((size_t)(cap + 16) * sizeof(VT) + 15) / 16 * 16 + (size_t)(cap + 8) * 4;
    }

    // MAXR > 0: every row has at most MAXR entries (from the analysis); the row is
    // read into registers with all its gathers issued before the fma chain, which
    // keeps MAXR loads in flight per thread.  The accumulation order is unchanged.
    template <class Op, int NT, int MAXR>
    __global__ void __launch_bounds__(NT)
        k_rowseq(csr_view<typename Op::val_t> A, Op op, int cap, red_buf red)
    {
        using VT = typename Op::val_t;
        using AT = typename Op::acc_t;
        extern __shared__ __align__(16) unsigned char smem_raw[];
        constexpr int VPC = 16 / sizeof(VT); // values per 16-byte chunk
        VT*           sv  = reinterpret_cast<VT*>(smem_raw);
        int32_t*      sc  = reinterpret_cast<int32_t*>(smem_raw + ((size_t)(cap + 16) * sizeof(VT) + 15) / 16 * 16);
        if(red.skip && *red.skip)
            return;

        const int r0  = blockIdx.x * NT;
        const int r1  = min(r0 + NT, A.m);
        const int j0  = A.rp[r0];
        const int j1  = A.rp[r1];
        const int j0v = j0 & ~(VPC - 1);
        const int j0c = j0 & ~3;
        const bool staged = (j1 - j0v) <= cap + 8 && (j1 - j0c) <= cap + 4;
        if(staged)
        {
            const int nv = (j1 - j0v + VPC - 1) / VPC;
            const int nc = (j1 - j0c + 3) / 4;
            for(int k = threadIdx.x; k < nv; k += NT)
                cp_async16(sv + (size_t)k * VPC, A.v + j0v + (size_t)k * VPC);
            for(int k = threadIdx.x; k < nc; k += NT)
                cp_async16(sc + (size_t)k * 4, A.ci + j0c + (size_t)k * 4);
            cp_async_wait_all();
        }
        __syncthreads();

        double contrib = 0.0;
        const int row  = r0 + threadIdx.x;
        if(row < r1)
        {
            const int a = A.rp[row], b = A.rp[row + 1];
            AT        s = AT(0);
            if(staged && MAXR > 0)
            {
                AT vv[MAXR > 0 ? MAXR : 1], xv[MAXR > 0 ? MAXR : 1];
#pragma unroll
                for(int k = 0; k < MAXR; k++)
                    if(a + k < b)
                    {
                        vv[k] = to_acc(sv[a + k - j0v], AT(0));
                        xv[k] = op.gather(sc[a + k - j0c]);
                    }
#pragma unroll
                for(int k = 0; k < MAXR; k++)
                    if(a + k < b)
                        s = acc_step<Op::kFma>(vv[k], xv[k], s);
            }
            else if(staged)
            {
                for(int j = a; j < b; j++)
                    s = acc_step<Op::kFma>(to_acc(sv[j - j0v], AT(0)), op.gather(sc[j - j0c]), s);
            }
            else
            {
                for(int j = a; j < b; j++)
                    s = acc_step<Op::kFma>(to_acc(A.v[j], AT(0)), op.gather(A.ci[j]), s);
            }
            contrib = op.finish(row, s);
        }
        if(Op::kReduce)
            reduce_finish_sum<NT>(contrib, red.partial, red.counter, red.out);
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

    // Persistent, double-buffered form of k_rowseq: each CTA walks row blocks
    // blockIdx.x, blockIdx.x + gridDim.x, ... and prefetches block k+1 into the
    // other shared-memory stage (cp.async groups) while it computes block k, so
    // the DRAM stream never waits for the gathers and the fma chains.  Same
    // per-row arithmetic as k_rowseq (bit-identical results).
    template <class Op, int NT, int MAXR>
    __global__ void __launch_bounds__(NT)
        k_rowseq_pipe(csr_view<typename Op::val_t> A, Op op, int cap, red_buf red, int nblocks)
    {
        using VT = typename Op::val_t;
        using AT = typename Op::acc_t;
        extern __shared__ __align__(16) unsigned char smem_raw[];
        constexpr int VPC    = 16 / sizeof(VT);
        const size_t  sv_b   = ((size_t)(cap + 16) * sizeof(VT) + 15) / 16 * 16;
        const size_t  sc_b   = ((size_t)(cap + 8) * 4 + 15) / 16 * 16;
        const size_t  stage_b = sv_b + sc_b;
        if(red.skip && *red.skip)
            return;

        auto issue = [&](int blk, int stage) {
            const int r0  = blk * NT;
            const int r1  = min(r0 + NT, A.m);
            const int j0  = A.rp[r0];
            const int j1  = A.rp[r1];
            const int j0v = j0 & ~(VPC - 1);
            const int j0c = j0 & ~3;
            if((j1 - j0v) <= cap + 8 && (j1 - j0c) <= cap + 4)
            {
                VT*      sv = reinterpret_cast<VT*>(smem_raw + stage * stage_b);
                int32_t* sc = reinterpret_cast<int32_t*>(smem_raw + stage * stage_b + sv_b);
                const int nv = (j1 - j0v + VPC - 1) / VPC;
                const int nc = (j1 - j0c + 3) / 4;
                for(int k = threadIdx.x; k < nv; k += NT)
                    cp_async16(sv + (size_t)k * VPC, A.v + j0v + (size_t)k * VPC);
                for(int k = threadIdx.x; k < nc; k += NT)
                    cp_async16(sc + (size_t)k * 4, A.ci + j0c + (size_t)k * 4);
            }
        };

        double contrib = 0.0;
        int    blk     = blockIdx.x;
        if(blk < nblocks)
            issue(blk, 0);
        cp_async_commit();
        for(int it = 0; blk < nblocks; it++, blk += gridDim.x)
        {
            const int nxt = blk + gridDim.x;
            if(nxt < nblocks)
                issue(nxt, (it + 1) & 1);
            cp_async_commit();
            cp_async_wait_group<1>(); // everything but the newest group has landed
            __syncthreads();
            const int stage = it & 1;
            const int r0    = blk * NT;
            const int r1    = min(r0 + NT, A.m);
            const int j0    = A.rp[r0];
            const int j1    = A.rp[r1];
            const int j0v   = j0 & ~(VPC - 1);
            const int j0c   = j0 & ~3;
            const bool staged = (j1 - j0v) <= cap + 8 && (j1 - j0c) <= cap + 4;
            const VT*      sv = reinterpret_cast<const VT*>(smem_raw + stage * stage_b);
            const int32_t* sc = reinterpret_cast<const int32_t*>(smem_raw + stage * stage_b + sv_b);
            const int row = r0 + threadIdx.x;
            if(row < r1)
            {
                const int a = A.rp[row], b = A.rp[row + 1];
                AT        s = AT(0);
                if(staged)
                {
                    AT vv[MAXR], xv[MAXR];
#pragma unroll
                    for(int k = 0; k < MAXR; k++)
                        if(a + k < b)
                        {
                            vv[k] = to_acc(sv[a + k - j0v], AT(0));
                            xv[k] = op.gather(sc[a + k - j0c]);
                        }
#pragma unroll
                    for(int k = 0; k < MAXR; k++)
                        if(a + k < b)
                            s = acc_step<Op::kFma>(vv[k], xv[k], s);
                }
                else
                {
                    for(int j = a; j < b; j++)
                        s = acc_step<Op::kFma>(to_acc(A.v[j], AT(0)), op.gather(A.ci[j]), s);
                }
                contrib += op.finish(row, s);
            }
            __syncthreads(); // this stage is refilled by the prefetch two blocks on
        }
        cp_async_wait_group<0>();
        if(Op::kReduce)
            reduce_finish_sum<NT>(contrib, red.partial, red.counter, red.out);
    }

    template <class Op, int NT, int W>
    __global__ void __launch_bounds__(NT)
        k_vector(csr_view<typename Op::val_t> A, Op op, red_buf red)
    {
        using AT       = typename Op::acc_t;
        if(red.skip && *red.skip)
            return;
        const int lane = threadIdx.x & (W - 1);
        const int row  = (int)(((int64_t)blockIdx.x * NT + threadIdx.x) / W);
        AT        s    = AT(0);
        if(row < A.m)
        {
            const int a = A.rp[row], b = A.rp[row + 1];
#pragma unroll 4
            for(int j = a + lane; j < b; j += W)
                s = acc_step<Op::kFma>(to_acc(A.v[j], AT(0)), op.gather(A.ci[j]), s);
        }
#pragma unroll
        for(int o = W / 2; o > 0; o >>= 1)
            s += __shfl_xor_sync(0xffffffffu, s, o, W);
        double contrib = 0.0;
        if(row < A.m && lane == 0)
            contrib = op.finish(row, s);
        if(Op::kReduce)
            reduce_finish_sum<NT>(contrib, red.partial, red.counter, red.out);
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

    template <class Op>
    lab_status launch_rowop(const lab_csr_impl* A, const typename Op::val_t* vals, const Op& op,
                            cudaStream_t s, red_buf red = red_buf())
    {
        using VT = typename Op::val_t;
        if(A->m == 0)
            return LAB_OK;
        csr_view<VT> V{A->row_ptr, A->col_ind, vals, (int32_t)A->m};
        const spmv_plan& p = A->plan;
        if(p.alg == LAB_SPMV_ROWSEQ)
        {
            int    cap  = kRowseqNT * std::max(1, p.max_row);
            size_t smem = rowseq_smem<VT>(cap);
            if(smem > 200 * 1024)
            {
                cap  = 0; // fall back to unstaged global reads
                smem = rowseq_smem<VT>(0);
            }
            // Raise the dynamic shared-memory cap once per instantiation.
            static const cudaError_t attr8 = cudaFuncSetAttribute(
                k_rowseq<Op, kRowseqNT, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
            static const cudaError_t attr16 = cudaFuncSetAttribute(
                k_rowseq<Op, kRowseqNT, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                200 * 1024);
            static const cudaError_t attr0 = cudaFuncSetAttribute(
                k_rowseq<Op, kRowseqNT, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
            LAB_CUDA(attr8);
            LAB_CUDA(attr16);
            LAB_CUDA(attr0);
            const unsigned grid = (unsigned)rowop_grid(A);
            if(p.max_row <= 16)
            {
                // persistent double-buffered kernel; stage capacity fixed per instantiation
                const int  nblocks = (int)grid;
                const bool r8      = p.max_row <= 8;
                const int  pcap    = kRowseqNT * (r8 ? 8 : 16);
                const size_t psmem = 2 * (((size_t)(pcap + 16) * sizeof(VT) + 15) / 16 * 16 +
                                          ((size_t)(pcap + 8) * 4 + 15) / 16 * 16);
                static int occ8 = -1, occ16 = -1;
                int&       occ  = r8 ? occ8 : occ16;
                if(occ < 0)
                {
                    if(r8)
                    {
                        LAB_CUDA(cudaFuncSetAttribute(k_rowseq_pipe<Op, kRowseqNT, 8>,
                                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                      (int)psmem));
                        LAB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                            &occ, k_rowseq_pipe<Op, kRowseqNT, 8>, kRowseqNT, psmem));
                    }
                    else
                    {
                        LAB_CUDA(cudaFuncSetAttribute(k_rowseq_pipe<Op, kRowseqNT, 16>,
                                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                      (int)psmem));
                        LAB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                            &occ, k_rowseq_pipe<Op, kRowseqNT, 16>, kRowseqNT, psmem));
                    }
                    occ = std::max(occ, 1);
                }
                const unsigned pgrid =
                    (unsigned)std::min<int64_t>(nblocks, (int64_t)num_sms() * occ);
                if(r8)
                    LAB_LAUNCH((k_rowseq_pipe<Op, kRowseqNT, 8>), pgrid, kRowseqNT, psmem, s, V,
                               op, pcap, red, nblocks);
                else
                    LAB_LAUNCH((k_rowseq_pipe<Op, kRowseqNT, 16>), pgrid, kRowseqNT, psmem, s, V,
                               op, pcap, red, nblocks);
                return LAB_OK;
            }
            LAB_LAUNCH((k_rowseq<Op, kRowseqNT, 0>), grid, kRowseqNT, smem, s, V, op, cap, red);
            return LAB_OK;
        }
        unsigned grid = (unsigned)rowop_grid(A);
        switch(p.lanes)
        {
        case 2:
            LAB_LAUNCH((k_vector<Op, kVectorNT, 2>), grid, kVectorNT, 0, s, V, op, red);
            break;
        case 4:
            LAB_LAUNCH((k_vector<Op, kVectorNT, 4>), grid, kVectorNT, 0, s, V, op, red);
            break;
        case 8:
            LAB_LAUNCH((k_vector<Op, kVectorNT, 8>), grid, kVectorNT, 0, s, V, op, red);
            break;
        case 16:
            LAB_LAUNCH((k_vector<Op, kVectorNT, 16>), grid, kVectorNT, 0, s, V, op, red);
            break;
        default:
            LAB_LAUNCH((k_vector<Op, kVectorNT, 32>), grid, kVectorNT, 0, s, V, op, red);
            break;
        }
        return LAB_OK;
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
    };
}
