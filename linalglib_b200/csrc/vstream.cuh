// Streamed VECTOR schedule (LAB_SPMV_VECTOR_STREAM) for large operators with
// long rows: the W-lanes-per-row arithmetic of k_vector, fed by a
// warp-specialised shared-memory pipeline.  Not the default: on the coarse SA
// levels of the 128^3 Poisson hierarchy it measured slower than k_vector (level 1
// 59 vs 49 us, level 2 44 vs 23 us, the level-0 restriction 64 vs 45 us per
// FP64 SpMV): those passes are bound by the scattered gathers of x through
// L1/TEX, which streaming the matrix does not reduce, and the stage ring leaves
// fewer warps per SM to hide the gather latency.  The autotuner times it as a
// candidate.
//
// A persistent CTA walks tiles of `rows` consecutive rows.  Warp 0 is the
// producer: one elected thread copies each tile's row pointers, values and
// columns from HBM into a ring of kStreamStages shared-memory stages with 1D
// bulk copies (cp.async.bulk, completion counted in bytes on the stage's "full"
// mbarrier).  Warps 1..kStreamConsumers are consumers: they wait on the full
// barrier of a stage, run the W-lane rows of the tile from shared memory (each
// warp a share of the rows), and arrive on the stage's "empty" barrier, which
// hands the stage back to the producer.  There is no block-wide barrier per
// tile: a consumer warp that finishes early starts on the next staged tile, and
// the matrix stream runs ahead of the dependent x gathers by up to
// kStreamStages tiles.
//
// Every wait is bounded (kStreamWaitLimit polls): a wait that runs out sets the
// CTA's abort flag, counts itself in the library's device status word, and the
// CTA winds down -- the producer first waits (again bounded) for its own copies
// still in flight, so no copy lands in shared memory after the CTA has left.
//
// Per row the lanes take the same entries in the same order as k_vector (FP64:
// lane-strided single entries; reduced precision: aligned quads), followed by
// the same xor-shuffle tree, so every row result is bit-identical to k_vector's.
#pragma once

// Included by spmv_engine.cuh (it uses the row-op machinery defined there).
namespace lab
{
    constexpr int      kStreamConsumers = 8;
    constexpr int      kStreamNT        = 32 * (kStreamConsumers + 1);
    constexpr int      kStreamStages    = 2;
    constexpr unsigned kStreamWaitLimit = 1u << 22;
    // operators with fewer rows keep k_vector (a few tiles cannot fill the GPU)
    constexpr int64_t kStreamMinRows = 8192;
    // entries per tile the tile height aims at, and the largest stage accepted
    constexpr int kStreamTileEntries = 2048;
    constexpr int kStreamMaxCap      = 4096;

    __host__ __device__ constexpr size_t round16(size_t b)
    {
        return (b + 15) / 16 * 16;
    }

    template <class VT, class IT>
    __host__ __device__ constexpr size_t stream_stage_bytes(int cap, int rows)
    {
        return round16((size_t)cap * sizeof(VT)) + round16((size_t)cap * sizeof(IT)) +
               round16((size_t)(rows + 4) * sizeof(int32_t));
    }

    // ------------------------------------------------------------ PTX wrappers
    __device__ __forceinline__ unsigned smem_u32(const void* p)
    {
        return (unsigned)__cvta_generic_to_shared(p);
    }

    __device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count)
    {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                     : "memory");
    }

    // make the initialised barriers visible to the bulk-copy (async) proxy
    __device__ __forceinline__ void fence_barrier_init()
    {
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }

    __device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes)
    {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                     "r"(bytes)
                     : "memory");
    }

    __device__ __forceinline__ void mbar_arrive(uint64_t* bar)
    {
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
    }

    __device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity)
    {
        unsigned ok;
        asm volatile("{\n\t.reg .pred p;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(ok)
                     : "r"(smem_u32(bar)), "r"(parity)
                     : "memory");
        return ok != 0;
    }

    // Bounded wait for the phase of `parity`; false when it ran out or the CTA is
    // aborting.
    __device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity,
                                              volatile int* abort_flag)
    {
        for(unsigned i = 0; i < kStreamWaitLimit; i++)
        {
            if(mbar_try_wait(bar, parity))
                return true;
            if((i & 63u) == 63u && *abort_flag)
                return false;
        }
        return false;
    }

    // 1D bulk copy global -> this CTA's shared memory, completing on `bar`.  No
    // multicast: the source is this GPU's own memory and one CTA receives it.
    __device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes,
                                             uint64_t* bar)
    {
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes "
                     "[%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
                     "l"(src), "r"(bytes), "r"(smem_u32(bar))
                     : "memory");
    }

    // plain 4-wide shared-memory loads (k_vector's ld4 reads global memory)
    __device__ __forceinline__ void lds4(const float* p, float (&o)[4])
    {
        const float4 u = *reinterpret_cast<const float4*>(p);
        o[0] = u.x, o[1] = u.y, o[2] = u.z, o[3] = u.w;
    }
    __device__ __forceinline__ void lds4(const __nv_bfloat16* p, __nv_bfloat16 (&o)[4])
    {
        const uint2           u = *reinterpret_cast<const uint2*>(p);
        const __nv_bfloat16* h = reinterpret_cast<const __nv_bfloat16*>(&u);
        o[0] = h[0], o[1] = h[1], o[2] = h[2], o[3] = h[3];
    }
    __device__ __forceinline__ void lds4(const int32_t* p, int32_t (&o)[4])
    {
        const int4 u = *reinterpret_cast<const int4*>(p);
        o[0] = u.x, o[1] = u.y, o[2] = u.z, o[3] = u.w;
    }
    __device__ __forceinline__ void lds4(const int16_t* p, int16_t (&o)[4])
    {
        const uint2    u = *reinterpret_cast<const uint2*>(p);
        const int16_t* h = reinterpret_cast<const int16_t*>(&u);
        o[0] = h[0], o[1] = h[1], o[2] = h[2], o[3] = h[3];
    }

    // status[0] counts bounded waits that ran out
    template <class Op, int W, class IT>
    __global__ void __launch_bounds__(kStreamNT)
        k_vstream(csr_view<typename Op::val_t, IT> A, Op op, int rows, int cap, int ntiles,
                  red_buf red, int* status)
    {
        using VT = typename Op::val_t;
        using AT = typename Op::acc_t;
        constexpr int VPC = 16 / sizeof(VT);
        constexpr int CPC = 16 / sizeof(IT);
        constexpr int RPW = 32 / W; // rows of a warp pass
        extern __shared__ __align__(128) unsigned char smem_stream[];
        __shared__ __align__(8) uint64_t full[kStreamStages];
        __shared__ __align__(8) uint64_t empty[kStreamStages];
        __shared__ int                   abort_flag;
        if(red.skip && *red.skip)
            return;
        const size_t sv_b    = round16((size_t)cap * sizeof(VT));
        const size_t sc_b    = round16((size_t)cap * sizeof(IT));
        const size_t stage_b = stream_stage_bytes<VT, IT>(cap, rows);
        const int    warp    = threadIdx.x >> 5;
        const int    lane    = threadIdx.x & 31;
        if(threadIdx.x == 0)
        {
            for(int q = 0; q < kStreamStages; q++)
            {
                mbar_init(&full[q], 1);
                mbar_init(&empty[q], kStreamConsumers);
            }
            abort_flag = 0;
            fence_barrier_init();
        }
        __syncthreads();
        volatile int* abort_v = &abort_flag;
        double        contrib = 0.0;
        if(warp == 0)
        {
            // the whole producer warp walks the tiles; every 32 tiles each lane loads
            // the entry bounds of one upcoming tile (one warp-wide load instead of a
            // dependent round trip per tile), and lane 0 issues the copies
            int it = 0, jb0 = 0, jb1 = 0;
            for(int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, it++)
            {
                const int k = it & 31;
                if(k == 0)
                {
                    const int t = tile + lane * gridDim.x;
                    if(t < ntiles)
                    {
                        jb0 = A.rp[t * rows];
                        jb1 = A.rp[min(t * rows + rows, A.m)];
                    }
                }
                const int j0 = __shfl_sync(0xffffffffu, jb0, k);
                const int j1 = __shfl_sync(0xffffffffu, jb1, k);
                int stop = 0;
                if(lane == 0)
                {
                    const int      st = it % kStreamStages;
                    const unsigned ph = (unsigned)(it / kStreamStages) & 1u;
                    // the stage is free once every consumer released its previous use
                    if(!mbar_wait(&empty[st], ph ^ 1u, abort_v))
                    {
                        if(!*abort_v)
                            atomicAdd(status, 1);
                        *abort_v = 1;
                        stop     = 1;
                    }
                    else
                    {
                        const int      r0   = tile * rows;
                        const int      r1   = min(r0 + rows, A.m);
                        const int      j0v  = j0 & ~(VPC - 1);
                        const int      j0c  = j0 & ~(CPC - 1);
                        const unsigned bv   = (unsigned)round16((size_t)(j1 - j0v) * sizeof(VT));
                        const unsigned bc   = (unsigned)round16((size_t)(j1 - j0c) * sizeof(IT));
                        const unsigned br   = (unsigned)round16((size_t)(r1 - r0 + 1) * sizeof(int32_t));
                        unsigned char* base = smem_stream + (size_t)st * stage_b;
                        mbar_arrive_expect_tx(&full[st], bv + bc + br);
                        bulk_g2s(base + sv_b + sc_b, A.rp + r0, br, &full[st]);
                        if(bv)
                            bulk_g2s(base, A.v + j0v, bv, &full[st]);
                        if(bc)
                            bulk_g2s(base + sv_b, A.ci + j0c, bc, &full[st]);
                    }
                }
                if(__shfl_sync(0xffffffffu, stop, 0))
                    break;
            }
            if(lane == 0)
            {
                // no copy may land after the CTA has left: wait for the copies of
                // the last stages issued (their phases complete as the bytes arrive);
                // `it` counts the tiles whose copies were issued
                for(int k = max(0, it - kStreamStages); k < it; k++)
                {
                    const int      st = k % kStreamStages;
                    const unsigned ph = (unsigned)(k / kStreamStages) & 1u;
                    bool           ok = false;
                    for(unsigned i = 0; i < kStreamWaitLimit && !ok; i++)
                        ok = mbar_try_wait(&full[st], ph);
                    if(!ok)
                        atomicAdd(status, 1);
                }
            }
        }
        else
        {
            const int cw = warp - 1;
            const int g  = lane / W;
            const int li = lane % W;
            int       it = 0;
            for(int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, it++)
            {
                const int      st = it % kStreamStages;
                const unsigned ph = (unsigned)(it / kStreamStages) & 1u;
                if(!mbar_wait(&full[st], ph, abort_v))
                {
                    if(lane == 0)
                    {
                        if(!*abort_v)
                            atomicAdd(status, 1);
                        *abort_v = 1;
                    }
                    break;
                }
                const unsigned char* base = smem_stream + (size_t)st * stage_b;
                const VT*            sv   = reinterpret_cast<const VT*>(base);
                const IT*            sc   = reinterpret_cast<const IT*>(base + sv_b);
                const int32_t*       sr   = reinterpret_cast<const int32_t*>(base + sv_b + sc_b);
                const int            r0   = tile * rows;
                const int            nr   = min(rows, A.m - r0);
                const int            j0   = sr[0];
                const int            j0v  = j0 & ~(VPC - 1);
                const int            j0c  = j0 & ~(CPC - 1);
                for(int kb = cw * RPW; kb < nr; kb += kStreamConsumers * RPW)
                {
                    const int  k    = kb + g;
                    const bool live = k < nr;
                    const int  row  = r0 + k;
                    AT         s    = AT(0);
                    pre_of<Op> pr{};
                    if(live && li == 0)
                        pr = pre_load(op, row);
                    if(live)
                    {
                        const int a = sr[k], b = sr[k + 1];
                        if constexpr(sizeof(VT) == 8)
                        {
#pragma unroll 4
                            for(int j = a + li; j < b; j += W)
                                s = acc_step<Op::kFma>(to_acc(sv[j - j0v], AT(0)),
                                                       op.gather(col_of<IT>(sc[j - j0c], row)), s);
                        }
                        else
                        {
#pragma unroll 2
                            for(int q = (a & ~3) + 4 * li; q < b; q += 4 * W)
                            {
                                VT v4[4];
                                IT c4[4];
                                lds4(sv + (q - j0v), v4);
                                lds4(sc + (q - j0c), c4);
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
                    }
#pragma unroll
                    for(int o = W / 2; o > 0; o >>= 1)
                        s += __shfl_xor_sync(0xffffffffu, s, o, W);
                    if(live && li == 0)
                        contrib += finish_with(op, row, s, pr);
                }
                __syncwarp();
                if(lane == 0)
                    mbar_arrive(&empty[st]);
            }
        }
        __syncthreads();
        if(Op::kReduce)
            reduce_finish_sum<kStreamNT>(contrib, red.partial, red.counter, red.out);
    }

    int* device_status_word();

    // Blocks per SM of one k_vstream instantiation at a given stage size (cached).
    template <class Op, int W, class IT>
    int vstream_occupancy(size_t smem)
    {
        const auto                   kernel = k_vstream<Op, W, IT>;
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
        if(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, kStreamNT, smem) !=
           cudaSuccess)
        {
            cudaGetLastError();
            occ = 0;
        }
        cache[smem] = occ;
        return occ;
    }

    // Launch the streaming form if the matrix has a stream geometry and the
    // stages fit; returns false (nothing launched) otherwise.
    template <class Op, int W, class IT>
    bool launch_vstream(const lab_csr_impl* A, const csr_view<typename Op::val_t, IT>& V,
                        const Op& op, cudaStream_t s, const red_buf& red, lab_status* st)
    {
        using VT             = typename Op::val_t;
        const spmv_plan& p   = A->plan;
        if(!p.stream || p.st_rows <= 0 || p.st_cap <= 0)
            return false;
        const size_t smem = (size_t)kStreamStages * stream_stage_bytes<VT, IT>(p.st_cap, p.st_rows);
        const int    occ  = vstream_occupancy<Op, W, IT>(smem);
        int*         word = device_status_word();
        if(occ <= 0 || !word)
            return false;
        const int     ntiles = (int)ceil_div<int64_t>(A->m, p.st_rows);
        const int64_t grid   = std::min<int64_t>(
            std::min<int64_t>(ntiles, (int64_t)num_sms() * occ), rowop_grid(A));
        *st = LAB_OK;
        k_vstream<Op, W, IT><<<(unsigned)grid, kStreamNT, smem, s>>>(V, op, p.st_rows, p.st_cap,
                                                                      ntiles, red, word);
        g_launches.fetch_add(1, std::memory_order_relaxed);
        cudaError_t e = cudaGetLastError();
        if(e != cudaSuccess)
            *st = cuda_status(e, "k_vstream", __FILE__, __LINE__);
        return true;
    }
}
