// Internal declarations shared by the liblinalg_b200 translation units.
#pragma once

#include "lab.h"

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <vector>

namespace lab
{
    // ------------------------------------------------------------ errors
    void       set_error(const char* fmt, ...);
    lab_status cuda_status(cudaError_t e, const char* what, const char* file, int line);

#define LAB_CUDA(call)                                                            \
    do                                                                            \
    {                                                                             \
        cudaError_t e_ = (call);                                                  \
        if(e_ != cudaSuccess)                                                     \
            return ::lab::cuda_status(e_, #call, __FILE__, __LINE__);             \
    } while(0)

#define LAB_TRY(x)                                                                \
    do                                                                            \
    {                                                                             \
        lab_status s_ = (x);                                                      \
        if(s_ != LAB_OK)                                                          \
            return s_;                                                            \
    } while(0)

#define LAB_ARG(cond, msg)                                                        \
    do                                                                            \
    {                                                                             \
        if(!(cond))                                                               \
        {                                                                         \
            ::lab::set_error("bad argument: %s (%s)", msg, #cond);                \
            return LAB_BAD_ARG;                                                   \
        }                                                                         \
    } while(0)

    // Kernel launches go through this macro so the library can count them.
    extern std::atomic<int64_t> g_launches;
#define LAB_LAUNCH(kernel, grid, block, smem, stream, ...)                        \
    do                                                                            \
    {                                                                             \
        kernel<<<(grid), (block), (smem), (stream)>>>(__VA_ARGS__);               \
        ::lab::g_launches.fetch_add(1, std::memory_order_relaxed);                \
        cudaError_t le_ = cudaGetLastError();                                     \
        if(le_ != cudaSuccess)                                                    \
            return ::lab::cuda_status(le_, #kernel, __FILE__, __LINE__);          \
    } while(0)

    // ------------------------------------------------------------ device / memory
    lab_status ensure_init();
    int        num_sms();
    inline cudaStream_t to_stream(lab_stream s)
    {
        return reinterpret_cast<cudaStream_t>(s);
    }

    // Fork-join of independent launches (row classes of one pass): next() hands out
    // the caller's stream first, then (for passes over few rows) streams of a
    // small library-owned pool that
    // wait for everything enqueued on the caller's stream so far; the destructor
    // makes the caller's stream wait for all of them, so temporaries freed on it
    // afterwards and later work are ordered after every forked launch.  On coarse
    // levels the classes are small, latency-bound launches that now overlap.
    class stream_fork
    {
    public:
        // Below this many rows a pass's class launches are latency-bound and gain
        // from overlapping; above it each launch fills the GPU and overlapping
        // only makes them compete (measured on the SA levels of a 128^3 Poisson
        // hierarchy: the 5.9k-row Galerkin product 1.12 -> 0.63 ms forked, the
        // 60k-row one 1.17 -> 1.44 ms).
        static constexpr int64_t kMaxRows = 16384;
        stream_fork(cudaStream_t s, int64_t rows) : s_(s), on_(rows <= kMaxRows) {}
        ~stream_fork();
        stream_fork(const stream_fork&)            = delete;
        stream_fork& operator=(const stream_fork&) = delete;
        cudaStream_t next();

    private:
        static constexpr int kSides = 7;
        cudaStream_t         s_;
        bool                 on_;
        cudaEvent_t          fork_ = nullptr;
        cudaEvent_t          done_[kSides] = {};
        int                  used_ = 0; // launches handed out (the first on s_)
    };

    // Stream-ordered allocation from the device's default memory pool (the pool
    // keeps freed blocks, so setup temporaries cost no driver round trips).
    // Every allocation is padded by 64 bytes so vectorised loads that round a
    // range out to a 16-byte boundary stay inside it.
    lab_status dmalloc(void** p, size_t bytes, cudaStream_t s);
    void       dfree(void* p, cudaStream_t s);

    template <class T>
    inline lab_status dalloc(T** p, size_t n, cudaStream_t s)
    {
        return dmalloc(reinterpret_cast<void**>(p), n * sizeof(T), s);
    }

    // RAII device buffer for temporaries.
    template <class T>
    struct dbuf
    {
        T*           p = nullptr;
        size_t       n = 0;
        cudaStream_t s = 0;
        dbuf()         = default;
        dbuf(const dbuf&) = delete;
        dbuf& operator=(const dbuf&) = delete;
        ~dbuf()
        {
            release();
        }
        lab_status alloc(size_t count, cudaStream_t st)
        {
            release();
            s = st;
            n = count;
            return dalloc(&p, count > 0 ? count : 1, st);
        }
        void release()
        {
            if(p)
                dfree(p, s);
            p = nullptr;
            n = 0;
        }
        T* get() const
        {
            return p;
        }
    };

    // Pinned host staging for scalar read-backs.
    lab_status pinned_scratch(void** p, size_t bytes);

    // ------------------------------------------------------------ CSR
    struct spmv_plan
    {
        int    analysed = 0;
        int    alg      = LAB_SPMV_ROWSEQ; // lab_spmv_alg
        int    lanes    = 1;               // lanes per row for LAB_SPMV_VECTOR
        int    vlanes   = 2;               // lanes a multi-lane kernel would use (mean row / 3)
        int    forced   = 0;
        int    max_row  = 0;
        double avg_row  = 0.0;
        // LAB_SPMV_ROWSEQ: row blocks of bounded nnz
        int  rows_per_block = 0;
        int  nblocks        = 0;
        int* block_row      = nullptr; // device int32[nblocks+1] (row starts), null = uniform
        // LAB_SPMV_MERGE: merge-path split points
        int  merge_items_per_block = 0;
        int* merge_coords          = nullptr; // device int32[2*(nblocks+1)]
        // streamed VECTOR form (vstream.cuh): rows per tile and stage capacity in
        // entries (the largest tile plus alignment slack; 0: no stream geometry),
        // and whether the plan uses it (LAB_SPMV_VECTOR_STREAM)
        int st_rows = 0;
        int st_cap  = 0;
        int stream  = 0;
        // halo form of VECTOR (spmv_engine.cuh, k_vhalo): chunks of hrows
        // consecutive rows; chunk c stages x at its hcnt[c] distinct columns
        // (hcol[c * hslot ...], ascending) in shared memory and every entry names
        // its column by hloc[j], the position in that list; hcnt[c] = -1: the chunk
        // reads x directly.  Built once per pattern (halo_state 1; -1: not square,
        // or no chunk can be staged) for LAB_SPMV_VECTOR_HALO and the autotuner;
        // used while halo_use is set (that schedule forced or tuned in).
        int       halo_state = 0;
        int       halo_use   = 0;
        int       hrows      = 0;
        int       hchunks    = 0;
        int       hslot      = 0; // largest staged count, the shared-memory entries
        int64_t   hdistinct  = 0; // staged columns over all chunks
        int       hdirect    = 0; // chunks left to direct reads (hcnt = -1)
        int32_t*  hcnt       = nullptr;
        int32_t*  hcol       = nullptr;
        uint16_t* hloc       = nullptr;
    };

    // Halo geometry: a chunk's columns are marked in a shared-memory bitmap over its
    // column span (at most kHaloBits columns), and at most kHaloCap distinct columns
    // are staged; chunks beyond either read x directly.
    constexpr int kHaloBits = 1 << 18;
    constexpr int kHaloCap  = 8192;

    struct csr_values_lp
    {
        float*          f32  = nullptr;
        __nv_bfloat16*  bf16 = nullptr;
        float*          invd32 = nullptr;
        // column minus row as int16 (when every offset fits), read with the
        // reduced-precision values: 2 instead of 4 index bytes per entry
        int16_t*        dcol       = nullptr;
        int             dcol_state = 0; // 0 not examined, 1 built, -1 offsets too wide
    };

    // Unique ids for cached solver state (graphs are keyed by object identity,
    // not by address, so a freed-and-reused address never matches).
    uint64_t next_uid();
    // Drop solver caches keyed by an object that is being destroyed.
    void solver_cache_forget(const void* key);

    struct lab_csr_impl
    {
        uint64_t  uid = next_uid();
        int64_t   m = 0, n = 0, nnz = 0;
        int32_t*  row_ptr = nullptr;
        int32_t*  col_ind = nullptr;
        double*   val     = nullptr;
        spmv_plan plan;
        // cached diagonal data for smoothers (built on demand)
        double* diag    = nullptr;
        double* invdiag = nullptr;
        csr_values_lp lp;
        struct tri_plan* tri = nullptr; // triangular-solve levels (tri.cu), on demand
    };
    void tri_release(lab_csr_impl* A);

    lab_status csr_alloc(lab_csr_impl** A, int64_t m, int64_t n, int64_t nnz, cudaStream_t s);
    void       csr_release(lab_csr_impl* A);
    lab_status csr_ensure_invdiag(lab_csr_impl* A, cudaStream_t s);
    // d[i] = the first stored a_ii in CSR order (0 if none), invd[i] = 1 / d[i];
    // either output may be null.
    lab_status diag_into(const lab_csr_impl* A, double* d, double* invd, cudaStream_t s);
    lab_status csr_ensure_lowp(lab_csr_impl* A, int precision, int use_bf16, cudaStream_t s);
    lab_status spmv_analyse(lab_csr_impl* A, cudaStream_t s);
    // The same for several matrices with one host round trip (nulls skipped).
    lab_status spmv_analyse_batch(lab_csr_impl* const* mats, int count, cudaStream_t s);
    // Builds A's halo plan (spmv_plan::hcnt/hcol/hloc) unless it was examined.
    lab_status halo_build(lab_csr_impl* A, cudaStream_t s);
    lab_status spmm_columns(const lab_csr_impl* A, int k, const double* X, int64_t ldx, double* Y,
                            int64_t ldy, cudaStream_t s, const int* skip);

    // ------------------------------------------------------------ shared device helpers
    lab_status scan_i32(int32_t* x, int64_t n, cudaStream_t s); // in-place exclusive
    lab_status scan_i64(int64_t* x, int64_t n, cudaStream_t s);
    // Exclusive scan of n counts into row_ptr[0..n] (row_ptr[n] = total); total to host.
    lab_status counts_to_rowptr(const int32_t* counts, int32_t* row_ptr, int64_t n,
                                int64_t* total, cudaStream_t s);
    lab_status max_i64(const int64_t* x, int64_t n, int64_t* result_host, cudaStream_t s);
    // max_i64 whose result lands in pinned host memory (pinned_small()) when the
    // stream next synchronises: read it only after a later synchronisation.
    lab_status max_i64_async(const int64_t* x, int64_t n, int64_t* host_out, cudaStream_t s);
    // A small pinned host buffer of the calling thread (64 int64 slots), or null.
    int64_t* pinned_small();
    lab_status copy_d2h_sync(void* dst, const void* src, size_t bytes, cudaStream_t s);

    // Fixed-shape reduction grid shared by every deterministic reduction.
    constexpr int kRedBlocks  = 1184; // 8 x 148 SMs
    constexpr int kRedThreads = 256;

    template <class T>
    __host__ __device__ inline T ceil_div(T a, T b)
    {
        return (a + b - 1) / b;
    }

    __device__ __forceinline__ double warp_sum(double v)
    {
#pragma unroll
        for(int o = 16; o > 0; o >>= 1)
            v += __shfl_xor_sync(0xffffffffu, v, o);
        return v;
    }

    // max that propagates NaN (fmax drops it, which would let a NaN residual
    // norm read as small)
    __device__ __forceinline__ double nanmax(double a, double b)
    {
        return (a != a || b != b) ? __longlong_as_double(0x7ff8000000000000ll) : fmax(a, b);
    }

    __device__ __forceinline__ double warp_max(double v)
    {
#pragma unroll
        for(int o = 16; o > 0; o >>= 1)
            v = nanmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        return v;
    }
}

struct lab_csr_s : lab::lab_csr_impl
{
};
