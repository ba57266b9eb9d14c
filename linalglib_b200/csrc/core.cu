// Runtime, memory, CSR containers, BLAS-1 and scans for liblinalg_b200.
#include "internal.cuh"
#include "reduce.cuh"

#include <cstdarg>
#include <cstring>
#include <mutex>

namespace lab
{
    std::atomic<int64_t> g_launches{0};
    static std::atomic<uint64_t> g_uid{1};
    uint64_t next_uid()
    {
        return g_uid.fetch_add(1);
    }

    static thread_local char t_err[512] = "";

    void set_error(const char* fmt, ...)
    {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(t_err, sizeof(t_err), fmt, ap);
        va_end(ap);
    }

    lab_status cuda_status(cudaError_t e, const char* what, const char* file, int line)
    {
        set_error("%s:%d %s: %s", file, line, what, cudaGetErrorString(e));
        if(e == cudaErrorMemoryAllocation)
            return LAB_OOM;
        if(e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
            return LAB_NO_DEVICE;
        return LAB_CUDA_ERROR;
    }

    static std::once_flag g_init_once;
    static lab_status     g_init_status = LAB_OK;
    static int            g_sms         = 148;
    static int            g_device      = -1;

    static lab_status do_init(int device)
    {
        int n = 0;
        if(cudaGetDeviceCount(&n) != cudaSuccess || n == 0)
        {
            cudaGetLastError();
            set_error("no CUDA device available");
            return LAB_NO_DEVICE;
        }
        if(device < 0)
            LAB_CUDA(cudaGetDevice(&device));
        LAB_CUDA(cudaSetDevice(device));
        cudaDeviceProp prop;
        LAB_CUDA(cudaGetDeviceProperties(&prop, device));
        if(prop.major < 10)
        {
            set_error("device %d is sm_%d%d; this library is built for sm_100a only", device,
                      prop.major, prop.minor);
            return LAB_NO_DEVICE;
        }
        g_sms    = prop.multiProcessorCount;
        g_device = device;
        // Keep freed pool memory cached: setup allocates many short-lived buffers.
        cudaMemPool_t pool;
        LAB_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
        uint64_t thr = UINT64_MAX;
        LAB_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
        return LAB_OK;
    }

    lab_status ensure_init()
    {
        std::call_once(g_init_once, [] { g_init_status = do_init(-1); });
        if(g_init_status != LAB_OK)
            set_error("device initialisation failed");
        return g_init_status;
    }

    int num_sms()
    {
        return g_sms;
    }

    lab_status dmalloc(void** p, size_t bytes, cudaStream_t s)
    {
        LAB_TRY(ensure_init());
        *p              = nullptr;
        cudaError_t e   = cudaMallocAsync(p, bytes + 64, s);
        if(e != cudaSuccess)
        {
            cudaGetLastError();
            set_error("device allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
            return e == cudaErrorMemoryAllocation ? LAB_OOM : LAB_CUDA_ERROR;
        }
        return LAB_OK;
    }

    void dfree(void* p, cudaStream_t s)
    {
        if(p)
            cudaFreeAsync(p, s);
    }

    // One small device word per device for kernels to report bounded waits that
    // ran out (word 0); allocated once and kept for the life of the process.
    int* device_status_word()
    {
        static std::mutex mu;
        static int*       words[64] = {};
        int               dev       = 0;
        if(cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
            return nullptr;
        std::lock_guard<std::mutex> g(mu);
        if(!words[dev])
        {
            int* p = nullptr;
            if(cudaMalloc(&p, 64) != cudaSuccess || cudaMemset(p, 0, 64) != cudaSuccess)
            {
                cudaGetLastError();
                return nullptr;
            }
            words[dev] = p;
        }
        return words[dev];
    }

    lab_status pinned_scratch(void** p, size_t bytes)
    {
        static thread_local void*  buf = nullptr;
        static thread_local size_t cap = 0;
        if(cap < bytes)
        {
            if(buf)
                cudaFreeHost(buf);
            buf = nullptr;
            cap = 0;
            LAB_CUDA(cudaMallocHost(&buf, bytes < 4096 ? 4096 : bytes));
            cap = bytes < 4096 ? 4096 : bytes;
        }
        *p = buf;
        return LAB_OK;
    }

    lab_status copy_d2h_sync(void* dst, const void* src, size_t bytes, cudaStream_t s)
    {
        void* h;
        LAB_TRY(pinned_scratch(&h, bytes));
        LAB_CUDA(cudaMemcpyAsync(h, src, bytes, cudaMemcpyDeviceToHost, s));
        LAB_CUDA(cudaStreamSynchronize(s));
        std::memcpy(dst, h, bytes);
        return LAB_OK;
    }

    // ------------------------------------------------------------ stream fork
    static cudaStream_t* side_pool()
    {
        static cudaStream_t pool[8] = {};
        static bool         ok      = [] {
            for(auto& x : pool)
                if(cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking) != cudaSuccess)
                {
                    cudaGetLastError();
                    return false;
                }
            return true;
        }();
        return ok ? pool : nullptr;
    }

    cudaStream_t stream_fork::next()
    {
        const int k = used_++;
        if(k == 0 || !on_)
            return s_;
        cudaStream_t* pool = side_pool();
        if(!pool || k > kSides)
            return s_; // serial fallback
        if(!fork_)
        {
            if(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming) != cudaSuccess ||
               cudaEventRecord(fork_, s_) != cudaSuccess)
            {
                cudaGetLastError();
                if(fork_)
                    cudaEventDestroy(fork_);
                fork_ = nullptr;
                used_ = kSides + 1; // everything else on s_
                return s_;
            }
        }
        cudaStream_t side = pool[k - 1];
        if(cudaEventCreateWithFlags(&done_[k - 1], cudaEventDisableTiming) != cudaSuccess)
        {
            cudaGetLastError();
            done_[k - 1] = nullptr;
            return s_;
        }
        if(cudaStreamWaitEvent(side, fork_, 0) != cudaSuccess)
        {
            cudaGetLastError();
            cudaEventDestroy(done_[k - 1]);
            done_[k - 1] = nullptr;
            return s_;
        }
        return side;
    }

    stream_fork::~stream_fork()
    {
        cudaStream_t* pool = side_pool();
        for(int k = 0; k < kSides; k++)
            if(done_[k])
            {
                if(pool && cudaEventRecord(done_[k], pool[k]) == cudaSuccess)
                    cudaStreamWaitEvent(s_, done_[k], 0);
                else
                    cudaStreamSynchronize(pool ? pool[k] : s_);
                cudaEventDestroy(done_[k]);
            }
        if(fork_)
            cudaEventDestroy(fork_);
    }

    // ------------------------------------------------------------ CSR containers
    lab_status csr_alloc(lab_csr_impl** out, int64_t m, int64_t n, int64_t nnz, cudaStream_t s)
    {
        LAB_ARG(m >= 0 && n >= 0 && nnz >= 0, "negative dimension");
        LAB_ARG(m < INT32_MAX && n < INT32_MAX && nnz < INT32_MAX, "int32 index range");
        lab_csr_s* A = new(std::nothrow) lab_csr_s();
        if(!A)
            return LAB_OOM;
        A->m   = m;
        A->n   = n;
        A->nnz = nnz;
        lab_status st = dalloc(&A->row_ptr, (size_t)m + 1, s);
        if(st == LAB_OK)
            st = dalloc(&A->col_ind, (size_t)(nnz > 0 ? nnz : 1), s);
        if(st == LAB_OK)
            st = dalloc(&A->val, (size_t)(nnz > 0 ? nnz : 1), s);
        if(st != LAB_OK)
        {
            csr_release(A);
            return st;
        }
        *out = A;
        return LAB_OK;
    }

    static void plan_release(spmv_plan& p)
    {
        if(p.block_row)
            cudaFree(p.block_row);
        if(p.merge_coords)
            cudaFree(p.merge_coords);
        if(p.hcnt)
            cudaFree(p.hcnt);
        if(p.hcol)
            cudaFree(p.hcol);
        if(p.hloc)
            cudaFree(p.hloc);
        p = spmv_plan();
    }

    static void lp_release(lab_csr_impl* A)
    {
        if(A->lp.f32)
            cudaFree(A->lp.f32);
        if(A->lp.bf16)
            cudaFree(A->lp.bf16);
        if(A->lp.invd32)
            cudaFree(A->lp.invd32);
        if(A->lp.dcol)
            cudaFree(A->lp.dcol);
        A->lp = csr_values_lp();
    }

    void csr_release(lab_csr_impl* A)
    {
        if(!A)
            return;
        // Freed with the synchronous call: a matrix may be released from any thread
        // after its last use on any stream.
        cudaDeviceSynchronize();
        solver_cache_forget(A);
        if(A->row_ptr)
            cudaFree(A->row_ptr);
        if(A->col_ind)
            cudaFree(A->col_ind);
        if(A->val)
            cudaFree(A->val);
        if(A->diag)
            cudaFree(A->diag);
        if(A->invdiag)
            cudaFree(A->invdiag);
        plan_release(A->plan);
        lp_release(A);
        tri_release(A);
        delete static_cast<lab_csr_s*>(A);
    }

    // ------------------------------------------------------------ validation kernel
    __global__ void k_csr_validate(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                   int64_t m, int64_t n, int64_t nnz, int* bad)
    {
        int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
        if(i <= m)
        {
            int32_t a = rp[i];
            if(a < 0 || a > nnz)
                atomicOr(bad, 1);
            if(i == 0 && a != 0)
                atomicOr(bad, 1);
            if(i == m && a != nnz)
                atomicOr(bad, 1);
            if(i < m && rp[i + 1] < a)
                atomicOr(bad, 2);
        }
        for(int64_t j = i; j < nnz; j += (int64_t)gridDim.x * blockDim.x)
        {
            int32_t c = ci[j];
            if(c < 0 || c >= n)
                atomicOr(bad, 4);
        }
    }

    // ------------------------------------------------------------ diagonal
    __global__ void k_diag(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                           const double* __restrict__ v, int64_t m, double* __restrict__ d,
                           double* __restrict__ invd)
    {
        int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
        if(i >= m)
            return;
        double dd = 0.0;
        for(int j = rp[i]; j < rp[i + 1]; j++)
            if(ci[j] == i)
            {
                dd = v[j];
                break;
            }
        if(d)
            d[i] = dd;
        if(invd)
            invd[i] = 1.0 / dd;
    }

    // Warp per row for long rows: the first diagonal entry in CSR order is the
    // lowest lane of the first 32-entry window that holds one.
    __global__ void k_diag_warp(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                const double* __restrict__ v, int64_t m, double* __restrict__ d,
                                double* __restrict__ invd)
    {
        const int64_t i    = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
        const int     lane = threadIdx.x & 31;
        if(i >= m)
            return;
        double dd = 0.0;
        for(int base = rp[i]; base < rp[i + 1]; base += 32)
        {
            const int      j   = base + lane;
            const unsigned hit = __ballot_sync(0xffffffffu, j < rp[i + 1] && ci[j] == i);
            if(hit)
            {
                dd = v[base + __ffs(hit) - 1];
                break;
            }
        }
        if(lane != 0)
            return;
        if(d)
            d[i] = dd;
        if(invd)
            invd[i] = 1.0 / dd;
    }

    lab_status diag_into(const lab_csr_impl* A, double* d, double* invd, cudaStream_t s)
    {
        if(A->m == 0)
            return LAB_OK;
        if(A->nnz > 12 * A->m)
            LAB_LAUNCH(k_diag_warp, (unsigned)ceil_div<int64_t>(A->m * 32, 256), 256, 0, s,
                       A->row_ptr, A->col_ind, (const double*)A->val, A->m, d, invd);
        else
            LAB_LAUNCH(k_diag, (unsigned)ceil_div<int64_t>(A->m, 256), 256, 0, s, A->row_ptr,
                       A->col_ind, (const double*)A->val, A->m, d, invd);
        return LAB_OK;
    }

    lab_status csr_ensure_invdiag(lab_csr_impl* A, cudaStream_t s)
    {
        if(A->invdiag)
            return LAB_OK;
        LAB_TRY(dalloc(&A->diag, (size_t)A->m + 1, s));
        LAB_TRY(dalloc(&A->invdiag, (size_t)A->m + 1, s));
        return diag_into(A, A->diag, A->invdiag, s);
    }

    // ------------------------------------------------------------ reductions
    template <int OP>
    __global__ void __launch_bounds__(kRedThreads)
        k_reduce(int64_t n, const double* __restrict__ x, const double* __restrict__ y,
                 double* __restrict__ partial, unsigned int* counter, double* out)
    {
        double acc = 0.0;
        for(int64_t i = blockIdx.x * (int64_t)kRedThreads + threadIdx.x; i < n;
            i += (int64_t)gridDim.x * kRedThreads)
        {
            if(OP == 0)
                acc += x[i] * y[i];
            else if(OP == 1)
                acc = nanmax(acc, fabs(x[i]));
            else
                acc += x[i] * x[i];
        }
        if(OP == 1)
            reduce_finish_max(acc, partial, counter, out);
        else
            reduce_finish_sum(acc, partial, counter, out);
    }

    struct red_scratch
    {
        double*       partial = nullptr;
        unsigned int* counter = nullptr;
        double*       out     = nullptr;
    };

    static lab_status get_red_scratch(red_scratch& r, cudaStream_t s)
    {
        // One scratch set per thread; reductions on one thread are stream ordered.
        static thread_local red_scratch t;
        if(!t.partial)
        {
            LAB_TRY(ensure_init());
            LAB_CUDA(cudaMalloc(&t.partial, sizeof(double) * kRedBlocks));
            LAB_CUDA(cudaMalloc(&t.counter, sizeof(unsigned int) * 4));
            LAB_CUDA(cudaMalloc(&t.out, sizeof(double) * 4));
            LAB_CUDA(cudaMemset(t.counter, 0, sizeof(unsigned int) * 4));
        }
        r = t;
        return LAB_OK;
    }

    template <int OP>
    static lab_status reduce_host(int64_t n, const double* x, const double* y, double* result,
                                  cudaStream_t s)
    {
        if(n <= 0)
        {
            *result = 0.0;
            return LAB_OK;
        }
        red_scratch r;
        LAB_TRY(get_red_scratch(r, s));
        int grid = (int)std::min<int64_t>(kRedBlocks, ceil_div<int64_t>(n, kRedThreads));
        LAB_LAUNCH(k_reduce<OP>, grid, kRedThreads, 0, s, n, x, y, r.partial, r.counter, r.out);
        return copy_d2h_sync(result, r.out, sizeof(double), s);
    }

    // ------------------------------------------------------------ scans
    constexpr int kScanThreads = 256;
    constexpr int kScanItems   = 8;
    constexpr int kScanTile    = kScanThreads * kScanItems;

    template <class T>
    __device__ T block_exclusive_scan(T v, T* smem_warp, T* total)
    {
        int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        T   inc  = v;
#pragma unroll
        for(int o = 1; o < 32; o <<= 1)
        {
            T t = __shfl_up_sync(0xffffffffu, inc, o);
            if(lane >= o)
                inc += t;
        }
        if(lane == 31)
            smem_warp[wid] = inc;
        __syncthreads();
        if(wid == 0)
        {
            T w = lane < (kScanThreads / 32) ? smem_warp[lane] : T(0);
            T wi = w;
#pragma unroll
            for(int o = 1; o < 32; o <<= 1)
            {
                T t = __shfl_up_sync(0xffffffffu, wi, o);
                if(lane >= o)
                    wi += t;
            }
            if(lane < (kScanThreads / 32))
                smem_warp[lane] = wi - w;
            if(lane == (kScanThreads / 32) - 1)
                *total = wi;
        }
        __syncthreads();
        T r = smem_warp[wid] + inc - v;
        __syncthreads();
        return r;
    }

    template <class T>
    __global__ void __launch_bounds__(kScanThreads) k_scan_tiles(T* x, int64_t n, T* bsum)
    {
        __shared__ T sw[32];
        __shared__ T tot;
        int64_t      base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
        T            s    = 0;
#pragma unroll
        for(int k = 0; k < kScanItems; k++)
            if(base + k < n)
                s += x[base + k];
        block_exclusive_scan<T>(s, sw, &tot);
        if(threadIdx.x == 0)
            bsum[blockIdx.x] = tot;
    }

    template <class T>
    __global__ void __launch_bounds__(1024) k_scan_bsums(T* bsum, int64_t nb)
    {
        __shared__ T sw[32];
        __shared__ T carry;
        if(threadIdx.x == 0)
            carry = 0;
        __syncthreads();
        for(int64_t c = 0; c < nb; c += 1024)
        {
            int64_t i    = c + threadIdx.x;
            T       v    = i < nb ? bsum[i] : T(0);
            int     lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
            T       inc  = v;
#pragma unroll
            for(int o = 1; o < 32; o <<= 1)
            {
                T t = __shfl_up_sync(0xffffffffu, inc, o);
                if(lane >= o)
                    inc += t;
            }
            if(lane == 31)
                sw[wid] = inc;
            __syncthreads();
            if(wid == 0)
            {
                T w  = sw[lane];
                T wi = w;
#pragma unroll
                for(int o = 1; o < 32; o <<= 1)
                {
                    T t = __shfl_up_sync(0xffffffffu, wi, o);
                    if(lane >= o)
                        wi += t;
                }
                sw[lane] = wi - w;
            }
            __syncthreads();
            T ex = carry + sw[wid] + inc - v;
            if(i < nb)
                bsum[i] = ex;
            __syncthreads();
            if(threadIdx.x == 1023)
                carry = ex + v;
            __syncthreads();
        }
    }

    template <class T>
    __global__ void __launch_bounds__(kScanThreads) k_scan_apply(T* x, int64_t n, const T* bsum)
    {
        __shared__ T sw[32];
        __shared__ T tot;
        int64_t      base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
        T            loc[kScanItems];
        T            s = 0;
#pragma unroll
        for(int k = 0; k < kScanItems; k++)
        {
            loc[k] = (base + k < n) ? x[base + k] : T(0);
            s += loc[k];
        }
        T ex = block_exclusive_scan<T>(s, sw, &tot) + bsum[blockIdx.x];
#pragma unroll
        for(int k = 0; k < kScanItems; k++)
        {
            if(base + k < n)
                x[base + k] = ex;
            ex += loc[k];
        }
    }

    // Short arrays (n <= kScanSmall): one CTA takes the tiles in sequence with a
    // running carry -- one launch instead of three (the setup scans many short
    // per-level arrays, where the launches cost more than the work).
    constexpr int64_t kScanSmall = 4 * kScanTile;

    // x[0..n) = exclusive scan of src[0..n_src) followed by zeros (src may be x).
    template <class T>
    __global__ void __launch_bounds__(kScanThreads)
        k_scan_small(const T* src, int64_t n_src, T* x, int64_t n)
    {
        __shared__ T sw[32];
        __shared__ T tot;
        T            carry = 0;
        for(int64_t t0 = 0; t0 < n; t0 += kScanTile)
        {
            const int64_t base = t0 + (int64_t)threadIdx.x * kScanItems;
            T             loc[kScanItems];
            T             s = 0;
#pragma unroll
            for(int k = 0; k < kScanItems; k++)
            {
                loc[k] = (base + k < n_src) ? src[base + k] : T(0);
                s += loc[k];
            }
            T ex = block_exclusive_scan<T>(s, sw, &tot) + carry;
#pragma unroll
            for(int k = 0; k < kScanItems; k++)
            {
                if(base + k < n)
                    x[base + k] = ex;
                ex += loc[k];
            }
            carry += tot; // read by every thread before the next tile's scan writes it
        }
    }

    template <class T>
    static lab_status scan_impl(T* x, int64_t n, cudaStream_t s)
    {
        if(n <= 0)
            return LAB_OK;
        if(n <= kScanSmall)
        {
            LAB_LAUNCH(k_scan_small<T>, 1, kScanThreads, 0, s, (const T*)x, n, x, n);
            return LAB_OK;
        }
        int64_t nb = ceil_div<int64_t>(n, kScanTile);
        dbuf<T> bsum;
        LAB_TRY(bsum.alloc((size_t)nb, s));
        LAB_LAUNCH(k_scan_tiles<T>, (unsigned)nb, kScanThreads, 0, s, x, n, bsum.get());
        LAB_LAUNCH(k_scan_bsums<T>, 1, 1024, 0, s, bsum.get(), nb);
        LAB_LAUNCH(k_scan_apply<T>, (unsigned)nb, kScanThreads, 0, s, x, n, bsum.get());
        return LAB_OK;
    }

    // In-place exclusive scan with caller-provided block-sum scratch
    // (bsum: ceil(n / 2048) entries); launches only, allocates nothing.
    lab_status scan_i64_into(int64_t* x, int64_t n, int64_t* bsum, cudaStream_t s)
    {
        if(n <= 0)
            return LAB_OK;
        int64_t nb = ceil_div<int64_t>(n, kScanTile);
        LAB_LAUNCH(k_scan_tiles<int64_t>, (unsigned)nb, kScanThreads, 0, s, x, n, bsum);
        LAB_LAUNCH(k_scan_bsums<int64_t>, 1, 1024, 0, s, bsum, nb);
        LAB_LAUNCH(k_scan_apply<int64_t>, (unsigned)nb, kScanThreads, 0, s, x, n,
                   (const int64_t*)bsum);
        return LAB_OK;
    }

    lab_status scan_i32(int32_t* x, int64_t n, cudaStream_t s)
    {
        return scan_impl<int32_t>(x, n, s);
    }
    lab_status scan_i64(int64_t* x, int64_t n, cudaStream_t s)
    {
        return scan_impl<int64_t>(x, n, s);
    }

    __global__ void k_counts_to_rowptr(const int32_t* counts, int32_t* rp, int64_t n)
    {
        int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
        if(i < n)
            rp[i] = counts[i];
        if(i == n)
            rp[n] = 0;
    }

    lab_status counts_to_rowptr(const int32_t* counts, int32_t* rp, int64_t n, int64_t* total,
                                cudaStream_t s)
    {
        if(n + 1 <= kScanSmall)
        {
            // one launch: the counts (and a zero for rp[n]) scanned straight into rp
            LAB_LAUNCH(k_scan_small<int32_t>, 1, kScanThreads, 0, s, counts, n, rp, n + 1);
        }
        else
        {
            if(counts != rp)
                LAB_LAUNCH(k_counts_to_rowptr, (unsigned)ceil_div<int64_t>(n + 1, 256), 256, 0, s,
                           counts, rp, n);
            else
                LAB_CUDA(cudaMemsetAsync(rp + n, 0, sizeof(int32_t), s));
            LAB_TRY(scan_i32(rp, n + 1, s));
        }
        // 64-bit total check: counts are int32 and sums above 2^31 would wrap.
        if(total)
        {
            int32_t t = 0;
            LAB_TRY(copy_d2h_sync(&t, rp + n, sizeof(int32_t), s));
            if(t < 0)
            {
                set_error("nonzero count exceeds int32 range");
                return LAB_NOT_SUPPORTED;
            }
            *total = t;
        }
        return LAB_OK;
    }

    __global__ void __launch_bounds__(kRedThreads)
        k_max_i64(const int64_t* x, int64_t n, int64_t* partial, unsigned int* counter,
                  int64_t* out)
    {
        int64_t acc = INT64_MIN;
        for(int64_t i = blockIdx.x * (int64_t)kRedThreads + threadIdx.x; i < n;
            i += (int64_t)gridDim.x * kRedThreads)
            acc = x[i] > acc ? x[i] : acc;
        reduce_finish_max_i64(acc, partial, counter, out);
    }

    lab_status max_i64(const int64_t* x, int64_t n, int64_t* result, cudaStream_t s)
    {
        if(n <= 0)
        {
            *result = INT64_MIN;
            return LAB_OK;
        }
        red_scratch r;
        LAB_TRY(get_red_scratch(r, s));
        int grid = (int)std::min<int64_t>(kRedBlocks, ceil_div<int64_t>(n, kRedThreads));
        LAB_LAUNCH(k_max_i64, grid, kRedThreads, 0, s, x, n, (int64_t*)r.partial, r.counter,
                   (int64_t*)r.out);
        return copy_d2h_sync(result, r.out, sizeof(int64_t), s);
    }

    int64_t* pinned_small()
    {
        static thread_local int64_t* p = nullptr;
        if(!p && cudaMallocHost(&p, 64 * sizeof(int64_t)) != cudaSuccess)
        {
            cudaGetLastError();
            p = nullptr;
        }
        return p;
    }

    lab_status max_i64_async(const int64_t* x, int64_t n, int64_t* host_out, cudaStream_t s)
    {
        if(n <= 0)
        {
            *host_out = INT64_MIN;
            return LAB_OK;
        }
        red_scratch r;
        LAB_TRY(get_red_scratch(r, s));
        int grid = (int)std::min<int64_t>(kRedBlocks, ceil_div<int64_t>(n, kRedThreads));
        LAB_LAUNCH(k_max_i64, grid, kRedThreads, 0, s, x, n, (int64_t*)r.partial, r.counter,
                   (int64_t*)r.out);
        LAB_CUDA(cudaMemcpyAsync(host_out, r.out, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        return LAB_OK;
    }

    // ------------------------------------------------------------ BLAS-1 kernels
    // Arithmetic follows host_axpy.cpp:35-82 operation by operation (no FMA
    // contraction: __dmul_rn / __dadd_rn), so results are bit-identical.
    __global__ void k_axpy(int64_t n, double a, const double* __restrict__ x, double* __restrict__ y)
    {
        for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
            i += (int64_t)gridDim.x * blockDim.x)
            y[i] = a == 1.0 ? __dadd_rn(x[i], y[i]) : __dadd_rn(__dmul_rn(a, x[i]), y[i]);
    }

    __global__ void k_axpby(int64_t n, double a, const double* __restrict__ x, double b,
                            double* __restrict__ y)
    {
        for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
            i += (int64_t)gridDim.x * blockDim.x)
        {
            if(a == 0.0)
                y[i] = __dmul_rn(b, y[i]);
            else if(b == 0.0)
                y[i] = __dmul_rn(a, x[i]);
            else
                y[i] = __dadd_rn(__dmul_rn(a, x[i]), __dmul_rn(b, y[i]));
        }
    }

    __global__ void k_axpbypgz(int64_t n, double a, const double* __restrict__ x, double b,
                               const double* __restrict__ y, double g, double* __restrict__ z)
    {
        for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
            i += (int64_t)gridDim.x * blockDim.x)
            z[i] = __dadd_rn(__dadd_rn(__dmul_rn(a, x[i]), __dmul_rn(b, y[i])), __dmul_rn(g, z[i]));
    }

    __global__ void k_fill(int64_t n, double v, double* __restrict__ x)
    {
        for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
            i += (int64_t)gridDim.x * blockDim.x)
            x[i] = v;
    }

    __global__ void k_jacobi_solve(int64_t n, const double* __restrict__ r,
                                   const double* __restrict__ d, double* __restrict__ x)
    {
        for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
            i += (int64_t)gridDim.x * blockDim.x)
            x[i] = __ddiv_rn(r[i], d[i]);
    }

    inline unsigned elem_grid(int64_t n)
    {
        int64_t g = ceil_div<int64_t>(n, 256);
        int64_t cap = (int64_t)num_sms() * 16;
        return (unsigned)std::max<int64_t>(1, std::min(g, cap));
    }
}

using namespace lab;

// ====================================================================== C ABI
extern "C" {

LAB_API const char* lab_status_string(lab_status s)
{
    switch(s)
    {
    case LAB_OK:
        return "ok";
    case LAB_NOT_CONVERGED:
        return "not converged";
    case LAB_BREAKDOWN:
        return "breakdown";
    case LAB_NAN:
        return "NaN in residual";
    case LAB_BAD_ARG:
        return "bad argument";
    case LAB_OOM:
        return "out of device memory";
    case LAB_TIMEOUT:
        return "device wait timed out";
    case LAB_CUDA_ERROR:
        return "CUDA error";
    case LAB_NOT_SUPPORTED:
        return "not supported";
    case LAB_NO_DEVICE:
        return "no usable CUDA device";
    }
    return "unknown status";
}

LAB_API const char* lab_last_error(void)
{
    return t_err;
}

LAB_API lab_status lab_init(int device)
{
    lab_status st = LAB_OK;
    bool       ran = false;
    std::call_once(g_init_once, [&] {
        ran           = true;
        g_init_status = do_init(device);
    });
    st = g_init_status;
    if(!ran && st == LAB_OK && device >= 0 && device != g_device)
    {
        set_error("library already bound to device %d", g_device);
        return LAB_BAD_ARG;
    }
    return st;
}

LAB_API lab_status lab_synchronize(lab_stream s)
{
    LAB_TRY(ensure_init());
    LAB_CUDA(cudaStreamSynchronize(to_stream(s)));
    return LAB_OK;
}

LAB_API int64_t lab_launch_count(void)
{
    return g_launches.load();
}

LAB_API lab_status lab_malloc(void** p, size_t bytes, lab_stream s)
{
    LAB_ARG(p, "null output");
    return dmalloc(p, bytes, to_stream(s));
}

LAB_API lab_status lab_free(void* p, lab_stream s)
{
    dfree(p, to_stream(s));
    return LAB_OK;
}

LAB_API lab_status lab_memcpy(void* dst, const void* src, size_t bytes, lab_stream s)
{
    LAB_TRY(ensure_init());
    LAB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, to_stream(s)));
    return LAB_OK;
}

LAB_API lab_status lab_csr_create(lab_csr* out, int64_t m, int64_t n, int64_t nnz,
                                  const int32_t* rp, const int32_t* ci, const double* v,
                                  lab_memory where, lab_stream ls)
{
    LAB_ARG(out, "null output handle");
    LAB_ARG(rp, "null row_ptr");
    LAB_ARG(nnz == 0 || (ci && v), "null col_ind / val");
    LAB_TRY(ensure_init());
    cudaStream_t  s = to_stream(ls);
    lab_csr_impl* A = nullptr;
    LAB_TRY(csr_alloc(&A, m, n, nnz, s));
    cudaMemcpyKind k = where == LAB_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    cudaError_t    e = cudaMemcpyAsync(A->row_ptr, rp, sizeof(int32_t) * (m + 1), k, s);
    if(e == cudaSuccess && nnz > 0)
        e = cudaMemcpyAsync(A->col_ind, ci, sizeof(int32_t) * nnz, k, s);
    if(e == cudaSuccess && nnz > 0)
        e = cudaMemcpyAsync(A->val, v, sizeof(double) * nnz, k, s);
    if(e != cudaSuccess)
    {
        csr_release(A);
        return cuda_status(e, "lab_csr_create copy", __FILE__, __LINE__);
    }
    // Structural validation on the device.
    int* bad = nullptr;
    LAB_TRY(dalloc(&bad, 1, s));
    cudaMemsetAsync(bad, 0, sizeof(int), s);
    int64_t work = std::max<int64_t>(m + 1, 1);
    k_csr_validate<<<(unsigned)std::min<int64_t>(ceil_div<int64_t>(work, 256), 65535), 256, 0,
                     s>>>(A->row_ptr, A->col_ind, m, n, nnz, bad);
    g_launches.fetch_add(1);
    int hbad = 0;
    lab_status st = copy_d2h_sync(&hbad, bad, sizeof(int), s);
    dfree(bad, s);
    if(st != LAB_OK || hbad)
    {
        csr_release(A);
        if(st != LAB_OK)
            return st;
        set_error("invalid CSR structure (flags %d: 1 row_ptr range, 2 decreasing row_ptr, "
                  "4 column out of range)",
                  hbad);
        return LAB_BAD_ARG;
    }
    *out = static_cast<lab_csr>(A);
    return LAB_OK;
}

LAB_API lab_status lab_csr_create_empty(lab_csr* out, int64_t m, int64_t n, int64_t nnz,
                                        lab_stream s)
{
    LAB_ARG(out, "null output handle");
    lab_csr_impl* A = nullptr;
    LAB_TRY(csr_alloc(&A, m, n, nnz, to_stream(s)));
    LAB_CUDA(cudaMemsetAsync(A->row_ptr, 0, sizeof(int32_t) * (m + 1), to_stream(s)));
    *out = static_cast<lab_csr>(A);
    return LAB_OK;
}

LAB_API lab_status lab_csr_destroy(lab_csr A)
{
    csr_release(A);
    return LAB_OK;
}

LAB_API lab_status lab_csr_info(lab_csr A, int64_t* m, int64_t* n, int64_t* nnz)
{
    LAB_ARG(A, "null matrix");
    if(m)
        *m = A->m;
    if(n)
        *n = A->n;
    if(nnz)
        *nnz = A->nnz;
    return LAB_OK;
}

LAB_API lab_status lab_csr_device_arrays(lab_csr A, int32_t** rp, int32_t** ci, double** v)
{
    LAB_ARG(A, "null matrix");
    if(rp)
        *rp = A->row_ptr;
    if(ci)
        *ci = A->col_ind;
    if(v)
        *v = A->val;
    return LAB_OK;
}

LAB_API lab_status lab_csr_copy_to(lab_csr A, int32_t* rp, int32_t* ci, double* v,
                                   lab_memory where, lab_stream ls)
{
    LAB_ARG(A, "null matrix");
    cudaStream_t   s = to_stream(ls);
    cudaMemcpyKind k = where == LAB_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    if(rp)
        LAB_CUDA(cudaMemcpyAsync(rp, A->row_ptr, sizeof(int32_t) * (A->m + 1), k, s));
    if(ci && A->nnz)
        LAB_CUDA(cudaMemcpyAsync(ci, A->col_ind, sizeof(int32_t) * A->nnz, k, s));
    if(v && A->nnz)
        LAB_CUDA(cudaMemcpyAsync(v, A->val, sizeof(double) * A->nnz, k, s));
    if(where == LAB_MEM_HOST)
        LAB_CUDA(cudaStreamSynchronize(s));
    return LAB_OK;
}

LAB_API lab_status lab_csr_clone(lab_csr A, lab_csr* B, lab_stream s)
{
    LAB_ARG(A && B, "null matrix");
    return lab_csr_create(B, A->m, A->n, A->nnz, A->row_ptr, A->col_ind, A->val, LAB_MEM_DEVICE,
                          s);
}

LAB_API lab_status lab_wait_timeouts(int64_t* count, lab_stream s)
{
    LAB_ARG(count, "null count");
    LAB_TRY(ensure_init());
    int* w = device_status_word();
    if(!w)
    {
        set_error("device status word unavailable");
        return LAB_CUDA_ERROR;
    }
    int h = 0;
    LAB_TRY(copy_d2h_sync(&h, w, sizeof(int), to_stream(s)));
    *count = h;
    return LAB_OK;
}

LAB_API lab_status lab_csr_values_changed(lab_csr A, lab_stream ls)
{
    LAB_ARG(A, "null matrix");
    cudaStream_t s = to_stream(ls);
    // stream-ordered: the cached arrays are released once the work already queued
    // on s (the matrix's last users) has run
    dfree(A->diag, s);
    dfree(A->invdiag, s);
    A->diag    = nullptr;
    A->invdiag = nullptr;
    dfree(A->lp.f32, s);
    dfree(A->lp.bf16, s);
    dfree(A->lp.invd32, s);
    A->lp.f32    = nullptr;
    A->lp.bf16   = nullptr;
    A->lp.invd32 = nullptr; // the 16-bit column offsets depend on the pattern only
    // a new identity: solver graphs captured on the old values (and on the cached
    // arrays just released) no longer match and are captured again
    A->uid = next_uid();
    return LAB_OK;
}

LAB_API lab_status lab_csr_structure_changed(lab_csr A, lab_stream ls)
{
    LAB_ARG(A, "null matrix");
    LAB_TRY(lab_csr_values_changed(A, ls));
    cudaStream_t s = to_stream(ls);
    dfree(A->lp.dcol, s);
    A->lp.dcol       = nullptr;
    A->lp.dcol_state = 0;
    dfree(A->plan.block_row, s);
    dfree(A->plan.merge_coords, s);
    dfree(A->plan.hcnt, s);
    dfree(A->plan.hcol, s);
    dfree(A->plan.hloc, s);
    A->plan = spmv_plan();
    if(A->tri)
    {
        LAB_CUDA(cudaStreamSynchronize(s));
        tri_release(A);
    }
    return LAB_OK;
}

LAB_API lab_status lab_axpy(int64_t n, double a, const double* x, double* y, lab_stream s)
{
    LAB_TRY(ensure_init());
    if(n <= 0)
        return LAB_OK;
    LAB_LAUNCH(k_axpy, elem_grid(n), 256, 0, to_stream(s), n, a, x, y);
    return LAB_OK;
}

LAB_API lab_status lab_axpby(int64_t n, double a, const double* x, double b, double* y,
                             lab_stream s)
{
    LAB_TRY(ensure_init());
    if(n <= 0)
        return LAB_OK;
    LAB_LAUNCH(k_axpby, elem_grid(n), 256, 0, to_stream(s), n, a, x, b, y);
    return LAB_OK;
}

LAB_API lab_status lab_axpbypgz(int64_t n, double a, const double* x, double b, const double* y,
                                double g, double* z, lab_stream s)
{
    LAB_TRY(ensure_init());
    if(n <= 0)
        return LAB_OK;
    LAB_LAUNCH(k_axpbypgz, elem_grid(n), 256, 0, to_stream(s), n, a, x, b, y, g, z);
    return LAB_OK;
}

LAB_API lab_status lab_dot(int64_t n, const double* x, const double* y, double* result,
                           lab_stream s)
{
    LAB_ARG(result, "null result");
    LAB_TRY(ensure_init());
    return reduce_host<0>(n, x, y, result, to_stream(s));
}

LAB_API lab_status lab_norm_inf(int64_t n, const double* x, double* result, lab_stream s)
{
    LAB_ARG(result, "null result");
    LAB_TRY(ensure_init());
    return reduce_host<1>(n, x, nullptr, result, to_stream(s));
}

LAB_API lab_status lab_norm_euclid(int64_t n, const double* x, double* result, lab_stream s)
{
    LAB_ARG(result, "null result");
    LAB_TRY(ensure_init());
    LAB_TRY(reduce_host<2>(n, x, nullptr, result, to_stream(s)));
    *result = std::sqrt(*result);
    return LAB_OK;
}

LAB_API lab_status lab_fill(int64_t n, double v, double* x, lab_stream s)
{
    LAB_TRY(ensure_init());
    if(n <= 0)
        return LAB_OK;
    LAB_LAUNCH(k_fill, elem_grid(n), 256, 0, to_stream(s), n, v, x);
    return LAB_OK;
}

LAB_API lab_status lab_diagonal(lab_csr A, double* d, lab_stream s)
{
    LAB_ARG(A && d, "null argument");
    if(A->m == 0)
        return LAB_OK;
    return diag_into(A, d, nullptr, to_stream(s));
}

LAB_API lab_status lab_jacobi_solve(int64_t n, const double* r, const double* d, double* x,
                                    lab_stream s)
{
    LAB_TRY(ensure_init());
    if(n <= 0)
        return LAB_OK;
    LAB_LAUNCH(k_jacobi_solve, elem_grid(n), 256, 0, to_stream(s), n, r, d, x);
    return LAB_OK;
}

LAB_API lab_status lab_exclusive_scan_i64(int64_t n, int64_t* x, lab_stream s)
{
    LAB_TRY(ensure_init());
    return scan_i64(x, n, to_stream(s));
}

LAB_API lab_status lab_exclusive_scan_i32(int64_t n, int32_t* x, lab_stream s)
{
    LAB_TRY(ensure_init());
    return scan_i32(x, n, to_stream(s));
}

} // extern "C"
