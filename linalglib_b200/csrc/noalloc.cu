// An entry point that allocates no memory: the exclusive scan with its
// block-sum scratch in a fixed file-scope device array.
//
// Who needs it: callers that cannot allocate device memory at the point of the
// call.  A process whose framework allocator has already reserved nearly all of
// the device has nothing left for a cudaMalloc; a latency-critical host thread
// cannot wait on the driver's allocator, which may synchronise; a deployment
// with a fixed memory budget forbids device allocation after start-up.  Every
// other scan entry point takes its scratch from the stream-ordered pool.
#include "internal.cuh"

#include <mutex>

namespace lab
{
    lab_status scan_i64_into(int64_t* x, int64_t n, int64_t* bsum, cudaStream_t s);

    // One block sum per 2048-element tile: 65,536 entries (512 KiB) cover
    // 134,217,728 elements.  Every GPU that loads the library holds this array
    // until the process exits.
    constexpr int64_t kNoAllocScanTiles = 65536;
    constexpr int64_t kNoAllocScanMaxN  = kNoAllocScanTiles * 2048;

    static __device__ __align__(256) int64_t g_noalloc_scan_scratch[kNoAllocScanTiles];

    // The array's name is a host-side stand-in in host code; its device address
    // is looked up once per device (with that device current) and cached.
    constexpr int     kMaxDevices = 64;
    static std::mutex g_noalloc_mu;
    static int64_t*   g_noalloc_ptr[kMaxDevices] = {};

    static lab_status noalloc_scratch(int64_t** out)
    {
        int dev = 0;
        LAB_CUDA(cudaGetDevice(&dev));
        if(dev < 0 || dev >= kMaxDevices)
        {
            set_error("device index %d out of range for the fixed scratch table", dev);
            return LAB_NOT_SUPPORTED;
        }
        std::lock_guard<std::mutex> g(g_noalloc_mu);
        if(!g_noalloc_ptr[dev])
        {
            void* p = nullptr;
            LAB_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scan_scratch));
            g_noalloc_ptr[dev] = static_cast<int64_t*>(p);
        }
        *out = g_noalloc_ptr[dev];
        return LAB_OK;
    }
}

using namespace lab;

extern "C" {

LAB_API lab_status lab_exclusive_scan_i64_noalloc(int64_t n, int64_t* x, lab_stream s)
{
    LAB_ARG(n >= 0, "negative length");
    if(n > kNoAllocScanMaxN)
    {
        set_error("lab_exclusive_scan_i64_noalloc: n = %lld exceeds the fixed scratch limit of "
                  "%lld elements (use lab_exclusive_scan_i64)",
                  (long long)n, (long long)kNoAllocScanMaxN);
        return LAB_BAD_ARG;
    }
    LAB_ARG(n == 0 || x, "null x");
    if(n == 0)
        return LAB_OK;
    LAB_TRY(ensure_init());
    int64_t* scratch = nullptr;
    LAB_TRY(noalloc_scratch(&scratch));
    // Each call writes every block sum it later reads, so nothing in the shared
    // scratch has to start at zero.
    return scan_i64_into(x, n, scratch, to_stream(s));
}

} // extern "C"
