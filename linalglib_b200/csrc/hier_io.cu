// Hierarchy (de)serialisation: write a built AMG hierarchy to a file and load
// it back onto the device, so a rerun on the same operator skips the setup.
// The reference has no such facility (its hierarchy lives only in memory,
// amg.h:65-144); the file holds exactly what the setup produced, so a loaded
// hierarchy is bit-identical to the saved one.
//
// Format (little-endian):
//   "LABHIER1"                        8-byte magic
//   int32 kind, int32 levels
//   levels+1 matrices A_0..A_L, then levels pairs P_l, R_l, each as
//     int64 m, n, nnz; int32 row_ptr[m+1]; int32 col_ind[nnz]; float64 val[nnz]
//   uint64 FNV-1a hash of every byte after the magic
#include "amg.cuh"

#include <cstdio>
#include <cstring>
#include <vector>

namespace lab
{
    namespace
    {
        constexpr char     kMagic[8]  = {'L', 'A', 'B', 'H', 'I', 'E', 'R', '1'};
        constexpr uint64_t kFnvBasis  = 1469598103934665603ull;
        constexpr uint64_t kFnvPrime  = 1099511628211ull;

        struct writer
        {
            FILE*    f    = nullptr;
            uint64_t hash = kFnvBasis;
            bool     ok   = true;
            void     put(const void* p, size_t n, bool hashed = true)
            {
                if(!ok || n == 0)
                    return;
                if(hashed)
                {
                    const unsigned char* b = static_cast<const unsigned char*>(p);
                    for(size_t i = 0; i < n; i++)
                        hash = (hash ^ b[i]) * kFnvPrime;
                }
                ok = std::fwrite(p, 1, n, f) == n;
            }
        };

        struct reader
        {
            FILE*    f    = nullptr;
            uint64_t hash = kFnvBasis;
            bool     ok   = true;
            void     get(void* p, size_t n, bool hashed = true)
            {
                if(!ok || n == 0)
                    return;
                ok = std::fread(p, 1, n, f) == n;
                if(ok && hashed)
                {
                    const unsigned char* b = static_cast<const unsigned char*>(p);
                    for(size_t i = 0; i < n; i++)
                        hash = (hash ^ b[i]) * kFnvPrime;
                }
            }
        };

        lab_status write_csr(writer& w, const lab_csr_impl* A, cudaStream_t s)
        {
            const int64_t        dims[3] = {A->m, A->n, A->nnz};
            std::vector<int32_t> rp((size_t)A->m + 1), ci((size_t)A->nnz);
            std::vector<double>  v((size_t)A->nnz);
            LAB_TRY(copy_d2h_sync(rp.data(), A->row_ptr, sizeof(int32_t) * rp.size(), s));
            if(A->nnz > 0)
            {
                LAB_TRY(copy_d2h_sync(ci.data(), A->col_ind, sizeof(int32_t) * ci.size(), s));
                LAB_TRY(copy_d2h_sync(v.data(), A->val, sizeof(double) * v.size(), s));
            }
            w.put(dims, sizeof(dims));
            w.put(rp.data(), sizeof(int32_t) * rp.size());
            w.put(ci.data(), sizeof(int32_t) * ci.size());
            w.put(v.data(), sizeof(double) * v.size());
            return LAB_OK;
        }

        lab_status read_csr(reader& r, lab_csr_impl** out, cudaStream_t s)
        {
            int64_t dims[3] = {0, 0, 0};
            r.get(dims, sizeof(dims));
            if(!r.ok || dims[0] < 0 || dims[1] < 0 || dims[2] < 0 || dims[0] >= INT32_MAX ||
               dims[1] >= INT32_MAX || dims[2] >= INT32_MAX)
            {
                set_error("hierarchy file: bad matrix header");
                return LAB_BAD_ARG;
            }
            std::vector<int32_t> rp((size_t)dims[0] + 1), ci((size_t)dims[2]);
            std::vector<double>  v((size_t)dims[2]);
            r.get(rp.data(), sizeof(int32_t) * rp.size());
            r.get(ci.data(), sizeof(int32_t) * ci.size());
            r.get(v.data(), sizeof(double) * v.size());
            if(!r.ok)
            {
                set_error("hierarchy file: truncated matrix data");
                return LAB_BAD_ARG;
            }
            lab_csr A = nullptr;
            // the library's own constructor: copies to the device and validates the structure
            LAB_TRY(lab_csr_create(&A, dims[0], dims[1], dims[2], rp.data(), ci.data(), v.data(),
                                   LAB_MEM_HOST, s));
            *out = static_cast<lab_csr_impl*>(A);
            return LAB_OK;
        }
    }
}

using namespace lab;

extern "C" {

LAB_API lab_status lab_hierarchy_save(lab_hierarchy h, const char* path, lab_stream ls)
{
    LAB_ARG(h && path, "null argument");
    LAB_TRY(ensure_init());
    cudaStream_t s = to_stream(ls);
    writer       w;
    w.f = std::fopen(path, "wb");
    if(!w.f)
    {
        set_error("lab_hierarchy_save: cannot open %s for writing", path);
        return LAB_BAD_ARG;
    }
    w.put(kMagic, sizeof(kMagic), false);
    const int32_t head[2] = {h->kind, h->levels};
    w.put(head, sizeof(head));
    lab_status st = LAB_OK;
    for(int l = 0; l <= h->levels && st == LAB_OK; l++)
        st = write_csr(w, h->A[l], s);
    for(int l = 0; l < h->levels && st == LAB_OK; l++)
    {
        st = write_csr(w, h->P[l], s);
        if(st == LAB_OK)
            st = write_csr(w, h->R[l], s);
    }
    const uint64_t hash = w.hash;
    w.put(&hash, sizeof(hash), false);
    const bool closed = std::fclose(w.f) == 0;
    if(st != LAB_OK)
        return st;
    if(!w.ok || !closed)
    {
        set_error("lab_hierarchy_save: write to %s failed", path);
        return LAB_BAD_ARG;
    }
    return LAB_OK;
}

LAB_API lab_status lab_hierarchy_load(const char* path, lab_hierarchy* out, lab_stream ls)
{
    LAB_ARG(path && out, "null argument");
    LAB_TRY(ensure_init());
    cudaStream_t s = to_stream(ls);
    reader       r;
    r.f = std::fopen(path, "rb");
    if(!r.f)
    {
        set_error("lab_hierarchy_load: cannot open %s", path);
        return LAB_BAD_ARG;
    }
    char magic[8] = {};
    r.get(magic, sizeof(magic), false);
    int32_t head[2] = {-1, -1};
    r.get(head, sizeof(head));
    if(!r.ok || std::memcmp(magic, kMagic, sizeof(kMagic)) != 0 || head[0] < LAB_AMG_SA ||
       head[0] > LAB_AMG_RS || head[1] < 0 || head[1] > kMaxLevels)
    {
        std::fclose(r.f);
        set_error("lab_hierarchy_load: %s is not a hierarchy file", path);
        return LAB_BAD_ARG;
    }
    lab_hier_s* h = new(std::nothrow) lab_hier_s();
    if(!h)
    {
        std::fclose(r.f);
        return LAB_OOM;
    }
    h->kind       = head[0];
    h->levels     = head[1];
    lab_status st = LAB_OK;
    for(int l = 0; l <= h->levels && st == LAB_OK; l++)
        st = read_csr(r, &h->A[l], s);
    for(int l = 0; l < h->levels && st == LAB_OK; l++)
    {
        st = read_csr(r, &h->P[l], s);
        if(st == LAB_OK)
            st = read_csr(r, &h->R[l], s);
    }
    const uint64_t computed = r.hash;
    uint64_t       stored   = 0;
    if(st == LAB_OK)
    {
        r.get(&stored, sizeof(stored), false);
        if(!r.ok || stored != computed)
        {
            set_error("lab_hierarchy_load: %s is corrupt (checksum mismatch)", path);
            st = LAB_BAD_ARG;
        }
    }
    std::fclose(r.f);
    // shapes must chain: A_l is m_l x m_l, P_l is m_l x m_{l+1}, R_l is m_{l+1} x m_l
    for(int l = 0; l < h->levels && st == LAB_OK; l++)
    {
        const int64_t m = h->A[l]->m, mc = h->A[l + 1]->m;
        if(h->A[l]->n != m || h->P[l]->m != m || h->P[l]->n != mc || h->R[l]->m != mc ||
           h->R[l]->n != m)
        {
            set_error("lab_hierarchy_load: level %d shapes do not chain", l);
            st = LAB_BAD_ARG;
        }
    }
    if(st == LAB_OK)
        st = hierarchy_plans(h, s);
    if(st != LAB_OK)
    {
        hierarchy_release(h);
        return st;
    }
    *out = h;
    return LAB_OK;
}

} // extern "C"
