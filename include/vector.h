// linalg::vector<T> -- the reference container (library/include/vector.h:57-210)
// with the same public interface, backed by a coherent host/device mirror.
//
// is_on_host() reports where the caller placed the vector (move_to_device /
// move_to_host, as in the reference).  Every computation runs on the GPU: a
// host-resident vector is uploaded on first use by a device operation and its
// host copy refreshed lazily when element access needs it, so code written for
// the reference's host backend runs unchanged.  get_vec() returns the pointer of
// the current residency (host memory for host vectors, device memory otherwise).
#ifndef LINALG_B200_VECTOR_H
#define LINALG_B200_VECTOR_H

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace linalg
{
    template <typename T>
    class vector
    {
    private:
        mutable std::vector<T> h;             // host mirror
        mutable T*             d     = nullptr; // device copy (library pool)
        mutable size_t         dcap  = 0;
        mutable int            valid = 1;       // bit 0: host copy valid, bit 1: device copy valid
        size_t                 n     = 0;
        bool                   on_host = true;

        void sync_host() const;
        void sync_device() const;

    public:
        vector();
        vector(size_t size);
        vector(size_t size, T val);
        vector(const std::vector<T>& vec);
        ~vector();

        vector(const vector&)            = delete;
        vector& operator=(const vector&) = delete;

        T&       operator[](size_t index);
        const T& operator[](size_t index) const;

        bool     is_on_host() const;
        size_t   get_size() const;
        T*       get_vec();
        const T* get_vec() const;
        void     resize(size_t size);
        void     resize(size_t size, T val);
        void     clear();
        void     copy_from(const vector& x);
        void     zeros();
        void     ones();
        void     rand(T min, T max);
        void     fill(T val);
        void     move_to_device();
        void     move_to_host();
        void     print_vector(const std::string name) const;

        // -- library access (not in the reference interface) --------------
        // Device pointer with the current contents (uploads if needed).
        const T* device_read() const;
        // Device pointer the caller will overwrite; the host copy becomes stale.
        T* device_write();
        // Device pointer read and written (upload if needed, host copy stale).
        T* device_readwrite();
    };
}

#endif
