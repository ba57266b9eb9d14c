// Deterministic block / grid reductions.
//
// Every reduction has a fixed shape: thread-sequential partial sums, a fixed
// xor-shuffle tree per warp, a fixed tree over warps, one partial per block, and
// the LAST block to finish (atomic ticket) sums the partials in index order.
// The result therefore does not depend on block scheduling, and a reduction
// is bit-reproducible run to run for a given grid size.
#pragma once

#include "internal.cuh"

namespace lab
{
    // Block-wide sum; the result is valid in every thread of warp 0.
    template <int NT>
    __device__ __forceinline__ double block_sum(double v)
    {
        __shared__ double sw[NT / 32];
        v        = warp_sum(v);
        int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        if(lane == 0)
            sw[wid] = v;
        __syncthreads();
        double r = 0.0;
        if(wid == 0)
        {
            r = lane < NT / 32 ? sw[lane] : 0.0;
            r = warp_sum(r);
        }
        __syncthreads();
        return r;
    }

    template <int NT>
    __device__ __forceinline__ double block_max(double v)
    {
        __shared__ double sw[NT / 32];
        v        = warp_max(v);
        int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        if(lane == 0)
            sw[wid] = v;
        __syncthreads();
        double r = 0.0;
        if(wid == 0)
        {
            r = lane < NT / 32 ? sw[lane] : 0.0;
            r = warp_max(r);
        }
        __syncthreads();
        return r;
    }

    // Returns true in every thread of the block that finished last.
    __device__ __forceinline__ bool grid_ticket(unsigned int* counter)
    {
        __shared__ bool last;
        __syncthreads();
        if(threadIdx.x == 0)
        {
            __threadfence();
            unsigned int t = atomicAdd(counter, 1u);
            last           = (t == gridDim.x - 1);
        }
        __syncthreads();
        return last;
    }

    template <int NT = 256>
    __device__ void reduce_finish_sum(double acc, double* partial, unsigned int* counter,
                                      double* out)
    {
        double b = block_sum<NT>(acc);
        if(threadIdx.x == 0)
            partial[blockIdx.x] = b;
        if(grid_ticket(counter))
        {
            double s = 0.0;
            for(unsigned i = threadIdx.x; i < gridDim.x; i += NT)
                s += __ldcg(partial + i);
            s = block_sum<NT>(s);
            if(threadIdx.x == 0)
            {
                *out     = s;
                *counter = 0;
            }
        }
    }

    template <int NT = 256>
    __device__ void reduce_finish_max(double acc, double* partial, unsigned int* counter,
                                      double* out)
    {
        double b = block_max<NT>(acc);
        if(threadIdx.x == 0)
            partial[blockIdx.x] = b;
        if(grid_ticket(counter))
        {
            double s = 0.0;
            for(unsigned i = threadIdx.x; i < gridDim.x; i += NT)
                s = nanmax(s, __ldcg(partial + i));
            s = block_max<NT>(s);
            if(threadIdx.x == 0)
            {
                *out     = s;
                *counter = 0;
            }
        }
    }

    __device__ __forceinline__ int64_t warp_max_i64(int64_t v)
    {
#pragma unroll
        for(int o = 16; o > 0; o >>= 1)
        {
            int64_t t = __shfl_xor_sync(0xffffffffu, v, o);
            v         = t > v ? t : v;
        }
        return v;
    }

    __device__ inline void reduce_finish_max_i64(int64_t acc, int64_t* partial,
                                                 unsigned int* counter, int64_t* out)
    {
        __shared__ int64_t sw[8];
        acc      = warp_max_i64(acc);
        int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        if(lane == 0)
            sw[wid] = acc;
        __syncthreads();
        if(wid == 0)
        {
            int64_t r = lane < 8 ? sw[lane] : INT64_MIN;
            r         = warp_max_i64(r);
            if(lane == 0)
                partial[blockIdx.x] = r;
        }
        if(grid_ticket(counter))
        {
            int64_t s = INT64_MIN;
            for(unsigned i = threadIdx.x; i < gridDim.x; i += 256)
            {
                int64_t t = __ldcg((const long long*)partial + i);
                s         = t > s ? t : s;
            }
            s = warp_max_i64(s);
            __syncthreads();
            if(lane == 0)
                sw[wid] = s;
            __syncthreads();
            if(threadIdx.x == 0)
            {
                int64_t r = INT64_MIN;
                for(int w = 0; w < 8; w++)
                    r = sw[w] > r ? sw[w] : r;
                *out     = r;
                *counter = 0;
            }
        }
    }
}
