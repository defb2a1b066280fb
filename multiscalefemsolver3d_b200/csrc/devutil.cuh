// Device helpers: deterministic reductions, streaming loads.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace msfem {

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;  // valid in lane 0
}

// Block-wide sum of up to three values with a fixed combination order (warp
// shuffles, then warp 0 over the per-warp results).  Result valid in thread 0.
template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K], double* sh /* [32*K] */)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < K; k++) v[k] = warp_sum(v[k]);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < K; k++) sh[k * 32 + warp] = v[k];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < K; k++) {
            double t = lane < nw ? sh[k * 32 + lane] : 0.0;
            v[k] = warp_sum(t);
        }
    }
    __syncthreads();
}

// Called by every thread of every block after thread 0 has stored the block's
// partial results.  Returns true (in all threads) in the block that arrives last;
// that block then owns the final reduction and resets the ticket.
__device__ __forceinline__ bool arrive_last(unsigned int* ticket)
{
    __shared__ bool am_last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        unsigned int t = atomicAdd(ticket, 1u);
        am_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (am_last) __threadfence();
    return am_last;
}

// Final reduction of `count` partials (stride `stride` apart, K series) by one
// block in a fixed order.  Result valid in thread 0.
template <int K>
__device__ __forceinline__ void reduce_partials(const double* partial, int count, int stride, double (&out)[K],
                                                double* sh)
{
    // Eight independent loads are issued before they are added, so the final
    // reduction costs about one L2 round trip per 8*blockDim partials instead of
    // one per blockDim (a plain `t += load` loop serialises on every load).  The
    // summation order is fixed, so the result is the same on every run.
#pragma unroll
    for (int k = 0; k < K; k++) {
        const double* p = partial + (size_t)k * stride;
        const int step = blockDim.x;
        double t = 0.0;
        int i = threadIdx.x;
        for (; i + 7 * step < count; i += 8 * step) {
            double a[8];
#pragma unroll
            for (int j = 0; j < 8; j++) a[j] = __ldcg(p + i + j * step);
#pragma unroll
            for (int j = 0; j < 8; j++) t += a[j];
        }
        for (; i < count; i += step) t += __ldcg(p + i);
        out[k] = t;
    }
    block_sum<K>(out, sh);
}

template <class T>
__device__ __forceinline__ T ld_stream(const T* p)
{
    return __ldcs(p);
}

__host__ __device__ __forceinline__ unsigned int hash32(unsigned int x)
{
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}

}  // namespace msfem
