// SELL-32 row kernels shared by the SpMV and the fused Krylov kernels.
#pragma once

#include "devutil.cuh"
#include "internal.cuh"

namespace msfem {

template <class VT>
struct SellView {
    int n_slices, bs, n_rows, n_brows;
    const int64_t* sp;
    const int32_t* col;
    const int16_t* col16;  // non-null: scalar columns stored as 16-bit deltas from min(row, n_rows-1)
    const VT* val;
};

template <class VT>
SellView<VT> sell_view(System& s);
unsigned spmv_grid(const System& s);                          // one warp per slice
unsigned spmv_grid_of(const void* kernel, const System& s);   // slice-strided, one full wave

template <class VT>
struct Vec4;
template <>
struct Vec4<float> {
    static __device__ __forceinline__ void load(const float* p, float (&v)[4])
    {
        const float4 q = __ldcs(reinterpret_cast<const float4*>(p));
        v[0] = q.x;
        v[1] = q.y;
        v[2] = q.z;
        v[3] = q.w;
    }
};
template <>
struct Vec4<double> {
    static __device__ __forceinline__ void load(const double* p, double (&v)[4])
    {
        const double2 a = __ldcs(reinterpret_cast<const double2*>(p));
        const double2 b = __ldcs(reinterpret_cast<const double2*>(p) + 1);
        v[0] = a.x;
        v[1] = a.y;
        v[2] = b.x;
        v[3] = b.y;
    }
};

// Row `warp*32 + lane` of a scalar SELL slice times x.  All lanes of the warp
// must call it (the loop runs to the slice width).
// 4 consecutive 16-bit column deltas of one lane (one 8-byte load)
__device__ __forceinline__ void load_delta4(const int16_t* p, int row0, int (&c)[4])
{
    const int2 q = __ldcs(reinterpret_cast<const int2*>(p));
    c[0] = row0 + (int)(short)(q.x & 0xffff);
    c[1] = row0 + (int)(short)((unsigned)q.x >> 16);
    c[2] = row0 + (int)(short)(q.y & 0xffff);
    c[3] = row0 + (int)(short)((unsigned)q.y >> 16);
}

template <class VT>
__device__ __forceinline__ VT sell_row_scalar16(const SellView<VT>& A, int warp, int lane, const VT* __restrict__ x)
{
    const int64_t base = A.sp[warp];
    const int w = (int)((A.sp[warp + 1] - base) >> 5);
    const int row0 = min(warp * kSlice + lane, A.n_rows - 1);
    const int16_t* cp = A.col16 + base + lane * kChunk;
    const VT* vp = A.val + base + lane * kChunk;
    VT acc = 0;
    int k = 0;
    for (; k + 4 * kChunk <= w; k += 4 * kChunk) {
        int c[4][4];
        VT v[4][4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            load_delta4(cp + (int64_t)(k + q * kChunk) * kSlice, row0, c[q]);
            Vec4<VT>::load(vp + (int64_t)(k + q * kChunk) * kSlice, v[q]);
        }
        VT xs[4][4];
#pragma unroll
        for (int q = 0; q < 4; q++)
#pragma unroll
            for (int e = 0; e < 4; e++) xs[q][e] = __ldg(x + c[q][e]);
#pragma unroll
        for (int q = 0; q < 4; q++)
#pragma unroll
            for (int e = 0; e < 4; e++) acc += v[q][e] * xs[q][e];
    }
    for (; k < w; k += kChunk) {
        int c[4];
        VT v[4];
        load_delta4(cp + (int64_t)k * kSlice, row0, c);
        Vec4<VT>::load(vp + (int64_t)k * kSlice, v);
#pragma unroll
        for (int e = 0; e < 4; e++) acc += v[e] * __ldg(x + c[e]);
    }
    return acc;
}

template <class VT>
__device__ __forceinline__ VT sell_row_scalar(const SellView<VT>& A, int warp, int lane, const VT* __restrict__ x)
{
    if (A.col16) return sell_row_scalar16<VT>(A, warp, lane, x);
    const int64_t base = A.sp[warp];
    const int w = (int)((A.sp[warp + 1] - base) >> 5);
    const int32_t* cp = A.col + base + lane * kChunk;
    const VT* vp = A.val + base + lane * kChunk;
    VT acc = 0;
    int k = 0;
    if constexpr (sizeof(VT) == 4) {
        // FP32: issue the column and value loads of 4 chunks (16 entries, a whole
        // interior Kuhn row) before the dependent x gathers, so that each warp
        // keeps 16 independent 128-bit loads in flight instead of 2
        for (; k + 4 * kChunk <= w; k += 4 * kChunk) {
            int4 c[4];
            VT v[4][4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                c[q] = __ldcs(reinterpret_cast<const int4*>(cp + (int64_t)(k + q * kChunk) * kSlice));
                Vec4<VT>::load(vp + (int64_t)(k + q * kChunk) * kSlice, v[q]);
            }
            VT xs[4][4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                xs[q][0] = __ldg(x + c[q].x);
                xs[q][1] = __ldg(x + c[q].y);
                xs[q][2] = __ldg(x + c[q].z);
                xs[q][3] = __ldg(x + c[q].w);
            }
#pragma unroll
            for (int q = 0; q < 4; q++)
#pragma unroll
                for (int e = 0; e < 4; e++) acc += v[q][e] * xs[q][e];
        }
    }
#pragma unroll 2
    for (; k < w; k += kChunk) {
        const int4 c = __ldcs(reinterpret_cast<const int4*>(cp + (int64_t)k * kSlice));
        VT v[4];
        Vec4<VT>::load(vp + (int64_t)k * kSlice, v);
        acc += v[0] * __ldg(x + c.x);
        acc += v[1] * __ldg(x + c.y);
        acc += v[2] * __ldg(x + c.z);
        acc += v[3] * __ldg(x + c.w);
    }
    return acc;
}

// Block row `warp*32 + lane` of a 3x3-block SELL slice times x (x node-major).
template <class VT>
__device__ __forceinline__ void sell_row_block(const SellView<VT>& A, int warp, int lane, const VT* __restrict__ x,
                                               VT (&acc)[3])
{
    const int64_t base = A.sp[warp];
    const int w = (int)((A.sp[warp + 1] - base) >> 5);
    acc[0] = acc[1] = acc[2] = 0;
#pragma unroll 2
    for (int k = 0; k < w; k++) {
        const int64_t blk = base + (int64_t)k * kSlice;
        const int c = __ldcs(A.col + blk + lane);
        const VT* vb = A.val + 9 * blk + lane;
        const VT x0 = __ldg(x + 3 * (int64_t)c), x1 = __ldg(x + 3 * (int64_t)c + 1), x2 = __ldg(x + 3 * (int64_t)c + 2);
        VT v[9];
#pragma unroll
        for (int e = 0; e < 9; e++) v[e] = __ldcs(vb + e * kSlice);
        acc[0] += v[0] * x0 + v[1] * x1 + v[2] * x2;
        acc[1] += v[3] * x0 + v[4] * x1 + v[5] * x2;
        acc[2] += v[6] * x0 + v[7] * x1 + v[8] * x2;
    }
}

}  // namespace msfem
