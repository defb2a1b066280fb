// SELL-32 copies of the assembled matrix and the SpMV kernels
// (the role of CSSD_Matrix::MultiplicationMatrixVector, CSSD_Matrix.h:395-423).
//
// One warp owns a slice of 32 consecutive rows (scalar) or block rows
// (elasticity), one lane per row, and walks the slice's columns in lock step.
// Values and column indices are stored column-major inside a slice, so every
// warp-wide load is one contiguous, fully used segment:
//   scalar: lanes read 4 consecutive entries each as 128-bit loads (int4 for
//           the columns, float4 / 2 x double2 for the values), 512 B per warp
//           instruction for FP32 values and columns;
//   3x3 blocks: one column index per block and 9 coalesced value loads of 32
//           lanes each; the x gather reads the 3 components of the column node.
// The matrix is read once per product with streaming (evict-first) loads so
// that the Krylov vectors, which are re-read every iteration, stay in the
// 126 MB L2.  The diagonal is kept at its sorted place, so a row's sum runs
// in column order.
#include <cub/cub.cuh>

#include "devutil.cuh"
#include "internal.cuh"
#include "spmv.cuh"

namespace msfem {
namespace {

inline unsigned grid_for(int64_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }

// slice widths: entries per lane (scalar, rounded up to kChunk) or blocks per lane
__global__ void k_slice_width(int n_rows, int n_slices, const int32_t* __restrict__ rp, int round_to, int64_t* w_out)
{
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= n_slices) return;
    const int row = warp * kSlice + lane;
    int len = row < n_rows ? rp[row + 1] - rp[row] : 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) len = max(len, __shfl_xor_sync(0xffffffffu, len, o));
    if (lane == 0) {
        int w = (len + round_to - 1) / round_to * round_to;
        w_out[warp] = (int64_t)w * kSlice;
    }
}

__global__ void k_sell_pattern_scalar(int n_rows, const int32_t* __restrict__ rp, const int32_t* __restrict__ ncol,
                                      const int64_t* __restrict__ sp, int32_t* __restrict__ col)
{
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    const int slice = row / kSlice, lane = row % kSlice;
    if (slice >= (n_rows + kSlice - 1) / kSlice) return;
    const int64_t base = sp[slice];
    const int w = (int)((sp[slice + 1] - base) / kSlice);
    const int b = row < n_rows ? rp[row] : 0, len = row < n_rows ? rp[row + 1] - b : 0;
    const int pad = row < n_rows ? row : 0;
    for (int k = 0; k < w; k++) {
        const int64_t pos = base + (int64_t)(k / kChunk) * (kSlice * kChunk) + lane * kChunk + (k % kChunk);
        col[pos] = k < len ? ncol[b + k] : pad;
    }
}

// 16-bit deltas of the scalar SELL columns from min(row, n-1); flags overflow
__global__ void k_sell_delta16(int n_rows, int n_slices, const int64_t* __restrict__ sp, const int32_t* __restrict__ col,
                               int16_t* __restrict__ col16, int* overflow)
{
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    const int slice = row / kSlice, lane = row % kSlice;
    if (slice >= n_slices) return;
    const int64_t base = sp[slice];
    const int w = (int)((sp[slice + 1] - base) / kSlice);
    const int row0 = min(row, n_rows - 1);
    for (int k = 0; k < w; k++) {
        const int64_t pos = base + (int64_t)(k / kChunk) * (kSlice * kChunk) + lane * kChunk + (k % kChunk);
        const int c = row < n_rows ? col[pos] : row0;
        const int d = c - row0;
        if (d < -32768 || d > 32767) atomicExch(overflow, 1);
        col16[pos] = (int16_t)d;
    }
}

// v64 = A; v32 = D^-1/2 A D^-1/2 (the Jacobi-scaled matrix the FP32 inner solves use), scale = 1/sqrt|a_ii|
__global__ void k_sell_values_scalar(int n_rows, const int32_t* __restrict__ rp, const int32_t* __restrict__ ncol,
                                     const double* __restrict__ val, const double* __restrict__ scale,
                                     const int64_t* __restrict__ sp, double* __restrict__ v64, float* __restrict__ v32)
{
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    const int slice = row / kSlice, lane = row % kSlice;
    if (slice >= (n_rows + kSlice - 1) / kSlice) return;
    const int64_t base = sp[slice];
    const int w = (int)((sp[slice + 1] - base) / kSlice);
    const int b = row < n_rows ? rp[row] : 0, len = row < n_rows ? rp[row + 1] - b : 0;
    const double si = row < n_rows ? scale[row] : 0.0;
    for (int k = 0; k < w; k++) {
        const int64_t pos = base + (int64_t)(k / kChunk) * (kSlice * kChunk) + lane * kChunk + (k % kChunk);
        const double v = k < len ? val[b + k] : 0.0;
        v64[pos] = v;
        v32[pos] = k < len ? (float)(v * si * scale[ncol[b + k]]) : 0.0f;
    }
}

__global__ void k_sell_pattern_block(int n_brows, const int32_t* __restrict__ rp, const int32_t* __restrict__ ncol,
                                     const int64_t* __restrict__ sp, int32_t* __restrict__ col)
{
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    const int slice = row / kSlice, lane = row % kSlice;
    if (slice >= (n_brows + kSlice - 1) / kSlice) return;
    const int64_t base = sp[slice];
    const int w = (int)((sp[slice + 1] - base) / kSlice);
    const int b = row < n_brows ? rp[row] : 0, len = row < n_brows ? rp[row + 1] - b : 0;
    const int pad = row < n_brows ? row : 0;
    for (int k = 0; k < w; k++) col[base + (int64_t)k * kSlice + lane] = k < len ? ncol[b + k] : pad;
}

__global__ void k_sell_values_block(int n_brows, const int32_t* __restrict__ rp, const int32_t* __restrict__ ncol,
                                    const double* __restrict__ val, const double* __restrict__ scale,
                                    const int64_t* __restrict__ sp, double* __restrict__ v64, float* __restrict__ v32)
{
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    const int slice = row / kSlice, lane = row % kSlice;
    if (slice >= (n_brows + kSlice - 1) / kSlice) return;
    const int64_t base = sp[slice];
    const int w = (int)((sp[slice + 1] - base) / kSlice);
    const int b = row < n_brows ? rp[row] : 0, len = row < n_brows ? rp[row + 1] - b : 0;
    for (int k = 0; k < w; k++) {
        const int64_t blk = 9 * (base + (int64_t)k * kSlice) + lane;
        const int j = k < len ? ncol[b + k] : 0;
        for (int e = 0; e < 9; e++) {
            const double v = k < len ? val[9 * (int64_t)(b + k) + e] : 0.0;
            v64[blk + (int64_t)e * kSlice] = v;
            v32[blk + (int64_t)e * kSlice] =
                k < len ? (float)(v * scale[3 * (int64_t)row + e / 3] * scale[3 * (int64_t)j + e % 3]) : 0.0f;
        }
    }
}

// diagonal of the scalar rows and its inverses
__global__ void k_diag(int n_rows, int bs, const int32_t* __restrict__ rp, const int32_t* __restrict__ ncol,
                       const double* __restrict__ val, double* __restrict__ d64, double* __restrict__ di64,
                       float* __restrict__ di32, double* __restrict__ scale, int* bad)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_rows) return;
    const int node = bs == 1 ? r : r / 3, a = bs == 1 ? 0 : r - 3 * (r / 3);
    double d = 0.0;
    for (int p = rp[node]; p < rp[node + 1]; p++)
        if (ncol[p] == node) d = bs == 1 ? val[p] : val[9 * (int64_t)p + 4 * a];
    d64[r] = d;
    if (d == 0.0) {
        atomicExch(bad, 1);
        di64[r] = 0.0;
        di32[r] = 0.0f;
        scale[r] = 1.0;
    } else {
        di64[r] = 1.0 / d;
        di32[r] = (float)(1.0 / d);
        scale[r] = 1.0 / sqrt(fabs(d));
    }
}

template <class VT>
__global__ void __launch_bounds__(256) k_spmv(SellView<VT> A, const VT* __restrict__ x, VT* __restrict__ y)
{
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; warp < A.n_slices; warp += nw) {
        if (A.bs == 1) {
            const VT acc = sell_row_scalar<VT>(A, warp, lane, x);
            const int row = warp * kSlice + lane;
            if (row < A.n_rows) y[row] = acc;
        } else {
            VT acc[3];
            sell_row_block<VT>(A, warp, lane, x, acc);
            const int brow = warp * kSlice + lane;
            if (brow < A.n_brows) {
                y[3 * (int64_t)brow] = acc[0];
                y[3 * (int64_t)brow + 1] = acc[1];
                y[3 * (int64_t)brow + 2] = acc[2];
            }
        }
    }
}

// r = f - A x and the block partial of (r, r); the last block stores the total
__global__ void __launch_bounds__(256) k_residual(SellView<double> A, const double* __restrict__ x,
                                                  const double* __restrict__ f, double* __restrict__ r,
                                                  double* __restrict__ partial, unsigned int* ticket,
                                                  double* __restrict__ out)
{
    __shared__ double sh[32];
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    double rr[1] = {0.0};
    for (int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; warp < A.n_slices; warp += nw) {
        if (A.bs == 1) {
            const double acc = sell_row_scalar<double>(A, warp, lane, x);
            const int row = warp * kSlice + lane;
            if (row < A.n_rows) {
                const double v = f[row] - acc;
                r[row] = v;
                rr[0] += v * v;
            }
        } else {
            double acc[3];
            sell_row_block<double>(A, warp, lane, x, acc);
            const int brow = warp * kSlice + lane;
            if (brow < A.n_brows)
                for (int c = 0; c < 3; c++) {
                    const double v = f[3 * (int64_t)brow + c] - acc[c];
                    r[3 * (int64_t)brow + c] = v;
                    rr[0] += v * v;
                }
        }
    }
    block_sum<1>(rr, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = rr[0];
    if (arrive_last(ticket)) {
        double tot[1];
        reduce_partials<1>(partial, gridDim.x, 0, tot, sh);
        if (threadIdx.x == 0) {
            *out = tot[0];
            *ticket = 0;
        }
    }
}

}  // namespace

// Times the FP32 product with the 32-bit columns and with the 16-bit deltas (3 warm-up and 20
// timed launches each, on the system's stream) and keeps the faster for every later FP32 product.
static int tune_fp32_columns(System& s)
{
    Sell& S = s.sell;
    cudaStream_t st = s.stream;
    DBuf<float> xy;
    MSFEM_TRY(xy.alloc(2 * (size_t)s.n_rows));
    MSFEM_CK(cudaMemsetAsync(xy.p, 0, sizeof(float) * 2 * (size_t)s.n_rows, st));
    cudaEvent_t e[2];
    MSFEM_CK(cudaEventCreate(&e[0]));
    MSFEM_CK(cudaEventCreate(&e[1]));
    const unsigned g = spmv_grid_of((const void*)k_spmv<float>, s);
    for (int variant = 0; variant < 2; variant++) {
        S.fp32_col16 = variant;
        const SellView<float> v = sell_view<float>(s);
        for (int i = 0; i < 3; i++) k_spmv<float><<<g, 256, 0, st>>>(v, xy.p, xy.p + s.n_rows);
        MSFEM_CK(cudaEventRecord(e[0], st));
        for (int i = 0; i < 20; i++) k_spmv<float><<<g, 256, 0, st>>>(v, xy.p, xy.p + s.n_rows);
        MSFEM_CK(cudaEventRecord(e[1], st));
        MSFEM_CK(cudaEventSynchronize(e[1]));
        MSFEM_CK(cudaEventElapsedTime(&S.tune_ms[variant], e[0], e[1]));
        S.tune_ms[variant] /= 20.f;
    }
    cudaEventDestroy(e[0]);
    cudaEventDestroy(e[1]);
    MSFEM_CK(cudaGetLastError());
    S.fp32_col16 = S.tune_ms[1] < S.tune_ms[0] ? 1 : 0;
    s.total_launches += 46;
    return MSFEM_OK;
}

int prepare_sell(System& s)
{
    Sell& S = s.sell;
    cudaStream_t st = s.stream;
    const int nbr = s.n_nodes;  // rows of the node-level portrait
    if (!S.pattern_ok) {
        S.n_slices = (nbr + kSlice - 1) / kSlice;
        DBuf<int64_t> w;
        MSFEM_TRY(w.alloc((size_t)S.n_slices + 1));
        MSFEM_TRY(S.slice_ptr.alloc((size_t)S.n_slices + 1));
        MSFEM_CK(cudaMemsetAsync(w.p + S.n_slices, 0, sizeof(int64_t), st));
        k_slice_width<<<grid_for((int64_t)S.n_slices * 32, 256), 256, 0, st>>>(nbr, S.n_slices, s.nrp.p,
                                                                               s.bs == 1 ? kChunk : 1, w.p);
        MSFEM_CK(cudaGetLastError());
        size_t tmp_bytes = 0;
        DBuf<unsigned char> tmp;
        cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, w.p, S.slice_ptr.p, S.n_slices + 1, st);
        MSFEM_TRY(tmp.alloc(tmp_bytes + 1));
        MSFEM_CK(cub::DeviceScan::ExclusiveSum(tmp.p, tmp_bytes, w.p, S.slice_ptr.p, S.n_slices + 1, st));
        int64_t stored = 0;
        MSFEM_CK(cudaMemcpyAsync(&stored, S.slice_ptr.p + S.n_slices, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
        MSFEM_CK(cudaStreamSynchronize(st));
        S.stored = stored;
        MSFEM_TRY(S.col.alloc((size_t)stored));
        const size_t nv = (size_t)stored * (s.bs == 1 ? 1 : 9);
        MSFEM_TRY(S.val64.alloc(nv));
        MSFEM_TRY(S.val32.alloc(nv));
        const int64_t nthreads = (int64_t)S.n_slices * kSlice;
        if (s.bs == 1)
            k_sell_pattern_scalar<<<grid_for(nthreads, 128), 128, 0, st>>>(nbr, s.nrp.p, s.ncol.p, S.slice_ptr.p,
                                                                           S.col.p);
        else
            k_sell_pattern_block<<<grid_for(nthreads, 128), 128, 0, st>>>(nbr, s.nrp.p, s.ncol.p, S.slice_ptr.p,
                                                                          S.col.p);
        MSFEM_CK(cudaGetLastError());
        S.col16.release();
        if (s.bs == 1) {
            // scalar columns as 16-bit deltas when they fit (a Kuhn grid up to ~180^3 in natural
            // numbering): 6 instead of 8 bytes per FP32 nonzero, 10 instead of 12 per FP64 one
            DBuf<int> ovf;
            MSFEM_TRY(ovf.alloc(1));
            MSFEM_TRY(S.col16.alloc((size_t)stored));
            MSFEM_CK(cudaMemsetAsync(ovf.p, 0, sizeof(int), st));
            k_sell_delta16<<<grid_for(nthreads, 128), 128, 0, st>>>(nbr, S.n_slices, S.slice_ptr.p, S.col.p,
                                                                    S.col16.p, ovf.p);
            int h_ovf = 0;
            MSFEM_CK(cudaMemcpyAsync(&h_ovf, ovf.p, sizeof(int), cudaMemcpyDeviceToHost, st));
            MSFEM_CK(cudaStreamSynchronize(st));
            if (h_ovf || s.force_col32) S.col16.release();
            s.total_launches += 1;
        }
        S.pattern_ok = true;
        S.values_ok = false;
        S.fp32_col16 = S.col16.p ? -1 : 0;
        s.total_launches += 2;
    }
    if (!S.values_ok) {
        const int64_t nthreads = (int64_t)S.n_slices * kSlice;
        MSFEM_TRY(s.diag64.alloc(s.n_rows));
        MSFEM_TRY(s.dinv64.alloc(s.n_rows));
        MSFEM_TRY(s.dinv32.alloc(s.n_rows));
        MSFEM_TRY(s.dscale.alloc(s.n_rows));
        DBuf<int>& bad = s.flag;
        MSFEM_TRY(bad.alloc(8));
        MSFEM_CK(cudaMemsetAsync(bad.p, 0, sizeof(int), st));
        k_diag<<<grid_for(s.n_rows, 256), 256, 0, st>>>(s.n_rows, s.bs, s.nrp.p, s.ncol.p, s.val.p, s.diag64.p,
                                                        s.dinv64.p, s.dinv32.p, s.dscale.p, bad.p);
        if (s.bs == 1)
            k_sell_values_scalar<<<grid_for(nthreads, 128), 128, 0, st>>>(nbr, s.nrp.p, s.ncol.p, s.val.p, s.dscale.p,
                                                                          S.slice_ptr.p, S.val64.p, S.val32.p);
        else
            k_sell_values_block<<<grid_for(nthreads, 128), 128, 0, st>>>(nbr, s.nrp.p, s.ncol.p, s.val.p, s.dscale.p,
                                                                         S.slice_ptr.p, S.val64.p, S.val32.p);
        MSFEM_CK(cudaGetLastError());
        int h_bad = 0;
        MSFEM_CK(cudaMemcpyAsync(&h_bad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        MSFEM_CK(cudaStreamSynchronize(st));
        s.sell.values_ok = true;
        s.zero_diag = h_bad != 0;  // only the Jacobi-preconditioned methods care; they check it
        s.total_launches += 2;
    }
    if (S.fp32_col16 < 0) MSFEM_TRY(tune_fp32_columns(s));
    return MSFEM_OK;
}

template <class VT>
SellView<VT> sell_view(System& s)
{
    SellView<VT> v;
    v.n_slices = s.sell.n_slices;
    v.bs = s.bs;
    v.n_rows = s.n_rows;
    v.n_brows = s.n_nodes;
    v.sp = s.sell.slice_ptr.p;
    v.col = s.sell.col.p;
    // 16-bit deltas pay off where the product is bandwidth-bound (FP64); the FP32 product is
    // bound by gather latency, so it uses them only where the timing at set-up says they are faster
    v.col16 = (sizeof(VT) == 8 || s.sell.fp32_col16 == 1) ? s.sell.col16.p : nullptr;
    if constexpr (sizeof(VT) == 8) v.val = reinterpret_cast<const VT*>(s.sell.val64.p);
    else v.val = reinterpret_cast<const VT*>(s.sell.val32.p);
    return v;
}
template SellView<double> sell_view<double>(System&);
template SellView<float> sell_view<float>(System&);

// Blocks for a slice-strided SpMV-type kernel: every SM filled exactly once (SMs x resident
// blocks of 256 threads), so no partial last wave idles the GPU; never more than one warp per slice.
unsigned spmv_grid_of(const void* kernel, const System& s)
{
    static int sms = 0;
    if (!sms) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s.device);
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 256, 0) != cudaSuccess || per_sm <= 0)
        per_sm = 4;
    const unsigned full = grid_for((int64_t)s.sell.n_slices * 32, 256);
    const unsigned fill = (unsigned)(sms * per_sm);
    return full < fill ? full : fill;
}

unsigned spmv_grid(const System& s) { return grid_for((int64_t)s.sell.n_slices * 32, 256); }

int spmv64(System& s, const double* x, double* y)
{
    MSFEM_TRY(prepare_sell(s));
    k_spmv<double><<<spmv_grid_of((const void*)k_spmv<double>, s), 256, 0, s.stream>>>(sell_view<double>(s), x, y);
    MSFEM_CK(cudaGetLastError());
    s.total_launches += 1;
    return MSFEM_OK;
}

int spmv32(System& s, const float* x, float* y)
{
    MSFEM_TRY(prepare_sell(s));
    k_spmv<float><<<spmv_grid_of((const void*)k_spmv<float>, s), 256, 0, s.stream>>>(sell_view<float>(s), x, y);
    MSFEM_CK(cudaGetLastError());
    s.total_launches += 1;
    return MSFEM_OK;
}

// r = f - A x (FP64); *rr_out (device pointer) = (r, r)
// The solver state, zeroed when it is first allocated: its arrival tickets must start at 0 (the
// last block of a two-stage reduction is the one that sees count - 1), and fresh device memory
// need not be zero.
int ensure_kstate(System& s)
{
    if (!s.kstate.p) {
        MSFEM_TRY(s.kstate.alloc(1));
        MSFEM_CK(cudaMemsetAsync(s.kstate.p, 0, sizeof(KState), s.stream));
    }
    return MSFEM_OK;
}

int residual64(System& s, const double* x, const double* f, double* r, double* rr_out)
{
    MSFEM_TRY(prepare_sell(s));
    const unsigned g = spmv_grid_of((const void*)k_residual, s);
    MSFEM_TRY(s.partial.alloc(std::max<size_t>(3 * (size_t)spmv_grid(s), 3 * (size_t)kReduceBlocks) + 64));
    MSFEM_TRY(ensure_kstate(s));
    k_residual<<<g, 256, 0, s.stream>>>(sell_view<double>(s), x, f, r, s.partial.p, &s.kstate.p->ticket[3], rr_out);
    MSFEM_CK(cudaGetLastError());
    return MSFEM_OK;
}

}  // namespace msfem
