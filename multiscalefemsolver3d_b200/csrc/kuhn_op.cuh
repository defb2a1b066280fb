// Host side of the matrix-free Kuhn-grid operators (kuhn.cuh, kuhn25.cuh): the z-marching kernel's
// launch configuration and the operator state a solver keeps.
#pragma once

#include <algorithm>

#include "internal.cuh"
#include "kuhn.cuh"
#include "kuhn25.cuh"

namespace msfem {

// the z-marching kernel (kuhn25.cuh): TX x TY hexahedron columns per CTA
template <int FORM, bool SC, class T, int TX, int TY, int MINB, class Epi>
struct KzKernel {
    using L = KzLayout<T, TX, TY, Epi::NE, SC>;
    static constexpr auto kernel_iso = k_kuhn_z<FORM, true, SC, T, TX, TY, MINB, Epi>;
    static constexpr auto kernel_aniso = k_kuhn_z<FORM, false, SC, T, TX, TY, MINB, Epi>;
    inline static int blocks_per_sm = 0;
    inline static uint64_t prepared = 0;
    static cudaError_t prepare()
    {
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        const uint64_t bit = 1ull << (dev & 63);
        if (prepared & bit) return cudaSuccess;
        e = cudaFuncSetAttribute(kernel_iso, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::smem);
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(kernel_aniso, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::smem);
        if (e != cudaSuccess) return e;
        int nb = 0, nb2 = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel_iso, L::THREADS, L::smem);
        if (e != cudaSuccess) return e;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb2, kernel_aniso, L::THREADS, L::smem);
        if (e != cudaSuccess) return e;
        blocks_per_sm = std::max(std::min(nb, nb2), 1);
        prepared |= bit;
        return cudaSuccess;
    }
    // The bulk copies need 16-byte-aligned sources (and read up to 12 bytes past a vector's last
    // element, so every staged vector carries 16 bytes of slack): refused here, never launched.
    static bool aligned(const void* p) { return ((uintptr_t)p & 15) == 0; }
    static cudaError_t launch(const KuhnView<T>& K, const T* x, const Epi& epi, int sms, int* err, cudaStream_t st)
    {
        cudaError_t e = prepare();
        if (e != cudaSuccess) return e;
        const T* ev[Epi::NE > 0 ? Epi::NE : 1] = {};
        epi.sources(ev);
        bool ok = aligned(x) && aligned(K.fix) && aligned(K.mat) && (SC ? (K.scale && aligned(K.scale)) : !K.scale);
        for (int q = 0; q < Epi::NE; q++) ok = ok && ev[q];
        if (!ok) return cudaErrorMisalignedAddress;
        KzArgs<T> A;
        A.K = K;
        A.x = x;
        A.err = err;
        A.tiles_x = (K.nx + 1 + L::OX - 1) / L::OX;
        A.tiles_y = (K.ny + 1 + L::OY - 1) / L::OY;
        const int nnz = K.nz + 1, tiles = A.tiles_x * A.tiles_y;
        // z segments: the count that minimises waves x steps per CTA (a segment of s layers takes
        // s + 1 steps; the CTAs run in ceil(tiles * segments / resident CTAs) waves)
        const int64_t slots = (int64_t)blocks_per_sm * sms;
        int64_t best = -1;
        for (int n_seg = 1; n_seg <= nnz; n_seg++) {
            const int len = (nnz + n_seg - 1) / n_seg;
            const int segs = (nnz + len - 1) / len;
            const int64_t cost = ((int64_t)tiles * segs + slots - 1) / slots * (len + 1);
            if (best < 0 || cost < best) {
                best = cost;
                A.seg_len = len;
                A.n_seg = segs;
            }
        }
        if (K.iso)
            kernel_iso<<<tiles * A.n_seg, L::THREADS, L::smem, st>>>(A, epi);
        else
            kernel_aniso<<<tiles * A.n_seg, L::THREADS, L::smem, st>>>(A, epi);
        return cudaGetLastError();
    }
};

// the pre-scaled z-marching kernel (k_kuhn_zp): x = s u with the eliminated columns zero, staged as
// it is; the grid and segment choice as KzKernel's
template <int FORM, class T, int TX, int TY, int MINB, class Epi>
struct KzpKernel {
    using L = KzpLayout<T, TX, TY, Epi::NE>;
    static constexpr auto kernel_iso = k_kuhn_zp<FORM, true, T, TX, TY, MINB, Epi>;
    static constexpr auto kernel_aniso = k_kuhn_zp<FORM, false, T, TX, TY, MINB, Epi>;
    inline static int blocks_per_sm = 0;
    inline static uint64_t prepared = 0;
    static cudaError_t prepare()
    {
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        const uint64_t bit = 1ull << (dev & 63);
        if (prepared & bit) return cudaSuccess;
        e = cudaFuncSetAttribute(kernel_iso, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::smem);
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(kernel_aniso, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::smem);
        if (e != cudaSuccess) return e;
        int nb = 0, nb2 = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel_iso, L::THREADS, L::smem);
        if (e != cudaSuccess) return e;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb2, kernel_aniso, L::THREADS, L::smem);
        if (e != cudaSuccess) return e;
        blocks_per_sm = std::max(std::min(nb, nb2), 1);
        prepared |= bit;
        return cudaSuccess;
    }
    // 16-byte-aligned sources with 16 bytes of slack, as KzKernel
    static bool aligned(const void* p) { return ((uintptr_t)p & 15) == 0; }
    static cudaError_t launch(const KuhnView<T>& K, const T* x, const Epi& epi, int sms, int* err, cudaStream_t st)
    {
        cudaError_t e = prepare();
        if (e != cudaSuccess) return e;
        const T* ev[Epi::NE > 0 ? Epi::NE : 1] = {};
        epi.sources(ev);
        bool ok = aligned(x) && aligned(K.fix) && aligned(K.mat);
        for (int q = 0; q < Epi::NE; q++) ok = ok && ev[q];
        if (!ok) return cudaErrorMisalignedAddress;
        KzArgs<T> A;
        A.K = K;
        A.x = x;
        A.err = err;
        A.tiles_x = (K.nx + 1 + L::OX - 1) / L::OX;
        A.tiles_y = (K.ny + 1 + L::OY - 1) / L::OY;
        const int nnz = K.nz + 1, tiles = A.tiles_x * A.tiles_y;
        const int64_t slots = (int64_t)blocks_per_sm * sms;
        int64_t best = -1;
        for (int n_seg = 1; n_seg <= nnz; n_seg++) {
            const int len = (nnz + n_seg - 1) / n_seg;
            const int segs = (nnz + len - 1) / len;
            const int64_t cost = ((int64_t)tiles * segs + slots - 1) / slots * (len + 1);
            if (best < 0 || cost < best) {
                best = cost;
                A.seg_len = len;
                A.n_seg = segs;
            }
        }
        if (K.iso)
            kernel_iso<<<tiles * A.n_seg, L::THREADS, L::smem, st>>>(A, epi);
        else
            kernel_aniso<<<tiles * A.n_seg, L::THREADS, L::smem, st>>>(A, epi);
        return cudaGetLastError();
    }
};

// one matrix-free operator, checked against the assembled matrix of `sys` at values_version
struct KuhnOperator {
    System* sys = nullptr;
    uint64_t version = 0;
    int form = 0;        // 1 the reference's assembly, 2 the textbook orientation
    bool fp64 = false;   // FP64 unscaled (A) or FP32 Jacobi-scaled (S K S)
    bool scaled = false;
    int sms = 0;
    double check_l2 = 0.0, check_max = 0.0;  // relative distance to the assembled product at set-up
    DBuf<int> err;       // raised by a z-marching launch whose staging wait expired
    DBuf<double> lame64;
    DBuf<float> lame32, scale32;
    KuhnView<double> v64{};
    KuhnView<float> v32{};
};

int kuhn_set_grid(System& s, int nx, int ny, int nz);
int kuhn_operator_build(System& s, int form, bool fp64, bool scaled, KuhnOperator& op);
int kuhn_operator_current(const KuhnOperator& op);
int kuhn_spmv64(KuhnOperator& op, const double* x, double* y, cudaStream_t st);
int kuhn_spmv32(KuhnOperator& op, const float* x, float* y, cudaStream_t st);
// y = S K S x through the pre-scaled kernel (k_kuhn_zp): xh (n + 16 elements, scratch) receives
// s x with the eliminated columns zero first; op.sys set
int kuhn_spmv32_pre(KuhnOperator& op, const float* x, float* xh, float* y, cudaStream_t st);
// MSFEM_ERR_CUDA (and the flag cleared) if a z-marching launch on op raised its staging error
int kuhn_check_err(KuhnOperator& op, cudaStream_t st);

// y = op x through the z-marching kernel
template <class T>
struct EpiStoreZ {
    static constexpr int NE = 0;
    T* y;
    __device__ __forceinline__ bool skip() const { return false; }
    __host__ __device__ __forceinline__ void sources(const T** ev) const { (void)ev; }
    __device__ __forceinline__ void operator()(int64_t g, const T* v, const T* xin, const T (*e)[3])
    {
        (void)xin;
        (void)e;
        y[3 * g] = v[0];
        y[3 * g + 1] = v[1];
        y[3 * g + 2] = v[2];
    }
    __device__ __forceinline__ void finish() {}
};
// the z-marching configurations: 16 x 16 hexahedron columns (15 x 15 owned nodes); FP32 two CTAs
// per SM, FP64 one
constexpr int kKzTX = 16, kKzTY = 16, kKzMinB = 2, kKzMinB64 = 1;

}  // namespace msfem
