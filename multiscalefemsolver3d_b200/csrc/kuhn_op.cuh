// Host side of the matrix-free Kuhn-grid operators (kuhn.cuh): the persistent kernel over bricks,
// its launch configuration, and the operator state a solver keeps.
#pragma once

#include <algorithm>

#include "internal.cuh"
#include "kuhn.cuh"

namespace msfem {

// brick shapes: FP32 8 x 8 x 8 nodes (82 KB of shared memory, two CTAs per SM), FP64 8 x 8 x 4
// (93 KB, two CTAs per SM)
struct KuhnCfg32 {
    static constexpr int BX = 8, BY = 8, BZ = 8, THREADS = 256;
};
struct KuhnCfg64 {
    static constexpr int BX = 8, BY = 8, BZ = 4, THREADS = 256;
};

// persistent: CTA b takes bricks b, b + grid, ... (a fixed assignment, so block partial sums are
// reproducible); the epilogue functor sees every owned node once and finishes the block
template <int FORM, int BX, int BY, int BZ, int THREADS, class T, class Epi>
__global__ void __launch_bounds__(THREADS) k_kuhn(KuhnView<T> K, const T* __restrict__ x, Epi epi)
{
    if (epi.skip()) return;
    using L = KuhnBrick<T, BX, BY, BZ>;
    extern __shared__ __align__(16) unsigned char kuhn_smem[];
    T* su = reinterpret_cast<T*>(kuhn_smem);
    T* sc = su + 3 * L::NH;
    T* sl = sc + 24 * L::NC;
    kuhn_stage_lame(K, sl);
    __syncthreads();
    const int nb = K.nbx * K.nby * K.nbz;
    for (int b = blockIdx.x; b < nb; b += gridDim.x) kuhn_brick<FORM, BX, BY, BZ, THREADS>(K, x, b, su, sc, sl, epi);
    epi.finish();
}

template <int FORM, class Cfg, class T, class Epi>
struct KuhnKernel {
    using L = KuhnBrick<T, Cfg::BX, Cfg::BY, Cfg::BZ>;
    static constexpr auto kernel = k_kuhn<FORM, Cfg::BX, Cfg::BY, Cfg::BZ, Cfg::THREADS, T, Epi>;
    inline static int blocks_per_sm = 0;
    inline static uint64_t prepared = 0;  // devices (bit = ordinal) where the attribute is set
    // shared-memory opt-in and occupancy, per device; call outside stream capture before the
    // first launch on a device
    static cudaError_t prepare()
    {
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        const uint64_t bit = 1ull << (dev & 63);
        if (prepared & bit) return cudaSuccess;
        e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::smem);
        if (e != cudaSuccess) return e;
        int nb = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, Cfg::THREADS, L::smem);
        if (e != cudaSuccess) return e;
        blocks_per_sm = std::max(nb, 1);
        prepared |= bit;
        return cudaSuccess;
    }
    static int grid(int n_bricks, int sms) { return std::max(1, std::min(n_bricks, blocks_per_sm * sms)); }
    static cudaError_t launch(const KuhnView<T>& K, const T* x, const Epi& epi, int sms, cudaStream_t st)
    {
        cudaError_t e = prepare();
        if (e != cudaSuccess) return e;
        const int nb = K.nbx * K.nby * K.nbz;
        kernel<<<grid(nb, sms), Cfg::THREADS, L::smem, st>>>(K, x, epi);
        return cudaGetLastError();
    }
};

template <int FORM, class Cfg, class T, class Epi>
inline cudaError_t kuhn_launch(const KuhnView<T>& K, const T* x, const Epi& epi, int /*n_bricks*/, int sms,
                               cudaStream_t st)
{
    return KuhnKernel<FORM, Cfg, T, Epi>::launch(K, x, epi, sms, st);
}

// one matrix-free operator, checked against the assembled matrix of `sys` at values_version
struct KuhnOperator {
    System* sys = nullptr;
    uint64_t version = 0;
    int form = 0;        // 1 the reference's assembly, 2 the textbook orientation
    bool fp64 = false;   // FP64 unscaled (A) or FP32 Jacobi-scaled (S K S)
    bool scaled = false;
    int sms = 0;
    double check_l2 = 0.0, check_max = 0.0;  // relative distance to the assembled product at set-up
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

}  // namespace msfem
