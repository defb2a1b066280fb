// msfem_residual_noalloc: r = f - A x and ||r||^2 for a caller-owned CSR matrix,
// without allocating any device memory.
//
// Some callers cannot let a library call cudaMalloc: applications that hand the
// whole device heap to their own arena at start-up (so a library allocation
// fails or fragments it), and loops that cannot afford the device-wide
// synchronisation that cudaFree implies.  The handle-based API allocates its
// buffers when a system is created and grows its scratch on first use; this
// entry point instead keeps the only scratch it needs -- the per-block partial
// sums of the residual norm and an arrival counter -- in a fixed file-scope
// device array.
//
// Limits and sharing:
//  * the array holds kMaxBlocks partial sums (one per 256 rows), so n_rows is
//    limited to kMaxBlocks * 256 = 4,194,304 rows; larger systems are rejected;
//  * every GPU that loads this library holds the array (128 KiB + 256 B) until
//    the process exits;
//  * all calls on a device share the array: two calls whose kernels overlap on
//    that GPU (different streams, or different host threads) race on it and
//    give wrong results.  Serialise them.
//  * the first call on a device (with that device current) looks up the
//    array's device address with cudaGetSymbolAddress; make that first call
//    before any stream capture is in progress on the calling thread.
//  * the address is kept per device ordinal and checked on every call with
//    cudaPointerGetAttributes; when it no longer names device memory of the
//    current device (after cudaDeviceReset, or under another context) it is
//    looked up again, so that call is a set-up call too.
#include <mutex>

#include "devutil.cuh"
#include "internal.cuh"

namespace msfem {
namespace {

constexpr int kNoAllocThreads = 256;
constexpr int kMaxBlocks = 16384;
constexpr int kMaxDevices = 64;

// [0, kMaxBlocks) doubles: block partials; then one unsigned int arrival counter
static __device__ __align__(256) double g_noalloc_scratch[kMaxBlocks + 32];

double* g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mutex;

__global__ void __launch_bounds__(kNoAllocThreads)
    k_residual_csr(int n, const int32_t* __restrict__ rp, const int32_t* __restrict__ col,
                   const double* __restrict__ val, const double* __restrict__ x, const double* __restrict__ f,
                   double* __restrict__ r, double* __restrict__ rr, double* __restrict__ scratch)
{
    __shared__ double sh[32];
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[1] = {0.0};
    if (row < n) {
        double s = 0.0;
        for (int p = rp[row]; p < rp[row + 1]; p++) s += val[p] * x[col[p]];
        const double v = f[row] - s;
        r[row] = v;
        acc[0] = v * v;
    }
    block_sum<1>(acc, sh);
    if (threadIdx.x == 0) scratch[blockIdx.x] = acc[0];
    unsigned int* ticket = reinterpret_cast<unsigned int*>(scratch + kMaxBlocks);
    if (arrive_last(ticket)) {
        double t[1];
        reduce_partials<1>(scratch, gridDim.x, 0, t, sh);
        if (threadIdx.x == 0) {
            *rr = t[0];
            *ticket = 0;
        }
    }
}

int scratch_address(double** out)
{
    int dev = 0;
    MSFEM_CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("msfem_residual_noalloc: device ordinal %d outside [0, %d)", dev, kMaxDevices);
        return MSFEM_ERR_LIMIT;
    }
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (g_scratch_addr[dev]) {
        // the cached address belongs to the context that was current at look-up; after a device
        // reset or under a different context it may name nothing, or other memory
        cudaPointerAttributes a{};
        const cudaError_t e = cudaPointerGetAttributes(&a, g_scratch_addr[dev]);
        if (e != cudaSuccess || a.type != cudaMemoryTypeDevice || a.device != dev) {
            (void)cudaGetLastError();  // a failed query must not surface as the launch's error
            g_scratch_addr[dev] = nullptr;
        }
    }
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            set_error("msfem_residual_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
            return MSFEM_ERR_CUDA;
        }
        g_scratch_addr[dev] = static_cast<double*>(p);
    }
    *out = g_scratch_addr[dev];
    return MSFEM_OK;
}

}  // namespace
}  // namespace msfem

using namespace msfem;

extern "C" int msfem_residual_noalloc(int n_rows, const int32_t* row_ptr, const int32_t* col, const double* val,
                                      const double* x, const double* f, double* r, double* rr, void* stream)
{
    if (n_rows <= 0 || !row_ptr || !col || !val || !x || !f || !r || !rr) {
        set_error("msfem_residual_noalloc: bad arguments (n_rows %d)", n_rows);
        return MSFEM_ERR_ARGUMENT;
    }
    const int64_t blocks = ((int64_t)n_rows + kNoAllocThreads - 1) / kNoAllocThreads;
    if (blocks > kMaxBlocks) {
        set_error("msfem_residual_noalloc: %d rows exceed the fixed scratch limit of %d rows", n_rows,
                  kMaxBlocks * kNoAllocThreads);
        return MSFEM_ERR_LIMIT;
    }
    double* scratch = nullptr;
    MSFEM_TRY(scratch_address(&scratch));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // the arrival counter must start at zero; the previous call normally leaves it
    // at zero, but a call cut short by an error might not
    MSFEM_CK(cudaMemsetAsync(scratch + kMaxBlocks, 0, sizeof(unsigned int), st));
    k_residual_csr<<<(unsigned)blocks, kNoAllocThreads, 0, st>>>(n_rows, row_ptr, col, val, x, f, r, rr, scratch);
    MSFEM_CK(cudaGetLastError());
    return MSFEM_OK;
}
