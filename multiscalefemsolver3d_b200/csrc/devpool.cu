// A caching allocator under every device buffer of the library (DBuf): a freed block keeps its
// memory in a per-device free list of its size class and the next allocation of that class takes
// it back, so a workload that builds and tears down the same handles step after step (coarse
// spaces, solver workspaces, temporaries) does not pay cudaMalloc / cudaFree each time.  Size
// classes: powers of two up to 1 MiB, multiples of 2 MiB above.  A free synchronises the device
// first, as cudaFree does, so no kernel still in flight can see the block handed out again.  The
// cache holds at most kCacheCap bytes per device; cudaMalloc failing for lack of memory empties
// the device's cache and retries; msfem_release_cached_memory empties every cache.
#include <map>
#include <mutex>
#include <vector>

#include "internal.cuh"

namespace msfem {
namespace {

constexpr size_t kCacheCap = size_t(48) << 30;

struct Pool {
    std::mutex mu;
    std::map<std::pair<int, size_t>, std::vector<void*>> free;  // (device, class) -> blocks
    std::map<int, size_t> cached;                                // device -> bytes held
};

Pool& pool()
{
    static Pool* p = new Pool();  // never destroyed: frees at process exit are the driver's
    return *p;
}

size_t size_class(size_t bytes)
{
    if (bytes <= (size_t(1) << 20)) {
        size_t c = 512;
        while (c < bytes) c <<= 1;
        return c;
    }
    const size_t g = size_t(2) << 20;
    return (bytes + g - 1) / g * g;
}

void drop_device(Pool& P, int dev)
{
    for (auto it = P.free.begin(); it != P.free.end();) {
        if (it->first.first == dev) {
            for (void* b : it->second) cudaFree(b);
            it = P.free.erase(it);
        } else {
            ++it;
        }
    }
    P.cached[dev] = 0;
}

}  // namespace

void* dev_alloc(size_t bytes, cudaError_t* err)
{
    *err = cudaSuccess;
    if (bytes == 0) return nullptr;
    int dev = 0;
    if ((*err = cudaGetDevice(&dev)) != cudaSuccess) return nullptr;
    const size_t cls = size_class(bytes);
    Pool& P = pool();
    {
        std::lock_guard<std::mutex> lock(P.mu);
        auto it = P.free.find({dev, cls});
        if (it != P.free.end() && !it->second.empty()) {
            void* b = it->second.back();
            it->second.pop_back();
            P.cached[dev] -= cls;
            return b;
        }
    }
    void* b = nullptr;
    cudaError_t e = cudaMalloc(&b, cls);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();  // clear the sticky-free allocation error before retrying
        {
            std::lock_guard<std::mutex> lock(P.mu);
            drop_device(P, dev);
        }
        e = cudaMalloc(&b, cls);
    }
    *err = e;
    return e == cudaSuccess ? b : nullptr;
}

void dev_free(void* p, size_t bytes)
{
    if (!p) return;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) {
        cudaFree(p);
        return;
    }
    const size_t cls = size_class(bytes);
    Pool& P = pool();
    std::lock_guard<std::mutex> lock(P.mu);
    if (P.cached[dev] + cls > kCacheCap) {
        cudaFree(p);
        return;
    }
    P.free[{dev, cls}].push_back(p);
    P.cached[dev] += cls;
}

}  // namespace msfem

extern "C" void msfem_release_cached_memory(void)
{
    using namespace msfem;
    Pool& P = pool();
    std::lock_guard<std::mutex> lock(P.mu);
    int cur = 0;
    cudaGetDevice(&cur);
    std::vector<int> devs;
    for (auto& kv : P.cached) devs.push_back(kv.first);
    for (int d : devs) {
        cudaSetDevice(d);
        drop_device(P, d);
    }
    cudaSetDevice(cur);
}
