// Stream-ordered device memory for the entry points that take host buffers and
// allocate their own device copies (gpgmp_gs_forward_host, gpgmp_gs_loss_grad_host,
// the batched forward's member table).
//
// The device's default memory pool returns freed memory to the driver at every
// synchronisation (release threshold 0), so a call that allocates, synchronises and
// frees maps fresh physical memory every time; on B200 that cost 1-20 ms per call.
// These allocations come instead from one pool per device created by the library
// with an unlimited release threshold: freed blocks stay mapped in the pool and the
// next call reuses them.  The pool holds the largest amount in use at once until the
// process exits.
#include <cstdint>
#include <mutex>
#include <cuda_runtime.h>
#include "host_common.h"

namespace gpgmp {
namespace {
constexpr int kMaxDevices = 64;
cudaMemPool_t g_pools[kMaxDevices] = {};
std::mutex g_pool_mutex;
}  // namespace

cudaError_t pool_of_current_device(cudaMemPool_t* out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    if (!g_pools[dev]) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool = nullptr;
        e = cudaMemPoolCreate(&pool, &props);
        if (e != cudaSuccess) return e;
        uint64_t keep = UINT64_MAX;
        e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        if (e != cudaSuccess) {
            cudaMemPoolDestroy(pool);
            return e;
        }
        g_pools[dev] = pool;
    }
    *out = g_pools[dev];
    return cudaSuccess;
}

cudaError_t pool_alloc(void** p, size_t bytes, cudaStream_t st) {
    cudaMemPool_t pool = nullptr;
    cudaError_t e = pool_of_current_device(&pool);
    if (e != cudaSuccess) return e;
    return cudaMallocFromPoolAsync(p, bytes > 0 ? bytes : 1, pool, st);
}

cudaError_t pool_free(void* p, cudaStream_t st) { return p ? cudaFreeAsync(p, st) : cudaSuccess; }

}  // namespace gpgmp
