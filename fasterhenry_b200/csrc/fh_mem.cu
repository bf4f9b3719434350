// Process-wide cache of device memory for the large buffers of assembly and
// sweeps: one stream-ordered memory pool per device that keeps what is freed
// (release threshold: never), so that a new system reuses the gigabytes the
// previous one released instead of returning them to the driver and mapping
// them again.  Allocations and frees are ordered on the stream of the work
// that uses them; the pool hands memory to another stream only after its
// free has completed.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "fh_device.cuh"

namespace fhb {
namespace {
constexpr int kMaxDevices = 64;
std::mutex g_mu;
cudaMemPool_t g_pool[kMaxDevices] = {};
}  // namespace

cudaError_t cache_pool(cudaMemPool_t *out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_pool[dev]) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        e = cudaMemPoolCreate(&g_pool[dev], &props);
        if (e != cudaSuccess) {
            g_pool[dev] = nullptr;
            return e;
        }
        uint64_t keep = UINT64_MAX;
        e = cudaMemPoolSetAttribute(g_pool[dev], cudaMemPoolAttrReleaseThreshold, &keep);
        if (e != cudaSuccess) return e;
    }
    *out = g_pool[dev];
    return cudaSuccess;
}

cudaError_t cache_alloc(void **p, size_t bytes, cudaStream_t s) {
    cudaMemPool_t pool;
    cudaError_t e = cache_pool(&pool);
    if (e != cudaSuccess) return e;
    e = cudaMallocFromPoolAsync(p, bytes ? bytes : 16, pool, s);
    if (e == cudaErrorMemoryAllocation) {
        // Let every pending free complete, hand the idle memory of all pools
        // back to the driver, and try once more.
        cudaGetLastError();
        cudaDeviceSynchronize();
        cudaMemPoolTrimTo(pool, 0);
        cudaMemPool_t def;
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetDefaultMemPool(&def, dev) == cudaSuccess) cudaMemPoolTrimTo(def, 0);
        e = cudaMallocFromPoolAsync(p, bytes ? bytes : 16, pool, s);
    }
    return e;
}

void cache_free(void *p, cudaStream_t s) {
    if (p) cudaFreeAsync(p, s);
}

size_t cache_idle_bytes() {
    cudaMemPool_t pool;
    if (cache_pool(&pool) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    uint64_t reserved = 0, used = 0;
    cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved);
    cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used);
    return reserved > used ? (size_t)(reserved - used) : 0;
}

}  // namespace fhb

extern "C" fh_status fh_release_cached_memory(void) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess) {
        cudaGetLastError();
        return FH_OK;
    }
    int cur = 0;
    cudaGetDevice(&cur);
    std::lock_guard<std::mutex> lk(fhb::g_mu);
    for (int d = 0; d < count && d < fhb::kMaxDevices; ++d) {
        if (!fhb::g_pool[d]) continue;
        cudaSetDevice(d);
        cudaDeviceSynchronize();
        cudaMemPoolTrimTo(fhb::g_pool[d], 0);
    }
    cudaSetDevice(cur);
    return FH_OK;
}
