#include "fp_pool.cuh"

#include <cstdint>
#include <mutex>

namespace nb {
namespace {
std::mutex g_mutex;
cudaMemPool_t g_pools[64] = {};
}

void* scratch_alloc(size_t bytes, cudaStream_t stream) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return nullptr;
    }
    cudaMemPool_t pool;
    {
        std::lock_guard<std::mutex> lock(g_mutex);
        if (!g_pools[dev]) {
            cudaMemPoolProps props{};
            props.allocType = cudaMemAllocationTypePinned;
            props.handleTypes = cudaMemHandleTypeNone;
            props.location.type = cudaMemLocationTypeDevice;
            props.location.id = dev;
            if (cudaMemPoolCreate(&g_pools[dev], &props) != cudaSuccess) {
                cudaGetLastError();
                g_pools[dev] = nullptr;
                return nullptr;
            }
            uint64_t threshold = UINT64_MAX;
            cudaMemPoolSetAttribute(g_pools[dev], cudaMemPoolAttrReleaseThreshold, &threshold);
        }
        pool = g_pools[dev];
    }
    void* p = nullptr;
    if (cudaMallocFromPoolAsync(&p, bytes, pool, stream) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return p;
}

void scratch_free(void* ptr, cudaStream_t stream) {
    if (ptr)
        cudaFreeAsync(ptr, stream);
}

} // namespace nb
