#include "fp_pool.cuh"

#include <atomic>
#include <cstdint>
#include <mutex>

namespace nb {
namespace {
constexpr int MAX_DEVICES = 64;
std::mutex g_mutex;
cudaMemPool_t g_pools[MAX_DEVICES] = {};
// Cap + 1 per device; 0 (the zero-initialised default) means no cap.
std::atomic<int64_t> g_cap_plus1[MAX_DEVICES];

int current_device() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) {
        cudaGetLastError();
        return -1;
    }
    return dev;
}

bool within_cap(int dev, size_t bytes) {
    const int64_t c = g_cap_plus1[dev].load(std::memory_order_relaxed);
    return c == 0 || bytes <= static_cast<uint64_t>(c - 1);
}
} // namespace

bool set_scratch_limit(int device, int64_t bytes) {
    if (device < 0 || device >= MAX_DEVICES)
        return false;
    g_cap_plus1[device].store(bytes < 0 ? 0 : bytes + 1, std::memory_order_relaxed);
    return true;
}

int64_t scratch_limit(int device) {
    if (device < 0 || device >= MAX_DEVICES)
        return -1;
    return g_cap_plus1[device].load(std::memory_order_relaxed) - 1;
}

void* scratch_alloc(size_t bytes, cudaStream_t stream) {
    const int dev = current_device();
    if (dev < 0 || !within_cap(dev, bytes))
        return nullptr;
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

void* device_alloc(size_t bytes) {
    const int dev = current_device();
    if (dev < 0 || !within_cap(dev, bytes))
        return nullptr;
    void* p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return p;
}

} // namespace nb
