#include "fp_pool.cuh"

#include <atomic>
#include <cstdint>
#include <cstring>
#include <memory>
#include <mutex>

namespace nb {
namespace {
constexpr int MAX_DEVICES = 64;
std::mutex g_mutex;
cudaMemPool_t g_pools[MAX_DEVICES] = {};
// Cap + 1 per device; 0 (the zero-initialised default) means no cap.
std::atomic<int64_t> g_cap_plus1[MAX_DEVICES];
// Allocations refused per device (above the cap or out of memory): each one sent a call down its
// path without that memory.
std::atomic<int64_t> g_refused[MAX_DEVICES];

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

// One kernel parameter block of upload_async: 7,500 words (30,000 bytes, under the 32,764-byte
// parameter limit with the other two arguments).
constexpr int UPLOAD_WORDS = 7500;
struct UploadChunk { unsigned w[UPLOAD_WORDS]; };

__global__ void upload_chunk_kernel(const __grid_constant__ UploadChunk c, unsigned* __restrict__ dst, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        dst[i] = c.w[i];
}
} // namespace

bool stream_capturing(cudaStream_t stream) {
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(stream, &st) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return st == cudaStreamCaptureStatusActive;
}

cudaError_t upload_async(void* dst, const void* src, size_t bytes, cudaStream_t stream) {
    if (bytes == 0)
        return cudaSuccess;
    if (bytes % 4 != 0)
        return cudaErrorInvalidValue;
    if (!stream_capturing(stream))
        return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream);
    const size_t words = bytes / 4;
    std::unique_ptr<UploadChunk> chunk(new UploadChunk);
    const unsigned* in = static_cast<const unsigned*>(src);
    unsigned* out = static_cast<unsigned*>(dst);
    for (size_t first = 0; first < words; first += UPLOAD_WORDS) {
        const int n = static_cast<int>(words - first < static_cast<size_t>(UPLOAD_WORDS) ? words - first : UPLOAD_WORDS);
        std::memcpy(chunk->w, in + first, static_cast<size_t>(n) * 4);
        upload_chunk_kernel<<<(n + 255) / 256, 256, 0, stream>>>(*chunk, out + first, n);
        const cudaError_t err = cudaGetLastError();
        if (err != cudaSuccess)
            return err;
    }
    return cudaSuccess;
}

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

int64_t refused_allocations(int device) {
    if (device < 0 || device >= MAX_DEVICES)
        return -1;
    return g_refused[device].load(std::memory_order_relaxed);
}

void* scratch_alloc(size_t bytes, cudaStream_t stream) {
    const int dev = current_device();
    if (dev < 0)
        return nullptr;
    if (!within_cap(dev, bytes)) {
        g_refused[dev].fetch_add(1, std::memory_order_relaxed);
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
        g_refused[dev].fetch_add(1, std::memory_order_relaxed);
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
    if (dev < 0)
        return nullptr;
    void* p = nullptr;
    if (!within_cap(dev, bytes) || cudaMalloc(&p, bytes) != cudaSuccess) {
        cudaGetLastError();
        g_refused[dev].fetch_add(1, std::memory_order_relaxed);
        return nullptr;
    }
    return p;
}

} // namespace nb
