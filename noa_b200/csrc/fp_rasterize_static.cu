// nb_rasterize_central_slices_3d_static_scratch: the rasterization of nb_rasterize_central_slices_3d
// with its accumulator in a fixed array of this library's device code, so the call allocates nothing.
//
// Why: the regular entry point takes its interleaved (value, weight) accumulator from a stream-ordered
// memory pool on every call. Some callers cannot let a library allocate device memory at call time:
// code running under a strict memory budget that was fixed up front (a serving process that reserved
// its HBM once), code whose allocator is owned by someone else, or code that must not trigger the
// driver's allocator in its steady state. This entry point serves them.
//
// Limits and rules:
//   * The accumulator is a file-scope __device__ array of STATIC_SCRATCH_BYTES (64 MiB). CUDA reserves
//     it on a GPU when it loads this file's module there: with the default lazy module loading, during
//     the first call on that GPU (the address lookup below loads it), or when the library is loaded
//     with CUDA_MODULE_LOADING=EAGER. From then on it is held until the process exits. So a caller
//     with a fixed memory budget makes one warm-up call per GPU while it sets that budget up; later
//     calls allocate nothing. With output weights, volumes up to
//     STATIC_SCRATCH_BYTES / 16 voxels (complex values) or / 8 voxels (real values) of the rfft grid
//     (D * H * (W/2+1)) are accepted; larger volumes are rejected with NB_ERROR_INVALID. Without output
//     weights the reductions go straight into the caller's grid and no scratch is used at all.
//   * The first call on a device looks up the array's device address (cudaGetSymbolAddress, with that
//     device current); make that first call before any stream capture.
//   * All calls share the one array. Each call clears the part it uses before accumulating, on its
//     stream, and leaves its partial sums behind. Calls that overlap on the GPU (different streams,
//     or different host threads, without ordering between them) race on the array: order them.
//   * No cudaMalloc, cudaFree or other allocating routine is called.
#include "fp_args.cuh"
#include "fp_rasterize_kernels.cuh"

#include <cstdio>
#include <mutex>

namespace nb {
namespace {

constexpr size_t STATIC_SCRATCH_BYTES = size_t(64) << 20;

static __device__ __align__(256) unsigned char g_static_scratch[STATIC_SCRATCH_BYTES];

std::mutex g_mutex;
void* g_scratch_ptr[64] = {};

// Device address of g_static_scratch on the current device (looked up once per device).
int static_scratch(void** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return report_error(NB_ERROR_CUDA, "no CUDA device for the static scratch");
    }
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch_ptr[dev]) {
        void* ptr = nullptr;
        const cudaError_t err = cudaGetSymbolAddress(&ptr, g_static_scratch);
        if (err != cudaSuccess || !ptr) {
            char msg[256];
            std::snprintf(msg, sizeof(msg), "cudaGetSymbolAddress of the static scratch failed: %s",
                          cudaGetErrorString(err));
            cudaGetLastError();
            return report_error(NB_ERROR_CUDA, msg);
        }
        g_scratch_ptr[dev] = ptr;
    }
    *out = g_scratch_ptr[dev];
    return NB_OK;
}

using namespace raster;

template<bool IN_C, bool OUT_C>
cudaError_t launch_static(const ProjArgs& a, void* scratch, cudaStream_t stream) {
    const int wp = a.slice_w / 2 + 1;
    const int ntx = (wp + TX - 1) / TX, nty = (a.slice_h + TY - 1) / TY;
    if (a.n_slices == 0)
        return cudaSuccess;
    const dim3 grid(static_cast<unsigned>(ntx * nty), static_cast<unsigned>(a.n_slices < 65535 ? a.n_slices : 65535));
    if (!a.out_w.present) {
        rasterize_kernel<IN_C, OUT_C, DIRECT><<<grid, RASTER_THREADS, 0, stream>>>(a, ntx, nullptr);
        return cudaGetLastError();
    }
    const int64_t vox = static_cast<int64_t>(a.vol_d) * a.vol_h * (a.vol_w / 2 + 1);
    const size_t bytes = static_cast<size_t>(vox) * (OUT_C ? sizeof(float4) : sizeof(float2));
    cudaError_t err = cudaMemsetAsync(scratch, 0, bytes, stream);
    if (err != cudaSuccess)
        return err;
    rasterize_kernel<IN_C, OUT_C, SCRATCH><<<grid, RASTER_THREADS, 0, stream>>>(a, ntx, scratch);
    const int64_t blocks = (vox + 255) / 256;
    const int grid_f = static_cast<int>(blocks < static_cast<int64_t>(sm_count()) * 16 ? blocks : sm_count() * 16);
    finalize_kernel<OUT_C><<<grid_f, 256, 0, stream>>>(a, scratch);
    return cudaGetLastError();
}

} // namespace
} // namespace nb

using namespace nb;

extern "C" int nb_rasterize_central_slices_3d_static_scratch(
    int32_t remap,
    const nb_array* slice, const nb_array* slice_weight, const int64_t slice_shape[4],
    const nb_array* volume, const nb_array* volume_weight, const int64_t volume_shape[4],
    const nb_transform* inv_scaling, const nb_transform* fwd_rotation,
    const nb_options* options, void* stream) {
    ProjArgs a{};
    int st = prepare_rasterize(remap, slice, slice_weight, slice_shape, volume, volume_weight, volume_shape,
                               inv_scaling, fwd_rotation, options, a);
    if (st != NB_OK)
        return st;
    void* scratch = nullptr;
    if (a.out_w.present) {
        const int64_t vox = static_cast<int64_t>(a.vol_d) * a.vol_h * (a.vol_w / 2 + 1);
        const int64_t elem = a.out_cplx ? 16 : 8;
        if (vox * elem > static_cast<int64_t>(STATIC_SCRATCH_BYTES)) {
            char msg[256];
            std::snprintf(msg, sizeof(msg),
                          "volume of %lld rfft voxels needs %lld bytes of accumulator, more than the %zu-byte "
                          "static scratch of this entry point (use nb_rasterize_central_slices_3d)",
                          static_cast<long long>(vox), static_cast<long long>(vox * elem), STATIC_SCRATCH_BYTES);
            return report_error(NB_ERROR_INVALID, msg);
        }
        if ((st = static_scratch(&scratch)) != NB_OK)
            return st;
    }
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t err;
    if (a.in_cplx && a.out_cplx)
        err = launch_static<true, true>(a, scratch, s);
    else if (a.in_cplx)
        err = launch_static<true, false>(a, scratch, s);
    else
        err = launch_static<false, false>(a, scratch, s);
    return finish_launch(err);
}
