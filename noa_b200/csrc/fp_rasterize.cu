// rasterize_central_slices_3d on sm_100a: one thread per slice pixel, trilinear scatter of the pixel
// into the 2x2x2 voxels around its rotated frequency, plus the Hermitian-plane mirror taps
// (FourierInsertRasterize, noa/xform/FourierProject.hpp:238-373).
//
// The scatter is bound by the L2 reduction rate, which counts one operation per lane whatever its
// width. So with output weights, a pixel's value and weight for one voxel travel in ONE reduction:
// the kernel accumulates into a dense interleaved scratch grid — float4 (re, im, w, -) for complex
// values, float2 (v, w) for real ones — taken from a stream-ordered pool, zeroed first, and a finalize
// pass adds it into the caller's value and weight grids (whatever their strides). Without weights the
// reductions go straight into the caller's grid (red.global.add.v2.f32 for complex values). If the
// scratch cannot be allocated, the kernel falls back to two reductions per tap on the caller's grids.
// CTAs own 16x16 pixel tiles of one slice (warps: 4x8), so a warp's reductions hit a compact patch.
//
// Deliberate deviation from the reference: the reference bounds the u tap by the LOGICAL volume width
// (FourierProject.hpp:327-329), so a tap at u = W/2+1 passes and lands in the next row (or past the
// end of the array). Here u is bounded by the physical width W/2+1. For even sizes and cutoffs <= 0.5
// such taps carry a zero weight, so the results are the same.
#include "fp_args.cuh"
#include "fp_pool.cuh"
#include "fp_rasterize_kernels.cuh"

namespace nb {
namespace {

using namespace raster;

template<bool IN_C, bool OUT_C>
cudaError_t launch_typed(const ProjArgs& a, cudaStream_t stream) {
    const int wp = a.slice_w / 2 + 1;
    const int ntx = (wp + TX - 1) / TX, nty = (a.slice_h + TY - 1) / TY;
    if (a.n_slices == 0)
        return cudaSuccess;
    const dim3 grid(static_cast<unsigned>(ntx * nty), static_cast<unsigned>(a.n_slices < 65535 ? a.n_slices : 65535));
    const int64_t vox = static_cast<int64_t>(a.vol_d) * a.vol_h * (a.vol_w / 2 + 1);
    void* scratch = nullptr;
    if (a.out_w.present && vox < (int64_t(1) << 31)) {
        const size_t bytes = static_cast<size_t>(vox) * (OUT_C ? sizeof(float4) : sizeof(float2));
        scratch = scratch_alloc(bytes, stream);
        if (scratch && cudaMemsetAsync(scratch, 0, bytes, stream) != cudaSuccess) {
            scratch_free(scratch, stream);
            return cudaGetLastError();
        }
    }
    if (scratch) {
        rasterize_kernel<IN_C, OUT_C, SCRATCH><<<grid, RASTER_THREADS, 0, stream>>>(a, ntx, scratch);
        const int64_t blocks = (vox + 255) / 256;
        const int grid_f = static_cast<int>(blocks < static_cast<int64_t>(sm_count()) * 16 ? blocks : sm_count() * 16);
        finalize_kernel<OUT_C><<<grid_f, 256, 0, stream>>>(a, scratch);
        const cudaError_t err = cudaGetLastError();
        scratch_free(scratch, stream);
        return err;
    }
    rasterize_kernel<IN_C, OUT_C, DIRECT><<<grid, RASTER_THREADS, 0, stream>>>(a, ntx, nullptr);
    return cudaGetLastError();
}

} // namespace

cudaError_t launch_rasterize(const ProjArgs& a, cudaStream_t stream) {
    if (a.in_cplx && a.out_cplx)
        return launch_typed<true, true>(a, stream);
    if (a.in_cplx)
        return launch_typed<true, false>(a, stream);
    return launch_typed<false, false>(a, stream);
}

} // namespace nb
