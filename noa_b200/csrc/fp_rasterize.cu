// rasterize_central_slices_3d on sm_100a: trilinear scatter of every slice pixel into the 2x2x2 voxels
// around its rotated frequency, plus the Hermitian-plane mirror taps (FourierInsertRasterize,
// noa/xform/FourierProject.hpp:238-373).
//
// The scatter is bound by the L2 reduction rate, which counts one operation per lane whatever its
// width. So a pixel's value and weight for one voxel travel in ONE reduction: the kernel accumulates
// into a private interleaved grid — float4 (re, im, w, -) for complex values with weights — taken from a
// stream-ordered pool, zeroed first, and a finalize pass adds it into the caller's value and weight
// grids (whatever their layout and strides). That grid is centered and padded to every tap the cutoff
// lets a pixel reach, so the scatter needs no bounds tests. Each thread walks a run of 16 rows of one
// column and merges the taps that successive pixels share before reducing (rasterize_runs_kernel), so
// a pixel costs about 5 reductions instead of 8. If the accumulator cannot be allocated (or would not
// fit 32-bit offsets), one thread per pixel reduces into an unpadded scratch or the caller's grids.
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

// Fallback without the padded accumulator: one thread per pixel, unpadded scratch (with weights) or
// reductions straight into the caller's grids.
template<bool IN_C, bool OUT_C>
cudaError_t launch_tiles(const ProjArgs& a, cudaStream_t stream) {
    const int wp = a.slice_w / 2 + 1;
    const int ntx = (wp + TX - 1) / TX, nty = (a.slice_h + TY - 1) / TY;
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

template<bool IN_C, bool OUT_C, bool W>
cudaError_t launch_runs(const ProjArgs& a, const AccGrid& g, cudaStream_t stream, bool& done) {
    done = false;
    using T = typename AccElem<OUT_C, W>::T;
    const size_t bytes = static_cast<size_t>(g.elements) * sizeof(T);
    void* acc = scratch_alloc(bytes, stream);
    if (!acc)
        return cudaSuccess;  // no memory for the accumulator: the caller takes the tile path
    cudaError_t err = cudaMemsetAsync(acc, 0, bytes, stream);
    if (err == cudaSuccess) {
        const int64_t threads = static_cast<int64_t>(a.slice_w / 2 + 1) * ((a.slice_h + RUN - 1) / RUN);
        const dim3 grid(static_cast<unsigned>((threads + RASTER_THREADS - 1) / RASTER_THREADS),
                        static_cast<unsigned>(a.n_slices < 65535 ? a.n_slices : 65535));
        rasterize_runs_kernel<IN_C, OUT_C, W><<<grid, RASTER_THREADS, 0, stream>>>(a, g, acc);
        const int64_t vox = static_cast<int64_t>(a.vol_d) * a.vol_h * (a.vol_w / 2 + 1);
        const int64_t blocks = (vox + 255) / 256;
        const int grid_f = static_cast<int>(blocks < static_cast<int64_t>(sm_count()) * 16 ? blocks : sm_count() * 16);
        finalize_padded_kernel<OUT_C, W><<<grid_f, 256, 0, stream>>>(a, g, acc);
        err = cudaGetLastError();
    }
    scratch_free(acc, stream);
    done = err == cudaSuccess;
    return err;
}

template<bool IN_C, bool OUT_C>
cudaError_t launch_typed(const ProjArgs& a, cudaStream_t stream) {
    if (a.n_slices == 0)
        return cudaSuccess;
    const AccGrid g = make_acc_grid(a);
    if (g.elements > 0) {
        bool done = false;
        const cudaError_t err = a.out_w.present ? launch_runs<IN_C, OUT_C, true>(a, g, stream, done)
                                                : launch_runs<IN_C, OUT_C, false>(a, g, stream, done);
        if (err != cudaSuccess || done)
            return err;
    }
    return launch_tiles<IN_C, OUT_C>(a, stream);
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
