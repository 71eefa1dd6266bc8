// extract_central_slices_3d on sm_100a: one thread per output pixel, 3-D spectrum interpolation of
// the volume (FourierExtract, noa/xform/FourierProject.hpp:632-694).
//
// Work decomposition: a CTA owns 256 consecutive pixels of the flattened (y, u) plane of ONE slice,
// so its rotation is uniform and its taps land on a compact patch of the volume, which the L1 and the
// 126 MB L2 keep resident (a 256^3 complex64 rfft volume is 67.6 MB). Taps are read through the
// non-coherent path (ld.global.nc); outputs are written once, coalesced.
//
// The w-windowed form (wsize > 1) keeps the reference's semantics — outputs are the windowed sum over
// the w offsets of the z-shifted samples — but sums in registers, in w order, instead of zeroing the
// outputs and adding atomically, so it is deterministic and needs no extra pass.
#include "fp_args.cuh"

namespace nb {
namespace {

constexpr int EXTRACT_THREADS = 256;

template<int I, bool IN_C, bool OUT_C>
__global__ void __launch_bounds__(EXTRACT_THREADS)
extract_kernel(const __grid_constant__ ProjArgs a, int tiles_per_slice, int64_t n_tiles) {
    const int wp = a.slice_w / 2 + 1;
    const int plane = a.slice_h * wp;
    const Spectrum3 sp{a.vol_d, a.vol_h, a.vol_w, a.in_centered};
    const bool has_out_w = a.out_w.present;
    const bool has_in_w = a.in_w.present;

    for (int64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        const int64_t b = tile / tiles_per_slice;
        const int p = static_cast<int>(tile - b * tiles_per_slice) * EXTRACT_THREADS + static_cast<int>(threadIdx.x);
        if (p >= plane)
            continue;
        const int y = p / wp;
        const int u = p - y * wp;
        const int v = index2frequency(a.out_centered, y, a.slice_h);

        float fz, fy, fx;
        slice2grid(div(static_cast<float>(v), a.f_slice0), div(static_cast<float>(u), a.f_slice1),
                   a.scale, a.rot, b, a.ews, fz, fy, fx);

        float2 value = make_float2(0.f, 0.f);
        float weight = 0.f;
        if (a.wsize <= 1) {
            if (dot3(fz, fy, fx, fz, fy, fx) <= a.cutoff_sqd) {
                const float q0 = mul(fz, a.target0), q1 = mul(fy, a.target1), q2 = mul(fx, a.target2);
                value = to_output<IN_C, OUT_C>(interp_spectrum_3d<I, IN_C>(a.in, sp, q0, q1, q2));
                if (has_out_w)
                    weight = has_in_w ? interp_spectrum_3d<I, false>(a.in_w, sp, q0, q1, q2).x : 1.f;
            }
        } else {
            for (int w = 0; w < a.wsize; ++w) {
                const float off = div(static_cast<float>(w - a.wsize / 2), a.target0);
                const float gz = add(fz, off);
                if (dot3(gz, fy, fx, gz, fy, fx) > a.cutoff_sqd)
                    continue;
                const float q0 = mul(gz, a.target0), q1 = mul(fy, a.target1), q2 = mul(fx, a.target2);
                const float cw = windowed_sinc(off, a.efs, a.efb);
                const float2 iv = to_output<IN_C, OUT_C>(interp_spectrum_3d<I, IN_C>(a.in, sp, q0, q1, q2));
                value = cadd(value, cmul(iv, cw));
                if (has_out_w) {
                    const float iw = has_in_w ? interp_spectrum_3d<I, false>(a.in_w, sp, q0, q1, q2).x : 1.f;
                    weight = add(weight, mul(iw, cw));
                }
            }
        }
        dst_store<OUT_C>(a.out, b, y, u, value);
        if (has_out_w)
            store_real(a.out_w, b, y, u, weight);
    }
}

template<int I, bool IN_C, bool OUT_C>
cudaError_t launch_typed(const ProjArgs& a, cudaStream_t stream) {
    const int wp = a.slice_w / 2 + 1;
    const int plane = a.slice_h * wp;
    const int tiles_per_slice = (plane + EXTRACT_THREADS - 1) / EXTRACT_THREADS;
    const int64_t n_tiles = static_cast<int64_t>(tiles_per_slice) * a.n_slices;
    if (n_tiles == 0)
        return cudaSuccess;
    const int64_t max_grid = static_cast<int64_t>(sm_count()) * 8 * 64;
    const int grid = static_cast<int>(n_tiles < max_grid ? n_tiles : max_grid);
    extract_kernel<I, IN_C, OUT_C><<<grid, EXTRACT_THREADS, 0, stream>>>(a, tiles_per_slice, n_tiles);
    return cudaGetLastError();
}

template<int I>
cudaError_t launch_interp(const ProjArgs& a, cudaStream_t stream) {
    if (a.in_cplx && a.out_cplx)
        return launch_typed<I, true, true>(a, stream);
    if (a.in_cplx)
        return launch_typed<I, true, false>(a, stream);
    return launch_typed<I, false, false>(a, stream);
}

} // namespace

cudaError_t launch_extract(const ProjArgs& a, cudaStream_t stream) {
    switch (a.interp) {
        case I_NEAREST: return launch_interp<I_NEAREST>(a, stream);
        case I_LINEAR: return launch_interp<I_LINEAR>(a, stream);
        case I_CUBIC: return launch_interp<I_CUBIC>(a, stream);
        case I_BSPLINE: return launch_interp<I_BSPLINE>(a, stream);
        case I_LANCZOS4: return launch_interp<I_LANCZOS4>(a, stream);
        case I_LANCZOS6: return launch_interp<I_LANCZOS6>(a, stream);
        case I_LANCZOS8: return launch_interp<I_LANCZOS8>(a, stream);
        default: return cudaErrorInvalidValue;
    }
}

} // namespace nb
