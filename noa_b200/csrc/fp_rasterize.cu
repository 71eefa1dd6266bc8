// rasterize_central_slices_3d on sm_100a: one thread per slice pixel, trilinear scatter of the pixel
// into the 2x2x2 voxels around its rotated frequency, plus the Hermitian-plane mirror taps
// (FourierInsertRasterize, noa/xform/FourierProject.hpp:238-373).
//
// Complex values are added with one vector reduction (red.global.add.v2.f32, sm_90+) per tap instead
// of two scalar ones; weights with a scalar f32 reduction.
//
// Deliberate deviation from the reference: the reference bounds the u tap by the LOGICAL volume width
// (FourierProject.hpp:327-329), so a tap at u = W/2+1 passes and lands in the next row (or past the
// end of the array). Here u is bounded by the physical width W/2+1. For even sizes and cutoffs <= 0.5
// such taps carry a zero weight, so the results are the same.
#include "fp_args.cuh"

namespace nb {
namespace {

constexpr int RASTER_THREADS = 256;

template<bool OUT_C>
__device__ __forceinline__ void red_value(const DstView& d, int64_t iw, int64_t iv, int64_t iu, float2 v) {
    const int64_t off = iw * d.s0 + iv * d.s1 + iu * d.s2;
    if constexpr (OUT_C)
        atomicAdd(static_cast<float2*>(d.data) + off, v);
    else
        atomicAdd(static_cast<float*>(d.data) + off, v.x);
}

__device__ __forceinline__ void red_weight(const DstView& d, int64_t iw, int64_t iv, int64_t iu, float w) {
    atomicAdd(static_cast<float*>(d.data) + (iw * d.s0 + iv * d.s1 + iu * d.s2), w);
}

template<bool IN_C, bool OUT_C>
__global__ void __launch_bounds__(RASTER_THREADS)
rasterize_kernel(const __grid_constant__ ProjArgs a, int tiles_per_slice, int64_t n_tiles) {
    const int wp = a.slice_w / 2 + 1;
    const int plane = a.slice_h * wp;
    const int D = a.vol_d, H = a.vol_h, WP = a.vol_w / 2 + 1;
    const bool vol_centered = a.out_centered;
    const bool has_out_w = a.out_w.present;
    const bool has_in_w = a.in_w.present;

    for (int64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        const int64_t b = tile / tiles_per_slice;
        const int p = static_cast<int>(tile - b * tiles_per_slice) * RASTER_THREADS + static_cast<int>(threadIdx.x);
        if (p >= plane)
            continue;
        const int y = p / wp;
        const int u = p - y * wp;
        const int v = index2frequency(a.in_centered, y, a.slice_h);

        float fz, fy, fx;
        slice2grid(div(static_cast<float>(v), a.f_slice0), div(static_cast<float>(u), a.f_slice1),
                   a.scale, a.rot, b, a.ews, fz, fy, fx);
        if (dot3(fz, fy, fx, fz, fy, fx) > a.cutoff_sqd)
            continue;

        float conjugate = 1.f;
        if (fx < 0.f) {
            fz = -fz; fy = -fy; fx = -fx;
            if (IN_C)
                conjugate = -1.f;
        }
        const float q0 = mul(fz, a.target0), q1 = mul(fy, a.target1), q2 = mul(fx, a.target2);

        float2 value = src_read<IN_C>(a.in, b, y, u);
        if constexpr (IN_C && OUT_C)
            value = cmul(value, conjugate); // noa multiplies by -1 here, it does not conjugate
        else
            value = to_output<IN_C, OUT_C>(value);
        float weight = 0.f;
        if (has_out_w)
            weight = has_in_w ? src_read_real(a.in_w, b, y, u) : 1.f;

        const float fl0 = floorf(q0), fl1 = floorf(q1), fl2 = floorf(q2);
        const int b0 = static_cast<int>(fl0), b1 = static_cast<int>(fl1), b2 = static_cast<int>(fl2);
        float fr[2][3];
        fr[1][0] = sub(q0, static_cast<float>(b0));
        fr[1][1] = sub(q1, static_cast<float>(b1));
        fr[1][2] = sub(q2, static_cast<float>(b2));
        fr[0][0] = sub(1.f, fr[1][0]);
        fr[0][1] = sub(1.f, fr[1][1]);
        fr[0][2] = sub(1.f, fr[1][2]);

#pragma unroll
        for (int w = 0; w < 2; ++w) {
            const int iw = frequency2index(vol_centered, b0 + w, D);
            if (iw < 0 || iw >= D)
                continue;
#pragma unroll
            for (int vv = 0; vv < 2; ++vv) {
                const int iv = frequency2index(vol_centered, b1 + vv, H);
                if (iv < 0 || iv >= H)
                    continue;
                const float kwv = mul(fr[w][0], fr[vv][1]);
#pragma unroll
                for (int uu = 0; uu < 2; ++uu) {
                    const int iu = b2 + uu;
                    if (iu < 0 || iu >= WP)
                        continue;
                    const float k = mul(kwv, fr[uu][2]);
                    red_value<OUT_C>(a.out, iw, iv, iu, cmul(value, k));
                    if (has_out_w)
                        red_weight(a.out_w, iw, iv, iu, mul(weight, k));
                }
            }
        }

        // Hermitian symmetry on the redundant x == 0 plane (FourierProject.hpp:347-372).
        if (b2 == 0) {
            float2 cv = value;
            if constexpr (OUT_C)
                cv.y = -cv.y;
#pragma unroll
            for (int w = 0; w < 2; ++w) {
                const int iw = frequency2index(vol_centered, -(b0 + w), D);
                if (iw < 0 || iw >= D)
                    continue;
#pragma unroll
                for (int vv = 0; vv < 2; ++vv) {
                    const int iv = frequency2index(vol_centered, -(b1 + vv), H);
                    if (iv < 0 || iv >= H)
                        continue;
                    const float k = mul(mul(fr[w][0], fr[vv][1]), fr[0][2]);
                    red_value<OUT_C>(a.out, iw, iv, 0, cmul(cv, k));
                    if (has_out_w)
                        red_weight(a.out_w, iw, iv, 0, mul(weight, k));
                }
            }
        }
    }
}

template<bool IN_C, bool OUT_C>
cudaError_t launch_typed(const ProjArgs& a, cudaStream_t stream) {
    const int wp = a.slice_w / 2 + 1;
    const int plane = a.slice_h * wp;
    const int tiles_per_slice = (plane + RASTER_THREADS - 1) / RASTER_THREADS;
    const int64_t n_tiles = static_cast<int64_t>(tiles_per_slice) * a.n_slices;
    if (n_tiles == 0)
        return cudaSuccess;
    const int64_t max_grid = static_cast<int64_t>(sm_count()) * 8 * 64;
    const int grid = static_cast<int>(n_tiles < max_grid ? n_tiles : max_grid);
    rasterize_kernel<IN_C, OUT_C><<<grid, RASTER_THREADS, 0, stream>>>(a, tiles_per_slice, n_tiles);
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
