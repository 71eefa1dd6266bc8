// Kernels of rasterize_central_slices_3d (see fp_rasterize.cu for the design), shared by the
// launchers that own their scratch differently.
#pragma once

#include "fp_args.cuh"

namespace nb {
namespace raster {

constexpr int TY = 16, TX = 16, RASTER_THREADS = TY * TX;

enum Mode { DIRECT = 0, SCRATCH = 1 };

// Where one tap goes: the caller's grids (DIRECT) or the dense interleaved scratch (SCRATCH).
template<bool OUT_C, int MODE>
struct Sink {
    DstView vol, volw;
    void* scratch;
    int sz, sy;           // dense scratch strides (x stride 1)
    bool has_w;

    __device__ __forceinline__ void add(int iw, int iv, int iu, float2 v, float w) const {
        if constexpr (MODE == SCRATCH) {
            const int off = iw * sz + iv * sy + iu;
            if constexpr (OUT_C)
                atomicAdd(static_cast<float4*>(scratch) + off, make_float4(v.x, v.y, w, 0.f));
            else
                atomicAdd(static_cast<float2*>(scratch) + off, make_float2(v.x, w));
        } else {
            const int64_t off = iw * vol.s0 + iv * vol.s1 + iu * vol.s2;
            if constexpr (OUT_C)
                atomicAdd(static_cast<float2*>(vol.data) + off, v);
            else
                atomicAdd(static_cast<float*>(vol.data) + off, v.x);
            if (has_w)
                atomicAdd(static_cast<float*>(volw.data) + (iw * volw.s0 + iv * volw.s1 + iu * volw.s2), w);
        }
    }
};

template<bool IN_C, bool OUT_C, int MODE>
__global__ void __launch_bounds__(RASTER_THREADS)
rasterize_kernel(const __grid_constant__ ProjArgs a, int ntx, void* scratch) {
    const int wp = a.slice_w / 2 + 1;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int y = (blockIdx.x / ntx) * TY + (warp >> 1) * 4 + (lane >> 3);
    const int u = (blockIdx.x % ntx) * TX + (warp & 1) * 8 + (lane & 7);
    if (u >= wp || y >= a.slice_h)
        return;
    const int D = a.vol_d, H = a.vol_h, WP = a.vol_w / 2 + 1;
    const bool vc = a.out_centered;
    const bool has_out_w = a.out_w.present;
    const bool has_in_w = a.in_w.present;
    const Sink<OUT_C, MODE> sink{a.out, a.out_w, scratch, H * WP, WP, has_out_w};
    const int v = index2frequency(a.in_centered, y, a.slice_h);
    const float f0 = div(static_cast<float>(v), a.f_slice0);
    const float f1 = div(static_cast<float>(u), a.f_slice1);

    for (int64_t b = blockIdx.y; b < a.n_slices; b += gridDim.y) {
        float fz, fy, fx;
        slice2grid(f0, f1, a.scale, a.rot, b, a.ews, fz, fy, fx);
        if (dot3(fz, fy, fx, fz, fy, fx) > a.cutoff_sqd)
            continue;

        float conjugate = 1.f;
        if (fx < 0.f) {
            fz = -fz; fy = -fy; fx = -fx;
            if (IN_C)
                conjugate = -1.f;
        }
        const float q0 = mul(fz, a.target0), q1 = mul(fy, a.target1), q2 = mul(fx, a.target2);

        float2 value = src_read_stream<IN_C>(a.in, b, y, u);
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
            const int iw = frequency2index(vc, b0 + w, D);
            if (iw < 0 || iw >= D)
                continue;
#pragma unroll
            for (int vv = 0; vv < 2; ++vv) {
                const int iv = frequency2index(vc, b1 + vv, H);
                if (iv < 0 || iv >= H)
                    continue;
                const float kwv = mul(fr[w][0], fr[vv][1]);
#pragma unroll
                for (int uu = 0; uu < 2; ++uu) {
                    const int iu = b2 + uu;
                    if (iu < 0 || iu >= WP)
                        continue;
                    const float k = mul(kwv, fr[uu][2]);
                    sink.add(iw, iv, iu, cmul(value, k), mul(weight, k));
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
                const int iw = frequency2index(vc, -(b0 + w), D);
                if (iw < 0 || iw >= D)
                    continue;
#pragma unroll
                for (int vv = 0; vv < 2; ++vv) {
                    const int iv = frequency2index(vc, -(b1 + vv), H);
                    if (iv < 0 || iv >= H)
                        continue;
                    const float k = mul(mul(fr[w][0], fr[vv][1]), fr[0][2]);
                    sink.add(iw, iv, 0, cmul(cv, k), mul(weight, k));
                }
            }
        }
    }
}

// grid += scratch values; weights += scratch weights (caller's strides).
template<bool OUT_C>
__global__ void finalize_kernel(const __grid_constant__ ProjArgs a, const void* __restrict__ scratch) {
    const int D = a.vol_d, H = a.vol_h, WP = a.vol_w / 2 + 1;
    const int64_t n = static_cast<int64_t>(D) * H * WP;
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int x = static_cast<int>(i % WP);
        const int64_t zy = i / WP;
        const int y = static_cast<int>(zy % H), z = static_cast<int>(zy / H);
        float2 v;
        float w;
        if constexpr (OUT_C) {
            const float4 s = static_cast<const float4*>(scratch)[i];
            v = make_float2(s.x, s.y);
            w = s.z;
        } else {
            const float2 s = static_cast<const float2*>(scratch)[i];
            v = make_float2(s.x, 0.f);
            w = s.y;
        }
        dst_store<OUT_C>(a.out, z, y, x, cadd(dst_load<OUT_C>(a.out, z, y, x), v));
        store_real(a.out_w, z, y, x, add(load_real(a.out_w, z, y, x), w));
    }
}

} // namespace raster
} // namespace nb
