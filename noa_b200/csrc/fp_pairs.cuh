// Pair copy of a volume for LINEAR extraction, shared by the per-call and batched extraction kernels.
//
// The copy is dense (D x H x W/2+1) and element (z, y, x) holds the two x-neighbours v[z][y][x] and
// v[z][y][x+1] (zero past the last column) as one float4, so the 2x2x2 trilinear cell is 4 aligned
// 16-byte loads instead of 8 scattered 8-byte ones. The taps, weights and summation order are those of
// interp_linear_3d, so results are bit-identical to the generic path.
#pragma once

#include "fp_args.cuh"

namespace nb {

__device__ __forceinline__ float2 interp_linear_pairs(const float4* __restrict__ pairs, int sz, int sy,
                                                      const Spectrum3& sp, float q0, float q1, float q2) {
    float conjugate = 1.f;
    if (q2 < 0.f) {
        q0 = -q0; q1 = -q1; q2 = -q2;
        conjugate = -1.f;
    }
    const float fl0 = floorf(q0), fl1 = floorf(q1), fl2 = floorf(q2);
    const int b0 = static_cast<int>(fl0), b1 = static_cast<int>(fl1), b2 = static_cast<int>(fl2);
    const float t0 = sub(q0, fl0), t1 = sub(q1, fl1), t2 = sub(q2, fl2);
    const float w0[2] = {sub(1.f, t0), t0};
    const float w1[2] = {sub(1.f, t1), t1};
    const float w20 = sub(1.f, t2);
    const int lo0 = -sp.n0 / 2, hi0 = (sp.n0 - 1) / 2;
    const int lo1 = -sp.n1 / 2, hi1 = (sp.n1 - 1) / 2;
    const int hi2 = sp.n2 / 2;
    const bool okx0 = b2 >= 0 && b2 <= hi2;
    const bool okx1 = b2 + 1 >= 0 && b2 + 1 <= hi2;
    float2 value = make_float2(0.f, 0.f);
    // Interior cells (every tap inside the volume, the two rows of each axis adjacent in memory: not
    // across the non-centered layout's wrap at -1): the same terms in the same order, from one base
    // offset, with the four loads issued together.
    if (b0 >= lo0 && b0 + 1 <= hi0 && b1 >= lo1 && b1 + 1 <= hi1 && okx0 && okx1 &&
        (sp.centered || (b0 != -1 && b1 != -1))) {
        const float4* p = pairs + (frequency2index(sp.centered, b0, sp.n0) * sz +
                                   frequency2index(sp.centered, b1, sp.n1) * sy + b2);
        float4 q[4];
        q[0] = ldg_evict_last_half(p);
        q[1] = ldg_evict_last_half(p + sy);
        q[2] = ldg_evict_last_half(p + sz);
        q[3] = ldg_evict_last_half(p + sz + sy);
#pragma unroll
        for (int z = 0; z < 2; ++z) {
            float2 vz = make_float2(0.f, 0.f);
#pragma unroll
            for (int y = 0; y < 2; ++y) {
                float2 vy = make_float2(0.f, 0.f);
                vy = cfma(make_float2(q[z * 2 + y].x, q[z * 2 + y].y), w20, vy);
                vy = cfma(make_float2(q[z * 2 + y].z, q[z * 2 + y].w), t2, vy);
                vz = cfma(vy, w1[y], vz);
            }
            value = cfma(vz, w0[z], value);
        }
        value.y *= conjugate;
        return value;
    }
#pragma unroll
    for (int z = 0; z < 2; ++z) {
        const int iz = b0 + z;
        const bool okz = iz >= lo0 && iz <= hi0;
        const int oz = frequency2index(sp.centered, iz, sp.n0) * sz;
        float2 vz = make_float2(0.f, 0.f);
#pragma unroll
        for (int y = 0; y < 2; ++y) {
            const int iy = b1 + y;
            const bool oky = iy >= lo1 && iy <= hi1;
            float2 vy = make_float2(0.f, 0.f);
            if (okz && oky && okx0) {
                const float4 p = ldg_evict_last_half(pairs + (oz + frequency2index(sp.centered, iy, sp.n1) * sy + b2));
                vy = cfma(make_float2(p.x, p.y), w20, vy);
                if (okx1)
                    vy = cfma(make_float2(p.z, p.w), t2, vy);
            }
            vz = cfma(vy, w1[y], vz);
        }
        value = cfma(vz, w0[z], value);
    }
    value.y *= conjugate;
    return value;
}

// slice2grid for a Mat33 rotation with no scaling and no Ewald curvature, when the slice's matrix
// column 0 is finite: rotate() computes ((m_k0 * 0) + (m_k1 * f0)) + (m_k2 * f1), and for finite m_k0
// the first product is a zero whose sign never reaches the result (the coordinates then decide the
// cutoff, the cell, its weights and the Friedel flip the same way), so it is left out.
__device__ __forceinline__ void slice2grid_lean(const float* m, float f0, float f1, float& z, float& y, float& x) {
    z = add(mul(m[1], f0), mul(m[2], f1));
    y = add(mul(m[4], f0), mul(m[5], f1));
    x = add(mul(m[7], f0), mul(m[8], f1));
}

// Whether slice b of `a` can take slice2grid_lean; `m` is then its matrix.
__device__ __forceinline__ bool lean_rotation(const ProjArgs& a, int64_t b, const float*& m) {
    if (a.rot.kind != 2 || a.scale.kind != 0 || a.ews.on)
        return false;
    m = xform_ptr(a.rot, b, 12);
    return isfinite(m[0]) && isfinite(m[3]) && isfinite(m[6]);
}

// Whether a call may read the pair copy: LINEAR, complex volume given as an array, no input weights,
// no w-window (per-call extractions take extract_pairs_w_kernel for that), a copy addressable in 32
// bits. Scaling and the Ewald-sphere curvature only change the coordinates (slice2grid), which the
// pair kernels compute as the generic ones do.
inline bool pairs_apply(const ProjArgs& a) {
    const int64_t vox = static_cast<int64_t>(a.vol_d) * a.vol_h * (a.vol_w / 2 + 1);
    return a.interp == I_LINEAR && a.in_cplx && !a.in_w.present && !a.in.is_value && a.wsize <= 1 &&
           vox < (int64_t(1) << 31);
}

// Writes the pair copy of a.in (a.vol_d x a.vol_h x a.vol_w/2+1 complex values) to `pairs`. With
// `priority`, the launch carries that scheduling priority (kept by a graph captured from it).
cudaError_t launch_make_pairs(const ProjArgs& a, float4* pairs, cudaStream_t stream, const int* priority = nullptr);

// The per-call LINEAR extraction over a pair copy of a.in: one grid of (slice tile, slice) CTAs
// (extract_pairs_kernel, or extract_pairs_w_kernel with a w-window).
cudaError_t launch_extract_pairs(const ProjArgs& a, const float4* pairs, cudaStream_t stream);

} // namespace nb
