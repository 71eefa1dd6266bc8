// Kernels of rasterize_central_slices_3d (see fp_rasterize.cu for the design), shared by the
// launchers that own their scratch differently.
#pragma once

#include "fp_args.cuh"

#include <algorithm>
#include <cmath>

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

// ---------------------------------------------------------------------------------------------------
// Run-accumulating form over a padded, centered accumulator.
//
// Accumulator: a private dense grid indexed by frequency, z and y in [-R0, R0] and [-R1, R1], x in
// [0, n2): R and n2 cover every tap a pixel inside the cutoff can reach (and the Hermitian mirror of
// it), so the hot loop needs no bounds test and no frequency2index. Elements interleave value and
// weight — float4 (re, im, w, -), float2 (re, im) or (v, w), or float — so one reduction carries a tap.
// The finalize pass adds into each voxel of the caller's grid, in the caller's layout, the cells the
// reference's per-tap index test sends there; the rest (taps it drops) are never read back.
//
// Runs: a thread walks RUN consecutive rows y of one column u. Consecutive rows land at most one voxel
// apart along each axis, so the 2x2x2 cells of successive pixels overlap: the thread keeps the pending
// sums of its cell in registers and, when the next pixel's cell moves by d in {-1, 0, +1} along the
// axes, emits only the corners it leaves and slides the rest over. A larger jump (the non-centered
// row wrap, the Friedel flip) emits the whole cell. Pending sums are keyed by target voxel only — each
// pixel's contribution already carries its own flip and conjugation — so merging changes nothing but
// the order of the float additions, which the atomic scatter leaves unspecified anyway.
// ---------------------------------------------------------------------------------------------------
constexpr int RUN = 16;

struct AccGrid {
    int r0, r1;     // z and y frequencies held: [-r0, r0], [-r1, r1]
    int n2;         // x frequencies held: [0, n2)
    int sz, sy;     // element strides (x stride 1)
    float qlim0, qlim1, qlim2;  // |q| bounds every tap cell fits in (only non-finite input exceeds them)
    int64_t elements;
};

// Accumulator geometry for a launch, or elements = -1 if it does not fit 32-bit offsets.
inline AccGrid make_acc_grid(const ProjArgs& a) {
    AccGrid g{};
    const double c = std::sqrt(static_cast<double>(a.cutoff_sqd)) * (1.0 + 1e-6);
    if (!std::isfinite(c) || !std::isfinite(a.target0) || !std::isfinite(a.target1) || !std::isfinite(a.target2)) {
        g.elements = -1;
        return g;
    }
    auto reach = [&](float t) {
        const double r = std::ceil(c * static_cast<double>(t)) + 2.0;
        return r > 1e9 ? int64_t(1) << 40 : static_cast<int64_t>(r);
    };
    const int64_t r0 = std::max<int64_t>(a.vol_d / 2, reach(a.target0));
    const int64_t r1 = std::max<int64_t>(a.vol_h / 2, reach(a.target1));
    const int64_t n2 = std::max<int64_t>(a.vol_w / 2 + 1, reach(a.target2) + 1);
    const int64_t e = (2 * r0 + 1) * (2 * r1 + 1) * n2;
    if (r0 > (1 << 20) || r1 > (1 << 20) || n2 > (1 << 20) || e >= (int64_t(1) << 31)) {
        g.elements = -1;
        return g;
    }
    g.r0 = static_cast<int>(r0);
    g.r1 = static_cast<int>(r1);
    g.n2 = static_cast<int>(n2);
    g.sy = g.n2;
    g.sz = static_cast<int>((2 * r1 + 1) * n2);
    g.qlim0 = static_cast<float>(r0 - 2);
    g.qlim1 = static_cast<float>(r1 - 2);
    g.qlim2 = static_cast<float>(n2 - 3);
    g.elements = e;
    return g;
}

template<bool OUT_C, bool W>
struct AccElem;
template<> struct AccElem<true, true> { using T = float4; };
template<> struct AccElem<true, false> { using T = float2; };
template<> struct AccElem<false, true> { using T = float2; };
template<> struct AccElem<false, false> { using T = float; };

// The reductions carry an L2 evict_last hint on half of the lines they touch: the accumulator is
// slightly larger than the L2 and the slices stream past it, so keeping part of it resident saves
// misses (2-3 % at 256^3 x 4096; a fraction of 1.0 gave 2 %).
__device__ __forceinline__ unsigned long long acc_policy() {
    unsigned long long pol;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 0.5;" : "=l"(pol));
    return pol;
}

template<bool OUT_C, bool W>
__device__ __forceinline__ void acc_add(void* acc, int off, float2 v, float w) {
    using T = typename AccElem<OUT_C, W>::T;
    T* p = static_cast<T*>(acc) + off;
    const unsigned long long pol = acc_policy();
    if constexpr (OUT_C && W)
        asm volatile("red.global.add.L2::cache_hint.v4.f32 [%0], {%1, %2, %3, %4}, %5;"
                     :: "l"(p), "f"(v.x), "f"(v.y), "f"(w), "f"(0.f), "l"(pol) : "memory");
    else if constexpr (OUT_C)
        asm volatile("red.global.add.L2::cache_hint.v2.f32 [%0], {%1, %2}, %3;"
                     :: "l"(p), "f"(v.x), "f"(v.y), "l"(pol) : "memory");
    else if constexpr (W)
        asm volatile("red.global.add.L2::cache_hint.v2.f32 [%0], {%1, %2}, %3;"
                     :: "l"(p), "f"(v.x), "f"(w), "l"(pol) : "memory");
    else
        asm volatile("red.global.add.L2::cache_hint.f32 [%0], %1, %2;" :: "l"(p), "f"(v.x), "l"(pol) : "memory");
}

// Corner c = 4 c0 + 2 c1 + c2 of a cell; its offset from corner 0.
__device__ __forceinline__ int corner_offset(int c, const AccGrid& g) {
    return (c >> 2) * g.sz + ((c >> 1) & 1) * g.sy + (c & 1);
}

// One stage of the slide: along the axis whose corner bit is S, move the cell by +1 (up) or -1 (dn).
// Vacated corners keep a dead copy; their mask bits are cleared by the caller.
template<int S>
__device__ __forceinline__ void slide_values(float2 (&v)[8], float (&w)[8], bool up, bool dn) {
#pragma unroll
    for (int lo = 0; lo < 8; ++lo) {
        if (lo & S)
            continue;
        const int hi = lo | S;
        const float2 vl = v[lo], vh = v[hi];
        const float wl = w[lo], wh = w[hi];
        v[lo] = up ? vh : vl;
        w[lo] = up ? wh : wl;
        v[hi] = dn ? vl : vh;
        w[hi] = dn ? wl : wh;
    }
}

template<int S>
__device__ __forceinline__ unsigned slide_mask(unsigned m, bool up, bool dn) {
    constexpr unsigned LO = S == 4 ? 0x0Fu : S == 2 ? 0x33u : 0x55u;  // corners with bit S clear
    if (up)
        return (m >> S) & LO;
    if (dn)
        return (m << S) & (~LO & 0xFFu);
    return m;
}

// One run: column u, rows [y0, y0 + RUN) of slice b, into the accumulator.
template<bool IN_C, bool OUT_C, bool W>
__device__ __forceinline__ void rasterize_run(const ProjArgs& a, const AccGrid& g, void* __restrict__ acc,
                                              int64_t b, int u, int y0) {
    const int y_end = min(y0 + RUN, a.slice_h);
    const bool has_in_w = a.in_w.present;
    const float f1 = div(static_cast<float>(u), a.f_slice1);
    {
        float2 cv[8];
        float cw[8];
        unsigned mask = 0;
        int c0 = 0, c1 = 0, c2 = 0;  // frequency of corner 0
        int base = 0;                // its accumulator offset

        for (int y = y0; y < y_end; ++y) {
            const float f0 = div(static_cast<float>(index2frequency(a.in_centered, y, a.slice_h)), a.f_slice0);
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
            if (!(fabsf(q0) <= g.qlim0 && fabsf(q1) <= g.qlim1 && q2 <= g.qlim2))
                continue;  // non-finite coordinates only: finite ones inside the cutoff always fit
            float2 value = src_read_stream<IN_C>(a.in, b, y, u);
            if constexpr (IN_C && OUT_C)
                value = cmul(value, conjugate); // noa multiplies by -1 here, it does not conjugate
            else
                value = to_output<IN_C, OUT_C>(value);
            float weight = 0.f;
            if constexpr (W)
                weight = has_in_w ? src_read_real(a.in_w, b, y, u) : 1.f;

            const int n0 = static_cast<int>(floorf(q0)), n1 = static_cast<int>(floorf(q1)),
                      n2 = static_cast<int>(floorf(q2));
            float fr[2][3];
            fr[1][0] = sub(q0, static_cast<float>(n0));
            fr[1][1] = sub(q1, static_cast<float>(n1));
            fr[1][2] = sub(q2, static_cast<float>(n2));
            fr[0][0] = sub(1.f, fr[1][0]);
            fr[0][1] = sub(1.f, fr[1][1]);
            fr[0][2] = sub(1.f, fr[1][2]);

            const int d0 = n0 - c0, d1 = n1 - c1, d2 = n2 - c2;
            const bool jump = d0 < -1 || d0 > 1 || d1 < -1 || d1 > 1 || d2 < -1 || d2 > 1;
            const bool up0 = d0 > 0, dn0 = d0 < 0, up1 = d1 > 0, dn1 = d1 < 0, up2 = d2 > 0, dn2 = d2 < 0;
            // Emit the corners the cell leaves (all of them on a jump), at the old position.
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                const bool leaves = jump || ((c & 4) ? dn0 : up0) || ((c & 2) ? dn1 : up1) || ((c & 1) ? dn2 : up2);
                if (leaves && ((mask >> c) & 1u))
                    acc_add<OUT_C, W>(acc, base + corner_offset(c, g), cv[c], cw[c]);
            }
            if (jump) {
                mask = 0;
            } else {
                slide_values<4>(cv, cw, up0, dn0);
                mask = slide_mask<4>(mask, up0, dn0);
                slide_values<2>(cv, cw, up1, dn1);
                mask = slide_mask<2>(mask, up1, dn1);
                slide_values<1>(cv, cw, up2, dn2);
                mask = slide_mask<1>(mask, up2, dn2);
            }
            c0 = n0; c1 = n1; c2 = n2;
            base = ((n0 + g.r0) * (2 * g.r1 + 1) + (n1 + g.r1)) * g.n2 + n2;

#pragma unroll
            for (int c = 0; c < 8; ++c) {
                const float k = mul(mul(fr[c >> 2][0], fr[(c >> 1) & 1][1]), fr[c & 1][2]);
                const float2 pv = cmul(value, k);
                const float pw = mul(weight, k);
                const bool m = (mask >> c) & 1u;
                cv[c] = m ? cadd(cv[c], pv) : pv;
                cw[c] = m ? add(cw[c], pw) : pw;
            }
            mask = 0xFFu;

            // Hermitian symmetry on the redundant x == 0 plane (FourierProject.hpp:347-372).
            if (n2 == 0) {
                float2 hv = value;
                if constexpr (OUT_C)
                    hv.y = -hv.y;
#pragma unroll
                for (int w = 0; w < 2; ++w) {
#pragma unroll
                    for (int vv = 0; vv < 2; ++vv) {
                        const float k = mul(mul(fr[w][0], fr[vv][1]), fr[0][2]);
                        const int off = ((g.r0 - (n0 + w)) * (2 * g.r1 + 1) + (g.r1 - (n1 + vv))) * g.n2;
                        acc_add<OUT_C, W>(acc, off, cmul(hv, k), mul(weight, k));
                    }
                }
            }
        }
#pragma unroll
        for (int c = 0; c < 8; ++c)
            if ((mask >> c) & 1u)
                acc_add<OUT_C, W>(acc, base + corner_offset(c, g), cv[c], cw[c]);
    }
}

// Four CTAs per SM (64 registers, 36 bytes of spills): 2.463-2.466 ms against 2.491 ms with three (77
// registers), 2.77 ms with two, 3.70 and 5.83 ms with five and six (heavy spills), 256^3 x 4096.
template<bool IN_C, bool OUT_C, bool W>
__global__ void __launch_bounds__(RASTER_THREADS, 4)
rasterize_runs_kernel(const __grid_constant__ ProjArgs a, const AccGrid g, void* __restrict__ acc) {
    const int wp = a.slice_w / 2 + 1;
    const int t = blockIdx.x * RASTER_THREADS + threadIdx.x;
    const int u = t % wp;
    const int y0 = (t / wp) * RUN;
    if (y0 >= a.slice_h)
        return;
    for (int64_t b = blockIdx.y; b < a.n_slices; b += gridDim.y)
        rasterize_run<IN_C, OUT_C, W>(a, g, acc, b, u, y0);
}

template<bool OUT_C, bool W>
__device__ __forceinline__ void acc_accumulate(const void* acc, int off, float2& v, float& w) {
    const typename AccElem<OUT_C, W>::T s = static_cast<const typename AccElem<OUT_C, W>::T*>(acc)[off];
    if constexpr (OUT_C && W) { v.x += s.x; v.y += s.y; w += s.z; }
    else if constexpr (OUT_C) { v.x += s.x; v.y += s.y; }
    else if constexpr (W) { v.x += s.x; w += s.y; }
    else { v.x += s; }
}

// Caller's grid += the accumulator cells that the reference's per-tap index test would have sent to
// each voxel: frequency2index(f) == i. Centered: f = i - n/2 only. Non-centered: f = i and f = i - n
// (frequency2index wraps negative frequencies, so a tap past the Nyquist frequency lands on the
// opposite side, as in the reference).
// Voxel i (linear index over D x H x W/2+1) of the caller's grids.
template<bool OUT_C, bool W>
__device__ __forceinline__ void finalize_padded_voxel(const ProjArgs& a, const AccGrid& g,
                                                      const void* __restrict__ acc, int64_t i) {
    const int D = a.vol_d, H = a.vol_h, WP = a.vol_w / 2 + 1;
    const bool vc = a.out_centered;
    const int ny = 2 * g.r1 + 1;
    {
        const int x = static_cast<int>(i % WP);
        const int64_t zy = i / WP;
        const int y = static_cast<int>(zy % H), z = static_cast<int>(zy / H);
        float2 v = make_float2(0.f, 0.f);
        float w = 0.f;
        if (vc) {
            acc_accumulate<OUT_C, W>(acc, ((z - D / 2 + g.r0) * ny + (y - H / 2 + g.r1)) * g.n2 + x, v, w);
        } else {
            const int fz[2] = {z, z - D}, fy[2] = {y, y - H};
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                if (fz[j] < -g.r0 || fz[j] > g.r0)
                    continue;
#pragma unroll
                for (int k = 0; k < 2; ++k) {
                    if (fy[k] < -g.r1 || fy[k] > g.r1)
                        continue;
                    acc_accumulate<OUT_C, W>(acc, ((fz[j] + g.r0) * ny + (fy[k] + g.r1)) * g.n2 + x, v, w);
                }
            }
        }
        dst_store<OUT_C>(a.out, z, y, x, cadd(dst_load<OUT_C>(a.out, z, y, x), v));
        if constexpr (W)
            store_real(a.out_w, z, y, x, add(load_real(a.out_w, z, y, x), w));
    }
}

template<bool OUT_C, bool W>
__global__ void finalize_padded_kernel(const __grid_constant__ ProjArgs a, const AccGrid g,
                                       const void* __restrict__ acc) {
    const int64_t n = static_cast<int64_t>(a.vol_d) * a.vol_h * (a.vol_w / 2 + 1);
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        finalize_padded_voxel<OUT_C, W>(a, g, acc, i);
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
