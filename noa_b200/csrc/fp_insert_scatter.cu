// Slice-major scatter form of insert_central_slices_3d (windowed sinc), nb_insert_central_slices_3d_scatter.
//
// The gather form (fp_insert.cu) sums, for every voxel, the terms of the slices whose slab
// |fz| <= fftfreq_blackman contains it (FourierInsertInterpolate, FourierProject.hpp:478-519). This form
// enumerates the same (voxel, slice) pairs from the slice side: slice i's slab is thin along the axis
// where its normal n_i (row 0 of the inverse rotation) has the largest component per voxel, so a thread
// owns one column of voxels along that axis, computes the k range the slab can cover there (widened
// by one voxel; the exact test below decides), and for each voxel of it evaluates the term exactly as
// the gather form does — same rounded coordinates, cutoff, window and 2-D interpolation — and adds it
// with one reduction (value and weight interleaved) into a dense accumulator. A finalize pass applies
// the output conversion (|z|^2 for complex -> real, to the sum, as the reference does) and adds the
// accumulator into the caller's grids. Every term is the gather form's; only the order of the sum over
// slices differs (float atomics).
//
// Not used with an Ewald-sphere curvature (the slab is curved) or when the accumulator cannot be
// allocated: both run the gather form.
#include "fp_args.cuh"
#include "fp_pool.cuh"

#include <algorithm>

namespace nb {
namespace {

constexpr int SCATTER_THREADS = 256;

template<bool IN_C, bool W> struct AccT;
template<> struct AccT<true, true> { using T = float4; };   // re, im, weight, -
template<> struct AccT<true, false> { using T = float2; };  // re, im
template<> struct AccT<false, true> { using T = float2; };  // value, weight
template<> struct AccT<false, false> { using T = float; };

template<bool IN_C, bool W>
__device__ __forceinline__ void acc_red(void* acc, int off, float2 v, float w) {
    auto* p = static_cast<typename AccT<IN_C, W>::T*>(acc) + off;
    if constexpr (IN_C && W)
        atomicAdd(p, make_float4(v.x, v.y, w, 0.f));
    else if constexpr (IN_C)
        atomicAdd(p, v);
    else if constexpr (W)
        atomicAdd(p, make_float2(v.x, w));
    else
        atomicAdd(p, v.x);
}

// Six CTAs per SM for the LINEAR and NEAREST instantiations (39 registers, no spills): 512^3 x 20,000
// slices, 378.6 -> 364.2-365.1 ms on one box (1000 slices: 19.32 -> 18.79-18.82 ms). The wider windows
// keep the compiler's choice.
template<int I>
constexpr int scatter_min_ctas() { return I == I_LINEAR || I == I_NEAREST ? 6 : 1; }

template<int I, bool IN_C, bool W>
__global__ void __launch_bounds__(SCATTER_THREADS, scatter_min_ctas<I>())
insert_scatter_kernel(const __grid_constant__ ProjArgs a, void* __restrict__ acc) {
    const int D = a.vol_d, H = a.vol_h, WP = a.vol_w / 2 + 1;
    const bool vc = a.out_centered;
    const Spectrum2 sp{a.slice_h, a.slice_w, a.in_centered, a.in_slice_narrow != 0};
    const bool has_in_w = a.in_w.present;
    // Frequency ranges: z in [-D/2, (D-1)/2], y in [-H/2, (H-1)/2], x in [0, W/2].
    auto lo_of = [&](int axis) { return axis == 0 ? -D / 2 : axis == 1 ? -H / 2 : 0; };
    auto hi_of = [&](int axis) { return axis == 0 ? (D - 1) / 2 : axis == 1 ? (H - 1) / 2 : WP - 1; };
    auto pick = [](int axis, float v0, float v1, float v2) { return axis == 0 ? v0 : axis == 1 ? v1 : v2; };
    const int col = blockIdx.x * SCATTER_THREADS + threadIdx.x;

    for (int64_t i = blockIdx.y; i < a.n_slices; i += gridDim.y) {
        const float3 n = rotation_row0(a.rot, i);
        const float c0 = n.x / a.target0, c1 = n.y / a.target1, c2 = n.z / a.target2;  // slab per index step
        const int ax = fabsf(c0) >= fabsf(c1) ? (fabsf(c0) >= fabsf(c2) ? 0 : 2) : (fabsf(c1) >= fabsf(c2) ? 1 : 2);
        const int p = ax == 0 ? 1 : 0, q = ax == 2 ? 1 : 2;   // the column's axes, q fastest
        const int ep = hi_of(p) - lo_of(p) + 1, eq = hi_of(q) - lo_of(q) + 1;
        if (col >= ep * eq)
            continue;
        const int kp = lo_of(p) + col / eq, kq = lo_of(q) + col % eq;
        const float fp = div(static_cast<float>(kp), pick(p, a.target0, a.target1, a.target2));
        const float fq = div(static_cast<float>(kq), pick(q, a.target0, a.target1, a.target2));
        if (fp * fp + fq * fq > a.cutoff_sqd * 1.0001f)
            continue;  // every voxel of the column is outside the cutoff
        int k_lo = lo_of(ax), k_hi = hi_of(ax);
        const float ca = pick(ax, c0, c1, c2);
        if (fabsf(ca) > 1e-30f) {
            const float s = pick(p, n.x, n.y, n.z) * fp + pick(q, n.x, n.y, n.z) * fq;
            const float t0 = (-a.fb - s) / ca, t1 = (a.fb - s) / ca;
            const float r0 = floorf(fminf(t0, t1)) - 1.f, r1 = ceilf(fmaxf(t0, t1)) + 1.f;
            // clamped in float first: the range stays within the axis whatever r0, r1 are (NaN included)
            k_lo = static_cast<int>(fmaxf(r0, static_cast<float>(k_lo)));
            k_hi = static_cast<int>(fminf(r1, static_cast<float>(k_hi)));
        }
        for (int ka = k_lo; ka <= k_hi; ++ka) {
            const int kz = ax == 0 ? ka : kp;
            const int ky = ax == 0 ? kp : (ax == 1 ? ka : kq);
            const int kx = ax == 2 ? ka : kq;
            // The gather form's term for voxel (kz, ky, kx) and slice i (fp_insert.cu,
            // FourierProject.hpp:479-518).
            const float fz = div(static_cast<float>(kz), a.target0);
            const float fy = div(static_cast<float>(ky), a.target1);
            const float fx = div(static_cast<float>(kx), a.target2);
            if (dot3(fz, fy, fx, fz, fy, fx) > a.cutoff_sqd)
                continue;
            float f0, f1;
            const float zz = grid2slice(fz, fy, fx, a.scale, a.rot, i, a.ews, f0, f1);
            if (!(fabsf(zz) <= a.fb))
                continue;
            const float window = windowed_sinc_fast(zz, a.pfs, a.ifs, a.pfb);
            const float q0 = mul(f0, a.f_slice0), q1 = mul(f1, a.f_slice1);
            const float2 v = cmul(interp_spectrum_2d<I, IN_C>(a.in, sp, i, q0, q1), window);
            float w = 0.f;
            if constexpr (W)
                w = has_in_w ? mul(interp_spectrum_2d<I, false>(a.in_w, sp, i, q0, q1).x, window) : window;
            const int off = (frequency2index(vc, kz, D) * H + frequency2index(vc, ky, H)) * WP + kx;
            acc_red<IN_C, W>(acc, off, v, w);
        }
    }
}

// Caller's grids += the accumulator (dense, the caller's index order), converted to the output type.
template<bool IN_C, bool OUT_C, bool W>
__global__ void scatter_finalize_kernel(const __grid_constant__ ProjArgs a, const void* __restrict__ acc) {
    using T = typename AccT<IN_C, W>::T;
    const int D = a.vol_d, H = a.vol_h, WP = a.vol_w / 2 + 1;
    const int64_t n = static_cast<int64_t>(D) * H * WP;
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int x = static_cast<int>(i % WP);
        const int64_t zy = i / WP;
        const int y = static_cast<int>(zy % H), z = static_cast<int>(zy / H);
        const T s = static_cast<const T*>(acc)[i];
        float2 v;
        float w = 0.f;
        if constexpr (IN_C && W) { v = make_float2(s.x, s.y); w = s.z; }
        else if constexpr (IN_C) { v = s; }
        else if constexpr (W) { v = make_float2(s.x, 0.f); w = s.y; }
        else { v = make_float2(s, 0.f); }
        const float2 o = to_output<IN_C, OUT_C>(v);
        dst_store<OUT_C>(a.out, z, y, x, cadd(dst_load<OUT_C>(a.out, z, y, x), o));
        if constexpr (W)
            store_real(a.out_w, z, y, x, add(load_real(a.out_w, z, y, x), w));
    }
}

template<int I, bool IN_C, bool OUT_C, bool W>
cudaError_t launch_typed(const ProjArgs& a, cudaStream_t stream, bool& done) {
    done = false;
    using T = typename AccT<IN_C, W>::T;
    const int64_t D = a.vol_d, H = a.vol_h, WP = a.vol_w / 2 + 1;
    const int64_t vox = D * H * WP;
    const size_t bytes = static_cast<size_t>(vox) * sizeof(T);
    void* acc = scratch_alloc(bytes, stream);
    if (!acc)
        return cudaSuccess;
    cudaError_t err = cudaMemsetAsync(acc, 0, bytes, stream);
    if (err == cudaSuccess) {
        const int64_t cols = std::max(H * WP, std::max(D * WP, D * H));
        const dim3 grid(static_cast<unsigned>((cols + SCATTER_THREADS - 1) / SCATTER_THREADS),
                        static_cast<unsigned>(a.n_slices < 65535 ? a.n_slices : 65535));
        insert_scatter_kernel<I, IN_C, W><<<grid, SCATTER_THREADS, 0, stream>>>(a, acc);
        const int64_t blocks = (vox + 255) / 256;
        const int grid_f = static_cast<int>(blocks < static_cast<int64_t>(sm_count()) * 16 ? blocks : sm_count() * 16);
        scatter_finalize_kernel<IN_C, OUT_C, W><<<grid_f, 256, 0, stream>>>(a, acc);
        err = cudaGetLastError();
    }
    scratch_free(acc, stream);
    done = err == cudaSuccess;
    return err;
}

template<int I, bool IN_C, bool OUT_C>
cudaError_t launch_w(const ProjArgs& a, cudaStream_t stream, bool& done) {
    return a.out_w.present ? launch_typed<I, IN_C, OUT_C, true>(a, stream, done)
                           : launch_typed<I, IN_C, OUT_C, false>(a, stream, done);
}

template<int I>
cudaError_t launch_interp(const ProjArgs& a, cudaStream_t stream, bool& done) {
    if (a.in_cplx && a.out_cplx)
        return launch_w<I, true, true>(a, stream, done);
    if (a.in_cplx)
        return launch_w<I, true, false>(a, stream, done);
    return launch_w<I, false, false>(a, stream, done);
}

} // namespace

cudaError_t launch_insert_scatter(const ProjArgs& a, cudaStream_t stream) {
    const int64_t vox = static_cast<int64_t>(a.vol_d) * a.vol_h * (a.vol_w / 2 + 1);
    if (a.n_slices == 0 || a.ews.on || vox >= (int64_t(1) << 31))
        return launch_insert(a, stream);
    bool done = false;
    cudaError_t err;
    switch (a.interp) {
        case I_NEAREST: err = launch_interp<I_NEAREST>(a, stream, done); break;
        case I_LINEAR: err = launch_interp<I_LINEAR>(a, stream, done); break;
        case I_CUBIC: err = launch_interp<I_CUBIC>(a, stream, done); break;
        case I_BSPLINE: err = launch_interp<I_BSPLINE>(a, stream, done); break;
        case I_LANCZOS4: err = launch_interp<I_LANCZOS4>(a, stream, done); break;
        case I_LANCZOS6: err = launch_interp<I_LANCZOS6>(a, stream, done); break;
        case I_LANCZOS8: err = launch_interp<I_LANCZOS8>(a, stream, done); break;
        default: return cudaErrorInvalidValue;
    }
    if (err != cudaSuccess || done)
        return err;
    return launch_insert(a, stream);
}

} // namespace nb
