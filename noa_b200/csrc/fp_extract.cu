// extract_central_slices_3d on sm_100a: one thread per output pixel, 3-D spectrum interpolation of
// the volume (FourierExtract, noa/xform/FourierProject.hpp:632-694).
//
// Work decomposition: a CTA owns a 16x16 tile of one slice (blockIdx.x = tile, blockIdx.y strides
// over slices), each warp a 4x8 sub-tile, so the rotation is uniform per CTA and a warp's taps fall on
// a compact patch of the volume; taps are read through the non-coherent L1 path. Volume offsets are
// 32-bit whenever the volume fits, and the LINEAR path resolves bounds and frequency2index once per
// axis rather than once per tap. LINEAR extraction of a complex volume with enough pixels first makes
// a pair copy of the volume (fp_pairs.cuh) and reads each trilinear cell as four 16-byte loads, four
// pixels per thread (extract_pairs_kernel; extract_pairs_w_kernel with the w-window).
//
// The w-windowed form (wsize > 1) keeps the reference's semantics — outputs are the windowed sum over
// the w offsets of the z-shifted samples — but sums in registers, in w order, instead of zeroing the
// outputs and adding atomically, so it is deterministic and needs no extra pass.
#include "fp_args.cuh"
#include "fp_pairs.cuh"
#include "fp_pool.cuh"

namespace nb {
namespace {

constexpr int TY = 16, TX = 16, EXTRACT_THREADS = TY * TX;

// ---------------------------------------------------------------------------------------------------
// Fast LINEAR path over a pair copy of the volume (fp_pairs.cuh). Each thread interpolates PAIR_PPT
// pixels (rows y, y+16, ...) of one column, keeping more loads in flight.
// ---------------------------------------------------------------------------------------------------
constexpr int PAIR_PPT = 4;

// The w-window's values depend on the offset alone, so a CTA tabulates them once (the same expression
// as the per-sample one, hence the same bits) instead of evaluating the window for every pixel and
// offset. Windows of more than W_TABLE offsets evaluate the rest per sample.
constexpr int W_TABLE = 64;

// Called by every thread of the CTA before any of them returns (it synchronizes when wsize > 1).
__device__ __forceinline__ void fill_w_table(const ProjArgs& a, float* table) {
    if (a.wsize <= 1)
        return;
    for (int w = threadIdx.x; w < a.wsize && w < W_TABLE; w += blockDim.x)
        table[w] = windowed_sinc(div(static_cast<float>(w - a.wsize / 2), a.target0), a.efs, a.efb);
    __syncthreads();
}

__device__ __forceinline__ float w_value(const ProjArgs& a, const float* table, int w, float off) {
    return w < W_TABLE ? table[w] : windowed_sinc(off, a.efs, a.efb);
}

// Idx: the type of the linear voxel index, 32-bit when the volume has fewer than 2^31 voxels (its
// divisions then cost a fifth of the 64-bit ones, which bounded the copy).
template<typename Idx>
__global__ void make_pairs(const __grid_constant__ ProjArgs a, float4* __restrict__ pairs) {
    const int D = a.vol_d, H = a.vol_h, WP = a.vol_w / 2 + 1;
    const Idx n = static_cast<Idx>(D) * H * WP;
    const float2* vol = static_cast<const float2*>(a.in.data);
    for (Idx i = blockIdx.x * static_cast<Idx>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<Idx>(gridDim.x) * blockDim.x) {
        const int x = static_cast<int>(i % static_cast<Idx>(WP));
        const Idx zy = i / static_cast<Idx>(WP);
        const int y = static_cast<int>(zy % static_cast<Idx>(H)), z = static_cast<int>(zy / static_cast<Idx>(H));
        const int64_t off = z * a.in.s0 + y * a.in.s1 + x * a.in.s2;
        const float2 v0 = vol[off];
        const float2 v1 = x + 1 < WP ? vol[off + a.in.s2] : make_float2(0.f, 0.f);
        pairs[i] = make_float4(v0.x, v0.y, v1.x, v1.y);
    }
}

template<bool OUT_C>
__global__ void __launch_bounds__(EXTRACT_THREADS)
extract_pairs_kernel(const __grid_constant__ ProjArgs a, const float4* __restrict__ pairs, int ntx) {
    const int wp = a.slice_w / 2 + 1;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int y0 = (blockIdx.x / ntx) * (TY * PAIR_PPT) + (warp >> 1) * 4 + (lane >> 3);
    const int u = (blockIdx.x % ntx) * TX + (warp & 1) * 8 + (lane & 7);
    if (u >= wp)
        return;
    const Spectrum3 sp{a.vol_d, a.vol_h, a.vol_w, a.in_centered};
    const int WP = a.vol_w / 2 + 1;
    const int sz = a.vol_h * WP, sy = WP;
    const bool has_out_w = a.out_w.present;
    const float f1 = div(static_cast<float>(u), a.f_slice1);
    float f0[PAIR_PPT];
#pragma unroll
    for (int r = 0; r < PAIR_PPT; ++r)
        f0[r] = div(static_cast<float>(index2frequency(a.out_centered, y0 + r * TY, a.slice_h)), a.f_slice0);

    for (int64_t b = blockIdx.y; b < a.n_slices; b += gridDim.y) {
        float2 value[PAIR_PPT];
        bool inside[PAIR_PPT];
        const float* m = nullptr;
        const bool lean = lean_rotation(a, b, m);
#pragma unroll
        for (int r = 0; r < PAIR_PPT; ++r) {
            float fz, fy, fx;
            if (lean)
                slice2grid_lean(m, f0[r], f1, fz, fy, fx);
            else
                slice2grid(f0[r], f1, a.scale, a.rot, b, a.ews, fz, fy, fx);
            value[r] = make_float2(0.f, 0.f);
            inside[r] = y0 + r * TY < a.slice_h && dot3(fz, fy, fx, fz, fy, fx) <= a.cutoff_sqd;
            if (inside[r])
                value[r] = to_output<true, OUT_C>(interp_linear_pairs(
                    pairs, sz, sy, sp, mul(fz, a.target0), mul(fy, a.target1), mul(fx, a.target2)));
        }
#pragma unroll
        for (int r = 0; r < PAIR_PPT; ++r) {
            const int y = y0 + r * TY;
            if (y >= a.slice_h)
                continue;
            dst_store_stream<OUT_C>(a.out, b, y, u, value[r]);
            if (has_out_w)
                store_real_stream(a.out_w, b, y, u, inside[r] ? 1.f : 0.f);
        }
    }
}

// The w-windowed form over the pair copy: per pixel, the windowed sum over the w offsets of the
// z-shifted samples, each read as 4 pair loads — extract_kernel's w loop step for step (same offsets,
// cutoff tests, window values and sum order), so the results are bit-identical to it.
template<bool OUT_C>
__global__ void __launch_bounds__(EXTRACT_THREADS)
extract_pairs_w_kernel(const __grid_constant__ ProjArgs a, const float4* __restrict__ pairs, int ntx) {
    const int wp = a.slice_w / 2 + 1;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int y0 = (blockIdx.x / ntx) * (TY * PAIR_PPT) + (warp >> 1) * 4 + (lane >> 3);
    const int u = (blockIdx.x % ntx) * TX + (warp & 1) * 8 + (lane & 7);
    __shared__ float s_w[W_TABLE];
    fill_w_table(a, s_w);
    if (u >= wp)
        return;
    const Spectrum3 sp{a.vol_d, a.vol_h, a.vol_w, a.in_centered};
    const int WP = a.vol_w / 2 + 1;
    const int sz = a.vol_h * WP, sy = WP;
    const bool has_out_w = a.out_w.present;
    const float f1 = div(static_cast<float>(u), a.f_slice1);

    for (int64_t b = blockIdx.y; b < a.n_slices; b += gridDim.y) {
#pragma unroll 1
        for (int r = 0; r < PAIR_PPT; ++r) {
            const int y = y0 + r * TY;
            if (y >= a.slice_h)
                break;
            const float f0 = div(static_cast<float>(index2frequency(a.out_centered, y, a.slice_h)), a.f_slice0);
            float fz, fy, fx;
            slice2grid(f0, f1, a.scale, a.rot, b, a.ews, fz, fy, fx);
            float2 value = make_float2(0.f, 0.f);
            float weight = 0.f;
            for (int w = 0; w < a.wsize; ++w) {
                const float off = div(static_cast<float>(w - a.wsize / 2), a.target0);
                const float gz = add(fz, off);
                if (dot3(gz, fy, fx, gz, fy, fx) > a.cutoff_sqd)
                    continue;
                const float cw = w_value(a, s_w, w, off);
                const float2 iv = to_output<true, OUT_C>(interp_linear_pairs(
                    pairs, sz, sy, sp, mul(gz, a.target0), mul(fy, a.target1), mul(fx, a.target2)));
                value = cadd(value, cmul(iv, cw));
                if (has_out_w)
                    weight = add(weight, mul(1.f, cw));
            }
            dst_store_stream<OUT_C>(a.out, b, y, u, value);
            if (has_out_w)
                store_real_stream(a.out_w, b, y, u, weight);
        }
    }
}

// Whether the per-call pair path applies: the pair copy is readable (pairs_apply) and there are enough
// pixels to amortise making it.
bool use_pairs(const ProjArgs& a) {
    const int64_t vox = static_cast<int64_t>(a.vol_d) * a.vol_h * (a.vol_w / 2 + 1);
    const int64_t pix = a.n_slices * a.slice_h * static_cast<int64_t>(a.slice_w / 2 + 1);
    ProjArgs plain = a;
    plain.wsize = 1;  // the w-windowed form reads the pair copy too (extract_pairs_w_kernel)
    return pairs_apply(plain) && pix >= 2 * vox;
}

cudaError_t launch_pairs(const ProjArgs& a, cudaStream_t stream, bool& done) {
    done = false;
    const int64_t wp_vol = a.vol_w / 2 + 1;
    const int64_t vox = static_cast<int64_t>(a.vol_d) * a.vol_h * wp_vol;
    float4* pairs = static_cast<float4*>(scratch_alloc(static_cast<size_t>(vox) * sizeof(float4), stream));
    if (!pairs)
        return cudaSuccess; // no scratch: the caller takes the generic path
    launch_make_pairs(a, pairs, stream);
    const cudaError_t err = launch_extract_pairs(a, pairs, stream);
    scratch_free(pairs, stream);
    done = err == cudaSuccess;
    return err;
}

template<int I, bool IN_C, bool OUT_C, typename Idx>
__global__ void __launch_bounds__(EXTRACT_THREADS)
extract_kernel(const __grid_constant__ ProjArgs a, int ntx) {
    const int wp = a.slice_w / 2 + 1;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int y = (blockIdx.x / ntx) * TY + (warp >> 1) * 4 + (lane >> 3);
    const int u = (blockIdx.x % ntx) * TX + (warp & 1) * 8 + (lane & 7);
    __shared__ float s_w[W_TABLE];
    fill_w_table(a, s_w);
    if (u >= wp || y >= a.slice_h)
        return;
    const Spectrum3 sp{a.vol_d, a.vol_h, a.vol_w, a.in_centered};
    const View3<Idx> vol{a.in.data, static_cast<Idx>(a.in.s0), static_cast<Idx>(a.in.s1), static_cast<Idx>(a.in.s2)};
    const View3<Idx> volw{a.in_w.data, static_cast<Idx>(a.in_w.s0), static_cast<Idx>(a.in_w.s1),
                          static_cast<Idx>(a.in_w.s2)};
    const bool has_out_w = a.out_w.present;
    const bool has_in_w = a.in_w.present;
    const int v = index2frequency(a.out_centered, y, a.slice_h);
    const float f0 = div(static_cast<float>(v), a.f_slice0);
    const float f1 = div(static_cast<float>(u), a.f_slice1);

    for (int64_t b = blockIdx.y; b < a.n_slices; b += gridDim.y) {
        float fz, fy, fx;
        slice2grid(f0, f1, a.scale, a.rot, b, a.ews, fz, fy, fx);

        float2 value = make_float2(0.f, 0.f);
        float weight = 0.f;
        if (a.wsize <= 1) {
            if (dot3(fz, fy, fx, fz, fy, fx) <= a.cutoff_sqd) {
                const float q0 = mul(fz, a.target0), q1 = mul(fy, a.target1), q2 = mul(fx, a.target2);
                value = to_output<IN_C, OUT_C>(interp_3d<I, IN_C>(vol, sp, q0, q1, q2));
                if (has_out_w)
                    weight = has_in_w ? interp_3d<I, false>(volw, sp, q0, q1, q2).x : 1.f;
            }
        } else {
            for (int w = 0; w < a.wsize; ++w) {
                const float off = div(static_cast<float>(w - a.wsize / 2), a.target0);
                const float gz = add(fz, off);
                if (dot3(gz, fy, fx, gz, fy, fx) > a.cutoff_sqd)
                    continue;
                const float q0 = mul(gz, a.target0), q1 = mul(fy, a.target1), q2 = mul(fx, a.target2);
                const float cw = w_value(a, s_w, w, off);
                const float2 iv = to_output<IN_C, OUT_C>(interp_3d<I, IN_C>(vol, sp, q0, q1, q2));
                value = cadd(value, cmul(iv, cw));
                if (has_out_w) {
                    const float iw = has_in_w ? interp_3d<I, false>(volw, sp, q0, q1, q2).x : 1.f;
                    weight = add(weight, mul(iw, cw));
                }
            }
        }
        dst_store_stream<OUT_C>(a.out, b, y, u, value);
        if (has_out_w)
            store_real_stream(a.out_w, b, y, u, weight);
    }
}

template<int I, bool IN_C, bool OUT_C>
cudaError_t launch_typed(const ProjArgs& a, cudaStream_t stream) {
    const int wp = a.slice_w / 2 + 1;
    const int ntx = (wp + TX - 1) / TX, nty = (a.slice_h + TY - 1) / TY;
    if (a.n_slices == 0)
        return cudaSuccess;
    const dim3 grid(static_cast<unsigned>(ntx * nty), static_cast<unsigned>(a.n_slices < 65535 ? a.n_slices : 65535));
    if (a.wide_in)
        extract_kernel<I, IN_C, OUT_C, int64_t><<<grid, EXTRACT_THREADS, 0, stream>>>(a, ntx);
    else
        extract_kernel<I, IN_C, OUT_C, int32_t><<<grid, EXTRACT_THREADS, 0, stream>>>(a, ntx);
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

cudaError_t launch_extract_pairs(const ProjArgs& a, const float4* pairs, cudaStream_t stream) {
    if (a.n_slices <= 0)
        return cudaSuccess;
    const int wp = a.slice_w / 2 + 1;
    const int ntx = (wp + TX - 1) / TX, nty = (a.slice_h + TY * PAIR_PPT - 1) / (TY * PAIR_PPT);
    const dim3 grid(static_cast<unsigned>(ntx * nty), static_cast<unsigned>(a.n_slices < 65535 ? a.n_slices : 65535));
    if (a.wsize > 1) {
        if (a.out_cplx)
            extract_pairs_w_kernel<true><<<grid, EXTRACT_THREADS, 0, stream>>>(a, pairs, ntx);
        else
            extract_pairs_w_kernel<false><<<grid, EXTRACT_THREADS, 0, stream>>>(a, pairs, ntx);
    } else if (a.out_cplx) {
        extract_pairs_kernel<true><<<grid, EXTRACT_THREADS, 0, stream>>>(a, pairs, ntx);
    } else {
        extract_pairs_kernel<false><<<grid, EXTRACT_THREADS, 0, stream>>>(a, pairs, ntx);
    }
    return cudaGetLastError();
}

cudaError_t launch_make_pairs(const ProjArgs& a, float4* pairs, cudaStream_t stream, const int* priority) {
    const int64_t vox = static_cast<int64_t>(a.vol_d) * a.vol_h * (a.vol_w / 2 + 1);
    const int threads = 256;
    const int64_t blocks = (vox + threads - 1) / threads;
    const int grid = static_cast<int>(blocks < static_cast<int64_t>(sm_count()) * 16 ? blocks : sm_count() * 16);
    if (grid <= 0)
        return cudaSuccess;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(static_cast<unsigned>(grid));
    cfg.blockDim = dim3(threads);
    cfg.stream = stream;
    cudaLaunchAttribute attr{};
    if (priority) {
        attr.id = cudaLaunchAttributePriority;
        attr.val.priority = *priority;
        cfg.attrs = &attr;
        cfg.numAttrs = 1;
    }
    if (vox < (int64_t(1) << 31))
        return cudaLaunchKernelEx(&cfg, make_pairs<uint32_t>, a, pairs);
    return cudaLaunchKernelEx(&cfg, make_pairs<int64_t>, a, pairs);
}

cudaError_t launch_extract(const ProjArgs& a, cudaStream_t stream) {
    if (a.n_slices > 0 && use_pairs(a)) {
        bool done = false;
        const cudaError_t err = launch_pairs(a, stream, done);
        if (err != cudaSuccess || done)
            return err;
    }
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
