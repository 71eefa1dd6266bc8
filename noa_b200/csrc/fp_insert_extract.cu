// insert_and_extract_central_slices_3d on sm_100a: every output pixel samples the virtual volume made
// of the input slices (FourierInsertExtract, noa/xform/FourierProject.hpp:858-977).
//
// A CTA owns 256 consecutive pixels of one output slice. The input slices are culled per CTA as in the
// gather insertion: slice i can only contribute to a pixel whose 3-D frequency g satisfies
// |n_i . g| < blackman, so with the CTA's bounding sphere (c, rho) of its pixels' frequencies the
// surviving indices are compacted, in increasing order, into shared memory. Summation order per pixel
// is therefore the reference's. The w-windowed form sums the w offsets in registers (in w order)
// rather than zero-filling and adding atomically; each offset re-samples the virtual volume at the
// z-shifted frequency.
#include "fp_args.cuh"

namespace nb {
namespace {

constexpr int IE_THREADS = 256;

__device__ __forceinline__ float3 row0(const XformView& r, int64_t i) {
    if (r.kind == 3) {
        float a0 = 1.f, a1 = 0.f, a2 = 0.f;
        float b0 = 0.f, b1 = 1.f, b2 = 0.f;
        float c0 = 0.f, c1 = 0.f, c2 = 1.f;
        rotate(r, i, a0, a1, a2);
        rotate(r, i, b0, b1, b2);
        rotate(r, i, c0, c1, c2);
        return make_float3(a0, b0, c0);
    }
    const float* m = xform_ptr(r, i, 12);
    return make_float3(m[0], m[1], m[2]);
}

template<int I, bool IN_C, bool OUT_C>
__global__ void __launch_bounds__(IE_THREADS)
insert_extract_kernel(const __grid_constant__ ProjArgs a, int tiles_per_slice, int64_t n_tiles) {
    __shared__ int s_list[IE_THREADS];
    __shared__ int s_warp_count[IE_THREADS / 32];
    __shared__ int s_count;
    __shared__ float s_box[6][IE_THREADS / 32];

    const int wp = a.slice_w / 2 + 1;
    const int plane = a.slice_h * wp;
    const Spectrum2 sp{a.in_h, a.in_w_, a.in_centered, a.in_slice_narrow != 0};
    const bool has_out_w = a.out_w.present;
    const bool has_in_w = a.in_w.present;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    for (int64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        const int64_t b = tile / tiles_per_slice;
        const int p = static_cast<int>(tile - b * tiles_per_slice) * IE_THREADS + tid;
        const bool valid = p < plane;
        const int y = valid ? p / wp : 0;
        const int u = valid ? p - y * wp : 0;
        const int v = index2frequency(a.out_centered, y, a.slice_h);
        float gz, gy, gx;
        slice2grid(div(static_cast<float>(v), a.f_slice0), div(static_cast<float>(u), a.f_slice1),
                   a.scale2, a.rot2, b, a.ews, gz, gy, gx);

        // The frequencies this pixel samples: g, plus the z offsets of the w window.
        const float wz_lo = a.wsize > 1 ? div(static_cast<float>(0 - a.wsize / 2), a.vz) : 0.f;
        const float wz_hi = a.wsize > 1 ? div(static_cast<float>(a.wsize - 1 - a.wsize / 2), a.vz) : 0.f;

        // CTA bounding box of the sampled frequencies (valid pixels only).
        float bmin[3] = {valid ? add(gz, wz_lo) : 3.4e38f, valid ? gy : 3.4e38f, valid ? gx : 3.4e38f};
        float bmax[3] = {valid ? add(gz, wz_hi) : -3.4e38f, valid ? gy : -3.4e38f, valid ? gx : -3.4e38f};
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
            for (int o = 16; o > 0; o >>= 1) {
                bmin[ax] = fminf(bmin[ax], __shfl_xor_sync(0xffffffffu, bmin[ax], o));
                bmax[ax] = fmaxf(bmax[ax], __shfl_xor_sync(0xffffffffu, bmax[ax], o));
            }
            if (lane == 0) {
                s_box[ax][warp] = bmin[ax];
                s_box[3 + ax][warp] = bmax[ax];
            }
        }
        __syncthreads();
        float lo[3], hi[3];
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
            lo[ax] = 3.4e38f;
            hi[ax] = -3.4e38f;
            for (int w = 0; w < IE_THREADS / 32; ++w) {
                lo[ax] = fminf(lo[ax], s_box[ax][w]);
                hi[ax] = fmaxf(hi[ax], s_box[3 + ax][w]);
            }
        }
        const float c0 = 0.5f * (lo[0] + hi[0]), c1 = 0.5f * (lo[1] + hi[1]), c2 = 0.5f * (lo[2] + hi[2]);
        const float h0 = 0.5f * (hi[0] - lo[0]), h1 = 0.5f * (hi[1] - lo[1]), h2 = 0.5f * (hi[2] - lo[2]);
        const float rho = sqrtf(h0 * h0 + h1 * h1 + h2 * h2);
        const float cn = sqrtf(c0 * c0 + c1 * c1 + c2 * c2);
        const float margin = 1e-5f * (cn + rho + 1.f);
        const bool cull = !a.ews.on;

        // Accumulators: one (value, weight) per w offset would be needed for the windowed form, so
        // the windowed form keeps a running windowed sum per offset instead (registers, bounded).
        const int nw = a.wsize > 1 ? a.wsize : 1;
        float2 acc = make_float2(0.f, 0.f);
        float accw = 0.f;

        // Each w offset is a separate virtual-volume sample; process them one after another so the
        // per-sample sums over input slices keep the reference's order.
        for (int w = 0; w < nw; ++w) {
            const float off = a.wsize > 1 ? div(static_cast<float>(w - a.wsize / 2), a.vz) : 0.f;
            const float sz = a.wsize > 1 ? add(gz, off) : gz;
            const bool in_cut = valid && dot3(sz, gy, gx, sz, gy, gx) <= a.cutoff_sqd;
            float2 value = make_float2(0.f, 0.f);
            float weight = 0.f;

            for (int64_t chunk = 0; chunk < a.n_in; chunk += IE_THREADS) {
                const int64_t i = chunk + tid;
                bool keep = false;
                if (i < a.n_in) {
                    if (cull) {
                        const float3 n = row0(a.rot, i);
                        const float nn = sqrtf(n.x * n.x + n.y * n.y + n.z * n.z);
                        const float d = fabsf(n.x * c0 + n.y * c1 + n.z * c2);
                        keep = d <= a.fb + nn * rho + margin * (1.f + nn);
                    } else {
                        keep = true;
                    }
                }
                const unsigned ballot = __ballot_sync(0xffffffffu, keep);
                if (lane == 0)
                    s_warp_count[warp] = __popc(ballot);
                __syncthreads();
                int base = 0;
                for (int k = 0; k < warp; ++k)
                    base += s_warp_count[k];
                if (keep)
                    s_list[base + __popc(ballot & ((1u << lane) - 1u))] = static_cast<int>(i - chunk);
                if (tid == IE_THREADS - 1)
                    s_count = base + __popc(ballot);
                __syncthreads();
                const int count = s_count;
                if (in_cut) {
                    for (int k = 0; k < count; ++k) {
                        const int64_t si = chunk + s_list[k];
                        float f0, f1;
                        const float fz = grid2slice(sz, gy, gx, a.scale, a.rot, si, a.ews, f0, f1);
                        if (fabsf(fz) < a.fb) {
                            const float ws = windowed_sinc_fast(fz, a.pfs, a.pfb);
                            const float q0 = mul(f0, a.f_in0), q1 = mul(f1, a.f_in1);
                            value = cadd(value, cmul(interp_spectrum_2d<I, IN_C>(a.in, sp, si, q0, q1), ws));
                            if (has_in_w)
                                weight = add(weight, mul(interp_spectrum_2d<I, false>(a.in_w, sp, si, q0, q1).x, ws));
                            else
                                weight = add(weight, ws);
                        }
                    }
                }
                __syncthreads();
            }

            if (a.wsize <= 1) {
                if (in_cut && a.correct_weights) {
                    const float fw = fmaxf(1.f, fabsf(weight));
                    value.x = div(value.x, fw);
                    value.y = div(value.y, fw);
                }
                acc = value;
                accw = weight;
            } else if (in_cut) {
                const float cw = windowed_sinc(off, a.efs, a.efb);
                acc = cadd(acc, cmul(to_output<IN_C, OUT_C>(value), cw));
                accw = add(accw, mul(weight, cw));
            }
        }

        if (!valid)
            continue;
        if (a.wsize <= 1) {
            const bool in_cut = dot3(gz, gy, gx, gz, gy, gx) <= a.cutoff_sqd;
            if (!in_cut) {
                if (!a.add_to_output) {
                    dst_store<OUT_C>(a.out, b, y, u, make_float2(0.f, 0.f));
                    if (has_out_w)
                        store_real(a.out_w, b, y, u, 0.f);
                }
                continue;
            }
            const float2 o = to_output<IN_C, OUT_C>(acc);
            if (a.add_to_output)
                dst_store<OUT_C>(a.out, b, y, u, cadd(dst_load<OUT_C>(a.out, b, y, u), o));
            else
                dst_store<OUT_C>(a.out, b, y, u, o);
            if (has_out_w) {
                if (a.add_to_output)
                    store_real(a.out_w, b, y, u, add(load_real(a.out_w, b, y, u), accw));
                else
                    store_real(a.out_w, b, y, u, accw);
            }
        } else {
            // Windowed form: the reference zero-fills (unless add_to_output) then adds every offset.
            float2 o = acc;
            float ow = accw;
            if (a.add_to_output) {
                o = cadd(dst_load<OUT_C>(a.out, b, y, u), acc);
                if (has_out_w)
                    ow = add(load_real(a.out_w, b, y, u), accw);
            }
            dst_store<OUT_C>(a.out, b, y, u, o);
            if (has_out_w)
                store_real(a.out_w, b, y, u, ow);
        }
    }
}

template<int I, bool IN_C, bool OUT_C>
cudaError_t launch_typed(const ProjArgs& a, cudaStream_t stream) {
    const int wp = a.slice_w / 2 + 1;
    const int plane = a.slice_h * wp;
    const int tiles_per_slice = (plane + IE_THREADS - 1) / IE_THREADS;
    const int64_t n_tiles = static_cast<int64_t>(tiles_per_slice) * a.n_slices;
    if (n_tiles == 0)
        return cudaSuccess;
    const int64_t max_grid = static_cast<int64_t>(sm_count()) * 8 * 16;
    const int grid = static_cast<int>(n_tiles < max_grid ? n_tiles : max_grid);
    insert_extract_kernel<I, IN_C, OUT_C><<<grid, IE_THREADS, 0, stream>>>(a, tiles_per_slice, n_tiles);
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

cudaError_t launch_insert_extract(const ProjArgs& a, cudaStream_t stream) {
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
