// insert_and_extract_central_slices_3d on sm_100a: every output pixel samples the virtual volume made
// of the input slices (FourierInsertExtract, noa/xform/FourierProject.hpp:858-977).
//
// A CTA owns a 16x16 tile of one output slice, each warp a 4x8 sub-tile. The input slices are culled
// twice: slice i can only contribute to a pixel whose 3-D frequency g satisfies |n_i . g| < blackman,
// and without curvature g is linear in the pixel's 2-D frequency, so n_i . g over a box of pixels is an
// interval known from two dot products (patch_reaches). The slices whose interval over the CTA's box
// meets the slab are compacted, in increasing order, into shared memory, 4096 at a time, each warp
// compacting its own range of slice indices so that building the list needs no barrier; each warp then
// re-tests the whole list against its own box (one candidate per lane) and walks the survivors' ballot
// in lane order, with no barrier until the next pass.
// Summation order per pixel is therefore the reference's (increasing slice index). With an Ewald
// sphere (curved slices) nothing is culled. The w-windowed form sums the w offsets in registers (in w order)
// rather than zero-filling and adding atomically; each offset re-samples the virtual volume at the
// z-shifted frequency.
#include "fp_args.cuh"

namespace nb {
namespace {

constexpr int IE_THREADS = 256;
constexpr int IE_TILE = 16;  // 16x16 pixels per CTA; warps own 4x8 sub-tiles
constexpr int IE_LIST = 4096;                           // input slices culled per pass (16 KB of indices)
constexpr int IE_REGION = IE_LIST / (IE_THREADS / 32);  // of which each warp compacts one range

// A box of 2-D output frequencies: centre and half-extent per axis.
struct Box2 {
    float c0, h0, c1, h1;
    __device__ static Box2 of(float lo0, float hi0, float lo1, float hi1) {
        return {0.5f * (lo0 + hi0), 0.5f * (hi0 - lo0), 0.5f * (lo1 + hi1), 0.5f * (hi1 - lo1)};
    }
};

// The 3-D frequencies of an output slice's unit 2-D steps (z, y, x).
struct Patch {
    float gv0, gv1, gv2, gu0, gu1, gu2;
};

// Whether input slice i (n = row 0 of its inverse rotation, so that its fz = n . g) can reach
// |fz| < blackman at a frequency g of the box, shifted along z by `off`: over the box, n . g spans
// centre +- (|n . Gv| h0 + |n . Gu| h1). The margin covers the rounding of the exact per-pixel test.
__device__ __forceinline__ bool patch_reaches(const float3 n, const Patch& p, const Box2& box, float off, float fb) {
    const float al = n.x * p.gv0 + n.y * p.gv1 + n.z * p.gv2;
    const float be = n.x * p.gu0 + n.y * p.gu1 + n.z * p.gu2;
    const float centre = al * box.c0 + be * box.c1 + n.x * off;
    const float half = fabsf(al) * box.h0 + fabsf(be) * box.h1;
    return fabsf(centre) <= fb + half + 1e-5f * (1.f + fabsf(centre) + half);
}

// Six CTAs per SM for the LINEAR and NEAREST instantiations (40 registers, small spills; five fit
// before): 4096 -> 256 slices at 256^3, 19.75-19.87 -> 15.95-16.10 ms on two boxes. The wider windows
// keep the compiler's choice.
template<int I>
constexpr int insert_extract_min_ctas() { return I == I_LINEAR || I == I_NEAREST ? 6 : 1; }

template<int I, bool IN_C, bool OUT_C>
__global__ void __launch_bounds__(IE_THREADS, insert_extract_min_ctas<I>())
insert_extract_kernel(const __grid_constant__ ProjArgs a, int ntx, int tiles_per_slice, int64_t n_tiles) {
    __shared__ int s_list[IE_LIST];
    __shared__ int s_warp_count[IE_THREADS / 32];
    __shared__ float s_box[4][IE_THREADS / 32];

    const int wp = a.slice_w / 2 + 1;
    const Spectrum2 sp{a.in_h, a.in_w_, a.in_centered, a.in_slice_narrow != 0};
    const bool has_out_w = a.out_w.present;
    const bool has_in_w = a.in_w.present;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const bool lean = a.rot.kind == 2 && a.scale.kind == 0 && !a.ews.on;

    for (int64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        const int64_t b = tile / tiles_per_slice;
        const int t = static_cast<int>(tile - b * tiles_per_slice);
        const int ty = t / ntx, tx = t - ty * ntx;
        const int py = ty * IE_TILE + (warp >> 1) * 4 + (lane >> 3);
        const int pu = tx * IE_TILE + (warp & 1) * 8 + (lane & 7);
        const bool valid = py < a.slice_h && pu < wp;
        const int y = valid ? py : 0;
        const int u = valid ? pu : 0;
        const int v = index2frequency(a.out_centered, y, a.slice_h);
        const float pf0 = div(static_cast<float>(v), a.f_slice0), pf1 = div(static_cast<float>(u), a.f_slice1);
        float gz, gy, gx;
        slice2grid(pf0, pf1, a.scale2, a.rot2, b, a.ews, gz, gy, gx);

        // Without curvature a pixel's frequency is linear in its 2-D frequency: g = pf0 Gv + pf1 Gu.
        // Over a box of 2-D frequencies, n . g therefore spans an interval whose centre and half-width
        // follow from n . Gv and n . Gu (patch_reaches); the boxes are the warp's and the CTA's.
        Patch patch;
        slice2grid(1.f, 0.f, a.scale2, a.rot2, b, a.ews, patch.gv0, patch.gv1, patch.gv2);
        slice2grid(0.f, 1.f, a.scale2, a.rot2, b, a.ews, patch.gu0, patch.gu1, patch.gu2);
        float bmin[2] = {valid ? pf0 : 3.4e38f, valid ? pf1 : 3.4e38f};
        float bmax[2] = {valid ? pf0 : -3.4e38f, valid ? pf1 : -3.4e38f};
#pragma unroll
        for (int ax = 0; ax < 2; ++ax) {
            for (int o = 16; o > 0; o >>= 1) {
                bmin[ax] = fminf(bmin[ax], __shfl_xor_sync(0xffffffffu, bmin[ax], o));
                bmax[ax] = fmaxf(bmax[ax], __shfl_xor_sync(0xffffffffu, bmax[ax], o));
            }
            if (lane == 0) {
                s_box[ax][warp] = bmin[ax];
                s_box[2 + ax][warp] = bmax[ax];
            }
        }
        // After the butterfly every lane holds its warp's box.
        const bool warp_valid = __any_sync(0xffffffffu, valid);
        const Box2 wbox = Box2::of(bmin[0], bmax[0], bmin[1], bmax[1]);
        __syncthreads();
        float lo[2], hi[2];
#pragma unroll
        for (int ax = 0; ax < 2; ++ax) {
            lo[ax] = 3.4e38f;
            hi[ax] = -3.4e38f;
            for (int w = 0; w < IE_THREADS / 32; ++w) {
                lo[ax] = fminf(lo[ax], s_box[ax][w]);
                hi[ax] = fmaxf(hi[ax], s_box[2 + ax][w]);
            }
        }
        const Box2 cbox = Box2::of(lo[0], hi[0], lo[1], hi[1]);
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

            for (int64_t super = 0; super < a.n_in; super += IE_LIST) {
                int cnt = 0;
                for (int r = 0; r < IE_REGION; r += 32) {
                    const int64_t i = super + warp * IE_REGION + r + lane;
                    if (super + warp * IE_REGION + r >= a.n_in)
                        break;
                    const bool keep = i < a.n_in &&
                                      (!cull || patch_reaches(rotation_row0(a.rot, i), patch, cbox, off, a.fb));
                    const unsigned ballot = __ballot_sync(0xffffffffu, keep);
                    if (keep)
                        s_list[warp * IE_REGION + cnt + __popc(ballot & ((1u << lane) - 1u))] =
                            static_cast<int>(i - super);
                    cnt += __popc(ballot);
                }
                if (lane == 0)
                    s_warp_count[warp] = cnt;
                __syncthreads();
                for (int region = 0; warp_valid && region < IE_THREADS / 32; ++region) {
                    const int count = s_warp_count[region];
                    const int* list = s_list + region * IE_REGION;
                    for (int g = 0; g < count; g += 32) {
                        const int k = g + lane;
                        const bool wkeep = k < count &&
                                           (!cull || patch_reaches(rotation_row0(a.rot, super + list[k]), patch, wbox,
                                                                   off, a.fb));
                        unsigned todo = __ballot_sync(0xffffffffu, wkeep);
                        while (todo) {
                            const int j = __ffs(todo) - 1;
                            todo &= todo - 1u;
                            if (!in_cut)
                                continue;
                            const int64_t si = super + list[g + j];
                            float f0, f1, fz;
                            if (lean) {
                                // grid2slice's Mat33 rows, the distance to the plane first: the in-plane
                                // rows are only needed inside the window (same products and sums).
                                const float* m = xform_ptr(a.rot, si, 12);
                                fz = dot3(m[0], m[1], m[2], sz, gy, gx);
                                if (!(fabsf(fz) < a.fb))
                                    continue;
                                f0 = dot3(m[3], m[4], m[5], sz, gy, gx);
                                f1 = dot3(m[6], m[7], m[8], sz, gy, gx);
                            } else {
                                fz = grid2slice(sz, gy, gx, a.scale, a.rot, si, a.ews, f0, f1);
                            }
                            if (fabsf(fz) < a.fb) {
                                const float ws = windowed_sinc_fast<true>(fz, a.pfs, a.ifs, a.pfb);
                                const float q0 = mul(f0, a.f_in0), q1 = mul(f1, a.f_in1);
                                value = cadd(value, cmul(interp_spectrum_2d<I, IN_C>(a.in, sp, si, q0, q1), ws));
                                if (has_in_w)
                                    weight = add(weight,
                                                 mul(interp_spectrum_2d<I, false>(a.in_w, sp, si, q0, q1).x, ws));
                                else
                                    weight = add(weight, ws);
                            }
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
    const int ntx = (wp + IE_TILE - 1) / IE_TILE, nty = (a.slice_h + IE_TILE - 1) / IE_TILE;
    const int tiles_per_slice = ntx * nty;
    const int64_t n_tiles = static_cast<int64_t>(tiles_per_slice) * a.n_slices;
    if (n_tiles == 0)
        return cudaSuccess;
    const int64_t max_grid = static_cast<int64_t>(sm_count()) * 8 * 16;
    const int grid = static_cast<int>(n_tiles < max_grid ? n_tiles : max_grid);
    insert_extract_kernel<I, IN_C, OUT_C><<<grid, IE_THREADS, 0, stream>>>(a, ntx, tiles_per_slice, n_tiles);
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
