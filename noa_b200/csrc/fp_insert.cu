// insert_central_slices_3d on sm_100a: deterministic gather-form windowed-sinc insertion
// (FourierInsertInterpolate, noa/xform/FourierProject.hpp:478-519).
//
// The reference visits every slice for every voxel, an O(voxels x slices) loop. Here a CTA owns a
// 4x8x8 brick of voxels and first culls the slices: slice i can only reach a voxel of the brick if
// the plane's normal n_i (row 0 of the inverse rotation) satisfies |n_i . c| <= blackman + |n_i| rho
// (+ a rounding margin), with c the brick's centre and rho its half-diagonal, all in fftfreq units.
// The surviving slice indices are compacted into shared memory IN INCREASING ORDER, and every thread
// then sums its voxel's contributions over that list. Skipped slices contribute exactly 0 in the
// reference (they fail |fz| <= blackman), so each voxel's sum sees the same terms in the same order.
// With an Ewald-sphere curvature the normal test is not conservative, and every slice is visited.
#include "fp_args.cuh"

namespace nb {
namespace {

constexpr int BZ = 4, BY = 8, BX = 8;
constexpr int INSERT_THREADS = BZ * BY * BX;

// CTAs per SM the LINEAR and NEAREST instantiations are compiled for (32 registers, small spills): the
// kernel is issue-bound and more resident warps hide its latencies: 512^3 x 20,000 slices, 328.9 ->
// 286.2-287.1 ms on one box (1000 slices: 16.13 -> 13.50-13.64 ms; six CTAs 13.80-13.86 ms). The
// wider windows keep the compiler's choice.
template<int I>
constexpr int insert_min_ctas() { return I == I_LINEAR || I == I_NEAREST ? 8 : 1; }

template<int I, bool IN_C, bool OUT_C>
__global__ void __launch_bounds__(INSERT_THREADS, insert_min_ctas<I>())
insert_kernel(const __grid_constant__ ProjArgs a, int nbz, int nby, int nbx) {
    __shared__ int s_list[INSERT_THREADS];
    __shared__ int s_warp_count[INSERT_THREADS / 32];
    __shared__ int s_count;
    // With a Mat33 rotation and neither scaling nor Ewald curvature, the kept slices' matrices are
    // staged here (in list order) so that the voxel loop reads them from shared memory, computes the
    // distance to the plane (row 0) first and the in-plane coordinates (rows 1 and 2) only inside the
    // window: the same products and sums as grid2slice, in the same order.
    __shared__ float s_mat[9][INSERT_THREADS];
    const bool lean = a.rot.kind == 2 && a.scale.kind == 0 && !a.ews.on;

    const int D = a.vol_d, H = a.vol_h, WP = a.vol_w / 2 + 1;
    const bool vc = a.out_centered;
    const Spectrum2 sp{a.slice_h, a.slice_w, a.in_centered, a.in_slice_narrow != 0};
    const bool has_out_w = a.out_w.present;
    const bool has_in_w = a.in_w.present;
    const int tid = threadIdx.x;
    const int tx = tid % BX, ty = (tid / BX) % BY, tz = tid / (BX * BY);
    const int lane = tid & 31, warp = tid >> 5;
    const int64_t n_bricks = static_cast<int64_t>(nbz) * nby * nbx;

    for (int64_t brick = blockIdx.x; brick < n_bricks; brick += gridDim.x) {
        const int bx = static_cast<int>(brick % nbx);
        const int by = static_cast<int>((brick / nbx) % nby);
        const int bz = static_cast<int>(brick / (static_cast<int64_t>(nbx) * nby));
        const int z0 = bz * BZ, y0 = by * BY, x0 = bx * BX;
        const int z = z0 + tz, y = y0 + ty, x = x0 + tx;
        const bool valid = z < D && y < H && x < WP;

        // This voxel's frequency (FourierProject.hpp:479-484).
        const float fz = div(static_cast<float>(index2frequency(vc, z, D)), a.target0);
        const float fy = div(static_cast<float>(index2frequency(vc, y, H)), a.target1);
        const float fx = div(static_cast<float>(x), a.target2);
        const bool active = valid && dot3(fz, fy, fx, fz, fy, fx) <= a.cutoff_sqd;
        if (!__syncthreads_or(active))
            continue;

        // Brick bounding box in fftfreq (per-axis min/max over the brick's valid indices; the
        // non-centered layout wraps, so scan rather than assume monotonic).
        float lo[3], hi[3];
        {
            const int n3[3] = {D, H, WP};
            const int s3[3] = {z0, y0, x0};
            const int e3[3] = {BZ, BY, BX};
            const float t3[3] = {a.target0, a.target1, a.target2};
            for (int ax = 0; ax < 3; ++ax) {
                float mn = 3.4e38f, mx = -3.4e38f;
                for (int k = 0; k < e3[ax]; ++k) {
                    const int idx = s3[ax] + k;
                    if (idx >= n3[ax])
                        break;
                    const int f = ax == 2 ? idx : index2frequency(vc, idx, n3[ax]);
                    const float ff = static_cast<float>(f) / t3[ax];
                    mn = fminf(mn, ff);
                    mx = fmaxf(mx, ff);
                }
                lo[ax] = mn;
                hi[ax] = mx;
            }
        }
        const float c0 = 0.5f * (lo[0] + hi[0]), c1 = 0.5f * (lo[1] + hi[1]), c2 = 0.5f * (lo[2] + hi[2]);
        const float h0 = 0.5f * (hi[0] - lo[0]), h1 = 0.5f * (hi[1] - lo[1]), h2 = 0.5f * (hi[2] - lo[2]);
        const float rho = sqrtf(h0 * h0 + h1 * h1 + h2 * h2);
        const float cn = sqrtf(c0 * c0 + c1 * c1 + c2 * c2);
        const float margin = 1e-5f * (cn + rho + 1.f);
        const bool cull = !a.ews.on;

        float2 value = make_float2(0.f, 0.f);
        float weights = 0.f;

        for (int64_t chunk = 0; chunk < a.n_slices; chunk += INSERT_THREADS) {
            const int64_t i = chunk + tid;
            bool keep = false;
            if (i < a.n_slices) {
                if (cull) {
                    const float3 n = rotation_row0(a.rot, i);
                    const float nn = sqrtf(n.x * n.x + n.y * n.y + n.z * n.z);
                    const float d = fabsf(n.x * c0 + n.y * c1 + n.z * c2);
                    keep = d <= a.fb + nn * rho + margin * (1.f + nn);
                } else {
                    keep = true;
                }
            }
            // Ordered compaction of the kept slice indices.
            const unsigned ballot = __ballot_sync(0xffffffffu, keep);
            if (lane == 0)
                s_warp_count[warp] = __popc(ballot);
            __syncthreads();
            int base = 0;
            for (int w = 0; w < warp; ++w)
                base += s_warp_count[w];
            if (keep) {
                const int slot = base + __popc(ballot & ((1u << lane) - 1u));
                s_list[slot] = static_cast<int>(i - chunk);
                if (lean) {
                    const float* m = xform_ptr(a.rot, i, 12);
#pragma unroll
                    for (int e = 0; e < 9; ++e)
                        s_mat[e][slot] = m[e];
                }
            }
            if (tid == INSERT_THREADS - 1)
                s_count = base + __popc(ballot);
            __syncthreads();
            const int count = s_count;

            if (active) {
                for (int k = 0; k < count; ++k) {
                    const int64_t si = chunk + s_list[k];
                    float f0, f1, zz;
                    if (lean) {
                        zz = dot3(s_mat[0][k], s_mat[1][k], s_mat[2][k], fz, fy, fx);
                        if (!(fabsf(zz) <= a.fb))
                            continue;
                        f0 = dot3(s_mat[3][k], s_mat[4][k], s_mat[5][k], fz, fy, fx);
                        f1 = dot3(s_mat[6][k], s_mat[7][k], s_mat[8][k], fz, fy, fx);
                    } else {
                        zz = grid2slice(fz, fy, fx, a.scale, a.rot, si, a.ews, f0, f1);
                    }
                    if (fabsf(zz) <= a.fb) {
                        const float window = windowed_sinc_fast<true>(zz, a.pfs, a.ifs, a.pfb);
                        const float q0 = mul(f0, a.f_slice0), q1 = mul(f1, a.f_slice1);
                        value = cadd(value, cmul(interp_spectrum_2d<I, IN_C>(a.in, sp, si, q0, q1), window));
                        if (has_out_w) {
                            const float iw = has_in_w ?
                                mul(interp_spectrum_2d<I, false>(a.in_w, sp, si, q0, q1).x, window) : window;
                            weights = add(weights, iw);
                        }
                    }
                }
            }
            __syncthreads();
        }

        if (active) {
            const float2 o = to_output<IN_C, OUT_C>(value);
            dst_store<OUT_C>(a.out, z, y, x, cadd(dst_load<OUT_C>(a.out, z, y, x), o));
            if (has_out_w)
                store_real(a.out_w, z, y, x, add(load_real(a.out_w, z, y, x), weights));
        }
    }
}

template<int I, bool IN_C, bool OUT_C>
cudaError_t launch_typed(const ProjArgs& a, cudaStream_t stream) {
    const int WP = a.vol_w / 2 + 1;
    const int nbz = (a.vol_d + BZ - 1) / BZ, nby = (a.vol_h + BY - 1) / BY, nbx = (WP + BX - 1) / BX;
    const int64_t n = static_cast<int64_t>(nbz) * nby * nbx;
    if (n == 0)
        return cudaSuccess;
    const int64_t max_grid = static_cast<int64_t>(sm_count()) * 8 * 16;
    const int grid = static_cast<int>(n < max_grid ? n : max_grid);
    insert_kernel<I, IN_C, OUT_C><<<grid, INSERT_THREADS, 0, stream>>>(a, nbz, nby, nbx);
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

cudaError_t launch_insert(const ProjArgs& a, cudaStream_t stream) {
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
