// nb_rasterize_batch_launch: many rasterize_central_slices_3d calls (FourierProject.hpp:1653-1692), each
// into its own value and weight grids, as one launch of each kernel instead of one set per call.
//
// Every request gets the per-call path's padded, centered accumulator (fp_rasterize_kernels.cuh), all
// of them carved from ONE stream-ordered allocation and zeroed by one memset. The scatter kernel's CTAs
// are laid out request after request (request i owns the CTAs [begin_i, begin_i + tiles_i x slices_i));
// a CTA finds its request from a table of CTA offsets, stages that request's descriptor in shared
// memory and runs the per-call kernel's run body on it. The finalize kernel does the same over the
// requests' voxels. Per request, the terms and reductions are those of nb_rasterize_central_slices_3d;
// only the atomic summation order may differ.
#include "fp_args.cuh"
#include "fp_pool.cuh"
#include "fp_rasterize_kernels.cuh"
#include "noa_b200/batch.h"

#include <algorithm>
#include <cstdio>
#include <vector>

namespace nb {
namespace {

using namespace raster;

constexpr int FINAL_PER_THREAD = 8;

struct RasterReq {
    ProjArgs a;
    AccGrid g;
    void* acc;
    int64_t cta_begin;     // first scatter CTA of this request
    int64_t fin_begin;     // first finalize CTA of this request
    int tiles;             // scatter CTAs per slice
    int pad;
};

// Index of the request whose range [begin, next begin) holds `cta` (begins are increasing).
template<bool FIN>
__device__ __forceinline__ int find_request(const RasterReq* __restrict__ reqs, int n, int64_t cta) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        const int64_t b = FIN ? reqs[mid].fin_begin : reqs[mid].cta_begin;
        if (b <= cta)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// Copies request r's descriptor into shared memory (all threads take part).
__device__ __forceinline__ void stage(const RasterReq* __restrict__ reqs, int r, RasterReq& dst) {
    static_assert(sizeof(RasterReq) % 4 == 0, "staged as 32-bit words");
    const unsigned* src = reinterpret_cast<const unsigned*>(reqs + r);
    unsigned* out = reinterpret_cast<unsigned*>(&dst);
    for (int i = threadIdx.x; i < static_cast<int>(sizeof(RasterReq) / 4); i += blockDim.x)
        out[i] = src[i];
}

template<bool IN_C, bool OUT_C, bool W>
__global__ void __launch_bounds__(RASTER_THREADS, 3)
rasterize_batch_kernel(const RasterReq* __restrict__ reqs, int n) {
    __shared__ __align__(16) RasterReq req;
    __shared__ int r_shared;
    const int64_t cta = blockIdx.x;
    if (threadIdx.x == 0)
        r_shared = find_request<false>(reqs, n, cta);
    __syncthreads();
    stage(reqs, r_shared, req);
    __syncthreads();
    const int64_t local = cta - req.cta_begin;
    const int64_t b = local / req.tiles;
    const int tile = static_cast<int>(local - b * req.tiles);
    const int wp = req.a.slice_w / 2 + 1;
    const int t = tile * RASTER_THREADS + threadIdx.x;
    const int u = t % wp;
    const int y0 = (t / wp) * RUN;
    if (y0 >= req.a.slice_h)
        return;
    rasterize_run<IN_C, OUT_C, W>(req.a, req.g, req.acc, b, u, y0);
}

template<bool OUT_C, bool W>
__global__ void __launch_bounds__(RASTER_THREADS)
finalize_batch_kernel(const RasterReq* __restrict__ reqs, int n) {
    __shared__ __align__(16) RasterReq req;
    __shared__ int r_shared;
    const int64_t cta = blockIdx.x;
    if (threadIdx.x == 0)
        r_shared = find_request<true>(reqs, n, cta);
    __syncthreads();
    stage(reqs, r_shared, req);
    __syncthreads();
    const int64_t vox = static_cast<int64_t>(req.a.vol_d) * req.a.vol_h * (req.a.vol_w / 2 + 1);
    const int64_t first = (cta - req.fin_begin) * RASTER_THREADS * FINAL_PER_THREAD + threadIdx.x;
    for (int k = 0; k < FINAL_PER_THREAD; ++k) {
        const int64_t i = first + static_cast<int64_t>(k) * RASTER_THREADS;
        if (i >= vox)
            break;
        finalize_padded_voxel<OUT_C, W>(req.a, req.g, req.acc, i);
    }
}

size_t acc_element(bool out_c, bool w) {
    return out_c ? (w ? sizeof(float4) : sizeof(float2)) : (w ? sizeof(float2) : sizeof(float));
}

// Byte range [lo, hi) of an output view over a D x H x (W/2+1) grid.
void out_range(const DstView& d, const ProjArgs& a, size_t esize, uintptr_t& lo, uintptr_t& hi) {
    const int64_t ext[3] = {a.vol_d - 1, a.vol_h - 1, a.vol_w / 2};
    const int64_t st[3] = {d.s0, d.s1, d.s2};
    int64_t lo_e = 0, hi_e = 0;
    for (int i = 0; i < 3; ++i) {
        const int64_t e = ext[i] * st[i];
        if (e < 0)
            lo_e += e;
        else
            hi_e += e;
    }
    lo = reinterpret_cast<uintptr_t>(d.data) + static_cast<uintptr_t>(lo_e * static_cast<int64_t>(esize));
    hi = reinterpret_cast<uintptr_t>(d.data) + static_cast<uintptr_t>((hi_e + 1) * static_cast<int64_t>(esize));
}

template<bool IN_C, bool OUT_C, bool W>
cudaError_t launch_all(const RasterReq* d_reqs, int n, int64_t ctas, int64_t fctas, cudaStream_t s) {
    rasterize_batch_kernel<IN_C, OUT_C, W><<<static_cast<unsigned>(ctas), RASTER_THREADS, 0, s>>>(d_reqs, n);
    finalize_batch_kernel<OUT_C, W><<<static_cast<unsigned>(fctas), RASTER_THREADS, 0, s>>>(d_reqs, n);
    return cudaGetLastError();
}

} // namespace
} // namespace nb

using namespace nb;

extern "C" int nb_rasterize_batch_launch(int32_t remap, const nb_rasterize_request* requests, int64_t n_requests,
                                         const nb_options* options, void* stream) {
    if (!requests || n_requests <= 0)
        return report_error(NB_ERROR_INVALID, "a batch needs at least one request");
    if (n_requests > (int64_t(1) << 20))
        return report_error(NB_ERROR_INVALID, "too many requests");
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    std::vector<RasterReq> reqs(static_cast<size_t>(n_requests));
    bool in_c = false, out_c = false, w = false;
    size_t acc_bytes = 0;
    int64_t ctas = 0, fctas = 0;
    std::vector<size_t> acc_off(reqs.size());
    for (size_t i = 0; i < reqs.size(); ++i) {
        const nb_rasterize_request& q = requests[i];
        RasterReq& r = reqs[i];
        r = RasterReq{};
        const int st = prepare_rasterize(remap, q.slice, q.slice_weight, q.slice_shape, q.volume, q.volume_weight,
                                         q.volume_shape, q.inv_scaling, q.fwd_rotation, options, r.a);
        if (st != NB_OK)
            return st;
        const bool ic = r.a.in_cplx, oc = r.a.out_cplx, ww = r.a.out_w.present;
        if (i == 0) {
            in_c = ic;
            out_c = oc;
            w = ww;
        } else if (ic != in_c || oc != out_c || ww != w) {
            return report_error(NB_ERROR_INVALID,
                                "all requests of a batch must have the same value types and all or none output weights");
        }
        r.g = make_acc_grid(r.a);
        if (r.g.elements <= 0)
            return report_error(NB_ERROR_UNSUPPORTED,
                                "a request's grid does not fit the batched accumulator; use nb_rasterize_central_slices_3d");
        // A request without slices adds nothing and leaves its grids untouched, as the per-call path:
        // it gets no accumulator and empty ranges of CTAs (the search then never selects it).
        const bool work = r.a.n_slices > 0;
        acc_off[i] = acc_bytes;
        if (work)
            acc_bytes += (static_cast<size_t>(r.g.elements) * acc_element(out_c, w) + 255) / 256 * 256;
        const int64_t wp = r.a.slice_w / 2 + 1;
        const int64_t threads = wp * ((r.a.slice_h + RUN - 1) / RUN);
        r.tiles = static_cast<int>((threads + RASTER_THREADS - 1) / RASTER_THREADS);
        r.cta_begin = ctas;
        ctas += work ? static_cast<int64_t>(r.tiles) * r.a.n_slices : 0;
        const int64_t vox = static_cast<int64_t>(r.a.vol_d) * r.a.vol_h * (r.a.vol_w / 2 + 1);
        r.fin_begin = fctas;
        fctas += work ? (vox + RASTER_THREADS * FINAL_PER_THREAD - 1) / (RASTER_THREADS * FINAL_PER_THREAD) : 0;
    }
    // The finalize pass adds into each request's grids without atomics: their memory must not overlap.
    {
        std::vector<std::pair<uintptr_t, uintptr_t>> ranges;
        for (const RasterReq& r : reqs) {
            uintptr_t lo, hi;
            out_range(r.a.out, r.a, out_c ? sizeof(float2) : sizeof(float), lo, hi);
            ranges.push_back({lo, hi});
            if (w) {
                out_range(r.a.out_w, r.a, sizeof(float), lo, hi);
                ranges.push_back({lo, hi});
            }
        }
        std::sort(ranges.begin(), ranges.end());
        for (size_t i = 1; i < ranges.size(); ++i)
            if (ranges[i].first < ranges[i - 1].second)
                return report_error(NB_ERROR_INVALID, "the requests of a batch must write disjoint grids");
    }
    if (ctas >= (int64_t(1) << 31) || fctas >= (int64_t(1) << 31))
        return report_error(NB_ERROR_INVALID, "batch too large for one launch");
    bool empty = true;
    for (const RasterReq& r : reqs)
        empty = empty && r.a.n_slices == 0;
    if (empty)
        return finish_launch(cudaSuccess);

    const size_t desc_bytes = (reqs.size() * sizeof(RasterReq) + 255) / 256 * 256;
    char* scratch = static_cast<char*>(scratch_alloc(desc_bytes + acc_bytes, s));
    if (!scratch)
        return report_error(NB_ERROR_OOM, "cannot allocate the batch's accumulators");
    for (size_t i = 0; i < reqs.size(); ++i)
        reqs[i].acc = scratch + desc_bytes + acc_off[i];
    auto* d_reqs = reinterpret_cast<RasterReq*>(scratch);
    // The host vector goes when this returns: upload_async copies it in a form a capture keeps.
    cudaError_t err = upload_async(d_reqs, reqs.data(), reqs.size() * sizeof(RasterReq), s);
    if (err == cudaSuccess)
        err = cudaMemsetAsync(scratch + desc_bytes, 0, acc_bytes, s);
    if (err == cudaSuccess) {
        const int n = static_cast<int>(reqs.size());
        if (in_c && out_c)
            err = w ? launch_all<true, true, true>(d_reqs, n, ctas, fctas, s) : launch_all<true, true, false>(d_reqs, n, ctas, fctas, s);
        else if (in_c)
            err = w ? launch_all<true, false, true>(d_reqs, n, ctas, fctas, s) : launch_all<true, false, false>(d_reqs, n, ctas, fctas, s);
        else
            err = w ? launch_all<false, false, true>(d_reqs, n, ctas, fctas, s) : launch_all<false, false, false>(d_reqs, n, ctas, fctas, s);
    }
    scratch_free(scratch, s);
    return finish_launch(err);
}
