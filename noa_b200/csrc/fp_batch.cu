// Batched extraction: many extract_central_slices_3d calls — different volumes, box sizes and slice
// counts — executed by ONE persistent kernel, replayed as a CUDA graph; LINEAR requests read through
// pair copies with enough pixels run instead as grids of the per-call pair kernel on parallel graph
// branches (nb_extract_batch_t::direct).
//
// Work decomposition: every request is cut into (slice, tile) items, a tile being TY x TX pixels of
// one output slice (4 TY x TX for a request read through its volume's pair copy, 4 rows per thread).
// Items are numbered request after request; a device counter hands them out in chunks of
// consecutive items (atomicAdd; about 64 claims per CTA over a launch, at most 64 items per claim), so
// uneven requests balance themselves across the SMs without a per-request launch and cheap items do
// not queue on the counter. A CTA stages the descriptor of its current request in shared memory and
// crosses a barrier only when its request changes. Each item runs the per-pixel
// code of nb_extract_central_slices_3d (extract_one restates the generic kernel body for one pixel,
// extract_rows_pairs the pair-copy kernel body for 4 rows), so results are bit-identical to the
// per-call entry point.
//
// nb_extract_batch_create validates every request like the per-call entry point, uploads the request
// descriptors once, optionally autotunes (tile shape x CTAs per SM, timed on the batch itself and
// cached per workload key in memory and in a small text file), and captures the launch — the pair
// copies of LINEAR batches, the direct grids, counter reset, persistent kernel — into a CUDA graph.
// nb_extract_batch_run replays that graph on a stream.
#include "fp_args.cuh"
#include "fp_pairs.cuh"
#include "fp_pool.cuh"
#include "noa_b200/batch.h"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <sstream>
#include <string>
#include <vector>

#include <sys/stat.h>

namespace nb {
namespace {

struct BatchReq {
    ProjArgs a;
    const float4* pairs;      // pair copy of the volume (LINEAR fast path), or null
    int ppt;                  // rows per thread: PAIRS_PPT with a pair copy, else 1
    int ntx;                  // tiles along u
    int tiles_per_slice;
    int64_t first_item;       // index of this request's first item
};
static_assert(sizeof(BatchReq) % 8 == 0, "BatchReq is staged in shared memory as 8-byte words");

constexpr int PAIRS_PPT = 4;
// Output pixels from which a request over a pair copy gets a grid of its own (about 8 slices of 128^2;
// smaller requests go through the persistent kernel). Measured on 12,000 LINEAR slices over 12
// volumes of 128-384 as 12, 120 and 600 requests: with grids of their own on 4 branches, 4.76, 4.61
// and 4.70 ms against 5.36, 5.78 and 6.57 ms all in the persistent kernel (per-call 4.94, 7.57, 13.2).
constexpr int64_t DIRECT_MIN_PIXELS = int64_t(1) << 16;
constexpr int N_SIDE = 4;  // graph branches the direct grids alternate on
// The same for the one-shot launch, whose grids are launched one by one from the host (a few
// microseconds each): 600 requests of ~20 slices as 596 grids took 16.9 ms against 6.6 ms in the
// persistent kernel, so only requests worth ~20 us of device time or more get a grid there.
constexpr int64_t ONESHOT_DIRECT_MIN_PIXELS = int64_t(1) << 21;

// PAIRS_PPT output pixels (rows y0, y0 + dy, ...) of column u read through the volume's pair copy:
// the body of extract_pairs_kernel (fp_extract.cu).
template<bool OUT_C>
__device__ __forceinline__ void extract_rows_pairs(const ProjArgs& a, const float4* pairs, int64_t b, int y0,
                                                   int dy, int u) {
    const Spectrum3 sp{a.vol_d, a.vol_h, a.vol_w, a.in_centered};
    const int WP = a.vol_w / 2 + 1;
    const float f1 = div(static_cast<float>(u), a.f_slice1);
    float2 value[PAIRS_PPT];
    bool inside[PAIRS_PPT];
    const float* m = nullptr;
    const bool lean = lean_rotation(a, b, m);
#pragma unroll
    for (int r = 0; r < PAIRS_PPT; ++r) {
        const int y = y0 + r * dy;
        value[r] = make_float2(0.f, 0.f);
        inside[r] = false;
        if (y >= a.slice_h)
            continue;
        const float f0 = div(static_cast<float>(index2frequency(a.out_centered, y, a.slice_h)), a.f_slice0);
        float fz, fy, fx;
        if (lean)
            slice2grid_lean(m, f0, f1, fz, fy, fx);
        else
            slice2grid(f0, f1, a.scale, a.rot, b, a.ews, fz, fy, fx);
        inside[r] = dot3(fz, fy, fx, fz, fy, fx) <= a.cutoff_sqd;
        if (inside[r])
            value[r] = to_output<true, OUT_C>(interp_linear_pairs(pairs, a.vol_h * WP, WP, sp, mul(fz, a.target0),
                                                                  mul(fy, a.target1), mul(fx, a.target2)));
    }
#pragma unroll
    for (int r = 0; r < PAIRS_PPT; ++r) {
        const int y = y0 + r * dy;
        if (y >= a.slice_h)
            continue;
        dst_store_stream<OUT_C>(a.out, b, y, u, value[r]);
        if (a.out_w.present)
            store_real_stream(a.out_w, b, y, u, inside[r] ? 1.f : 0.f);
    }
}

// One output pixel (b, y, u) of request `a`: the body of extract_kernel (fp_extract.cu), with 32-bit
// volume offsets (batches require volumes addressable in 31 bits).
template<int I, bool IN_C, bool OUT_C>
__device__ __forceinline__ void extract_one(const ProjArgs& a, int64_t b, int y, int u) {
    const Spectrum3 sp{a.vol_d, a.vol_h, a.vol_w, a.in_centered};
    const View3<int> vol{a.in.data, static_cast<int>(a.in.s0), static_cast<int>(a.in.s1), static_cast<int>(a.in.s2)};
    const View3<int> volw{a.in_w.data, static_cast<int>(a.in_w.s0), static_cast<int>(a.in_w.s1),
                          static_cast<int>(a.in_w.s2)};
    const bool has_out_w = a.out_w.present;
    const bool has_in_w = a.in_w.present;
    const int v = index2frequency(a.out_centered, y, a.slice_h);
    const float f0 = div(static_cast<float>(v), a.f_slice0);
    const float f1 = div(static_cast<float>(u), a.f_slice1);
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
            const float cw = windowed_sinc(off, a.efs, a.efb);
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

// Kernel variants of the autotuner: tile shape (256 threads; a warp covers WY x WX pixels) and the
// minimum resident CTAs per SM promised to the compiler (4 caps registers at 64 per thread, trading
// spills of the wide stencils for twice the resident warps).
constexpr int N_VARIANTS = 3;
struct Variant { int ty, tx, wy, wx, min_ctas; };
constexpr Variant VARIANTS[N_VARIANTS] = {{16, 16, 4, 8, 1}, {8, 32, 2, 16, 1}, {16, 16, 4, 8, 4}};

// PAIRS_ONLY: every request reads a pair copy (LINEAR, complex); the generic path is compiled out so
// the kernel fits 40 registers (6 CTAs per SM, like extract_pairs_kernel).
template<int I, bool IN_C, bool OUT_C, int V, bool PAIRS_ONLY = false>
__global__ void __launch_bounds__(256, PAIRS_ONLY ? 6 : VARIANTS[V].min_ctas)
batch_extract_kernel(const BatchReq* __restrict__ reqs, int n_req, int64_t n_items,
                     unsigned long long* __restrict__ counter) {
    constexpr Variant VT = VARIANTS[V];
    constexpr int WORDS = sizeof(BatchReq) / 8;
    __shared__ unsigned long long s_req_words[WORDS];  // the current request, staged once per change
    const BatchReq& R = *reinterpret_cast<const BatchReq*>(s_req_words);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr int WARPS_X = VT.tx / VT.wx;
    const int ly = (warp / WARPS_X) * VT.wy + lane / VT.wx;
    const int lx = (warp % WARPS_X) * VT.wx + lane % VT.wx;
    int staged = -1;   // request held in s_req_words
    int found = 0;     // request of the last item (a CTA's items only increase)
    // Items are claimed in chunks of consecutive items, ~64 claims per CTA over the launch (at most 64
    // items per claim), so cheap items do not queue on the counter. Thread 0 claims the next chunk
    // while the current one is processed, so the counter's round trip is hidden behind the work.
    const long long per_cta = n_items / (static_cast<long long>(gridDim.x) * 64);
    const long long chunk = per_cta < 1 ? 1 : (per_cta > 64 ? 64 : per_cta);
    __shared__ long long s_chunk[2];
    long long next = threadIdx.x == 0 ? static_cast<long long>(atomicAdd(counter, static_cast<unsigned long long>(chunk))) : 0;
    for (int round = 0;; ++round) {
        if (threadIdx.x == 0) {
            s_chunk[round & 1] = next;
            if (next < n_items)
                next = static_cast<long long>(atomicAdd(counter, static_cast<unsigned long long>(chunk)));
        }
        __syncthreads();
        // Double-buffered: thread 0 writes the other slot next round, after at least one more barrier.
        const long long c0 = s_chunk[round & 1];
        if (c0 >= n_items)
            break;
        const long long c1 = c0 + chunk < n_items ? c0 + chunk : n_items;
        // (slice, tile row, tile column) of the item: divided out once per chunk or request, then
        // advanced item by item (consecutive items walk a slice's tiles row-major).
        int64_t b = 0;
        int ty = 0, tx = 0, nty = 1;
        bool fresh = true;
        for (long long item = c0; item < c1; ++item) {
            // Every thread finds the item's request the same way (uniform), from the previous one.
            if (found + 1 < n_req && reqs[found + 1].first_item <= item) {
                int lo = found + 1, hi = n_req - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) / 2;
                    if (reqs[mid].first_item <= item)
                        lo = mid;
                    else
                        hi = mid - 1;
                }
                found = lo;
            }
            if (found != staged) {
                __syncthreads();  // nobody still reads the previous descriptor
                const auto* src = reinterpret_cast<const unsigned long long*>(reqs + found);
                for (int i = threadIdx.x; i < WORDS; i += blockDim.x)
                    s_req_words[i] = src[i];
                staged = found;
                fresh = true;
                __syncthreads();
            }
            if (fresh) {
                const int64_t local = item - R.first_item;
                b = local / R.tiles_per_slice;
                const int tile = static_cast<int>(local - b * R.tiles_per_slice);
                ty = tile / R.ntx;
                tx = tile - ty * R.ntx;
                nty = R.tiles_per_slice / R.ntx;
                fresh = false;
            }
            const int u = tx * VT.tx + lx;
            if (u < R.a.slice_w / 2 + 1) {
                bool done = false;
                if constexpr (I == I_LINEAR && IN_C) {
                    if (PAIRS_ONLY || R.pairs) {
                        extract_rows_pairs<OUT_C>(R.a, R.pairs, b, ty * (VT.ty * PAIRS_PPT) + ly, VT.ty, u);
                        done = true;
                    }
                }
                if constexpr (!PAIRS_ONLY) {
                    const int y = ty * VT.ty + ly;
                    if (!done && y < R.a.slice_h)
                        extract_one<I, IN_C, OUT_C>(R.a, b, y, u);
                }
            }
            if (++tx == R.ntx) {
                tx = 0;
                if (++ty == nty) {
                    ty = 0;
                    ++b;
                }
            }
        }
    }
}

// Pairs-only batch graphs of at most PACK requests pass their descriptors as a kernel parameter: the
// request fields are then read through the constant bank like a per-call kernel's arguments, with no
// staging in shared memory and no barrier when a CTA's request changes (28.4 KB of parameters, within
// the 32 KB that sm_70+ kernels accept). Only captured graphs use it, where the parameters are set
// once: one-shot launches keep the shared-memory descriptors.
constexpr int PACK = 48;
struct ReqPack { BatchReq r[PACK]; };
static_assert(sizeof(ReqPack) + 64 <= 32764, "the descriptor pack must fit the kernel parameter space");

template<bool OUT_C>
__global__ void __launch_bounds__(256, 6)
batch_pairs_param_kernel(const __grid_constant__ ReqPack pack, int n_req, int64_t n_items,
                         unsigned long long* __restrict__ counter) {
    constexpr Variant VT = VARIANTS[0];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr int WARPS_X = VT.tx / VT.wx;
    const int ly = (warp / WARPS_X) * VT.wy + lane / VT.wx;
    const int lx = (warp % WARPS_X) * VT.wx + lane % VT.wx;
    int found = 0;
    const long long per_cta = n_items / (static_cast<long long>(gridDim.x) * 64);
    const long long chunk = per_cta < 1 ? 1 : (per_cta > 64 ? 64 : per_cta);
    __shared__ long long s_chunk[2];
    long long next = threadIdx.x == 0 ? static_cast<long long>(atomicAdd(counter, static_cast<unsigned long long>(chunk))) : 0;
    for (int round = 0;; ++round) {
        if (threadIdx.x == 0) {
            s_chunk[round & 1] = next;
            if (next < n_items)
                next = static_cast<long long>(atomicAdd(counter, static_cast<unsigned long long>(chunk)));
        }
        __syncthreads();
        const long long c0 = s_chunk[round & 1];
        if (c0 >= n_items)
            break;
        const long long c1 = c0 + chunk < n_items ? c0 + chunk : n_items;
        int64_t b = 0;
        int ty = 0, tx = 0, nty = 1;
        bool fresh = true;
        for (long long item = c0; item < c1; ++item) {
            if (found + 1 < n_req && pack.r[found + 1].first_item <= item) {
                int lo = found + 1, hi = n_req - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) / 2;
                    if (pack.r[mid].first_item <= item)
                        lo = mid;
                    else
                        hi = mid - 1;
                }
                found = lo;
                fresh = true;
            }
            const BatchReq& R = pack.r[found];
            if (fresh) {
                const int64_t local = item - R.first_item;
                b = local / R.tiles_per_slice;
                const int tile = static_cast<int>(local - b * R.tiles_per_slice);
                ty = tile / R.ntx;
                tx = tile - ty * R.ntx;
                nty = R.tiles_per_slice / R.ntx;
                fresh = false;
            }
            const int u = tx * VT.tx + lx;
            if (u < R.a.slice_w / 2 + 1)
                extract_rows_pairs<OUT_C>(R.a, R.pairs, b, ty * (VT.ty * PAIRS_PPT) + ly, VT.ty, u);
            if (++tx == R.ntx) {
                tx = 0;
                if (++ty == nty) {
                    ty = 0;
                    ++b;
                }
            }
        }
    }
}

using KernelFn = void (*)(const BatchReq*, int, int64_t, unsigned long long*);

template<int I, bool IN_C, bool OUT_C>
KernelFn pick_v(int v) {
    switch (v) {
        case 0: return batch_extract_kernel<I, IN_C, OUT_C, 0>;
        case 1: return batch_extract_kernel<I, IN_C, OUT_C, 1>;
        default: return batch_extract_kernel<I, IN_C, OUT_C, 2>;
    }
}

template<int I>
KernelFn pick_t(bool in_c, bool out_c, int v) {
    if (in_c && out_c) return pick_v<I, true, true>(v);
    if (in_c) return pick_v<I, true, false>(v);
    return pick_v<I, false, false>(v);
}

KernelFn pick_kernel(int interp, bool in_c, bool out_c, int v) {
    switch (interp) {
        case I_NEAREST: return pick_t<I_NEAREST>(in_c, out_c, v);
        case I_LINEAR: return pick_t<I_LINEAR>(in_c, out_c, v);
        case I_CUBIC: return pick_t<I_CUBIC>(in_c, out_c, v);
        case I_BSPLINE: return pick_t<I_BSPLINE>(in_c, out_c, v);
        case I_LANCZOS4: return pick_t<I_LANCZOS4>(in_c, out_c, v);
        case I_LANCZOS6: return pick_t<I_LANCZOS6>(in_c, out_c, v);
        default: return pick_t<I_LANCZOS8>(in_c, out_c, v);
    }
}

// ---------------------------------------------------------------------------------------------------
// Autotune cache: "key variant blocks_per_sm ms" lines, in memory and in a text file
// ($NB_AUTOTUNE_CACHE, else $HOME/.cache/noa_b200/autotune.txt).
// ---------------------------------------------------------------------------------------------------
std::mutex g_tune_mutex;
std::map<std::string, std::pair<int, int>> g_tuned;
std::string g_loaded_path;
bool g_tune_loaded = false;

std::string cache_path() {
    if (const char* p = std::getenv("NB_AUTOTUNE_CACHE"))
        return p;
    if (const char* h = std::getenv("HOME"))
        return std::string(h) + "/.cache/noa_b200/autotune.txt";
    return "";
}

void load_cache_locked() {
    const std::string path = cache_path();
    if (g_tune_loaded && path == g_loaded_path)
        return;
    g_tune_loaded = true;
    g_loaded_path = path;
    g_tuned.clear();
    if (path.empty())
        return;
    std::ifstream f(path);
    std::string line;
    while (std::getline(f, line)) {
        std::istringstream is(line);
        std::string key;
        int v = 0, bps = 0;
        double ms = 0;
        if (is >> key >> v >> bps >> ms && v >= 0 && v < N_VARIANTS && bps > 0)
            g_tuned[key] = {v, bps};
    }
}

void store_cache_locked(const std::string& key, int v, int bps, double ms) {
    g_tuned[key] = {v, bps};
    const std::string path = cache_path();
    if (path.empty())
        return;
    const size_t slash = path.rfind('/');
    if (slash != std::string::npos && slash > 0) {
        const std::string dir = path.substr(0, slash);
        for (size_t i = 1; i <= dir.size(); ++i) {
            if (i == dir.size() || dir[i] == '/')
                mkdir(dir.substr(0, i).c_str(), 0755);  // existing levels fail harmlessly
        }
    }
    std::ofstream f(path, std::ios::app);
    if (f)
        f << key << ' ' << v << ' ' << bps << ' ' << ms << '\n';
}

struct Config {
    int variant;
    int blocks_per_sm;
};

} // namespace
} // namespace nb

using namespace nb;

struct nb_extract_batch_t {
    int device = 0;
    int interp = 1;
    bool in_cplx = true, out_cplx = true;
    std::vector<BatchReq> host_reqs;     // ProjArgs of every request; tile fields per variant
    BatchReq* d_reqs = nullptr;
    unsigned long long* d_counter = nullptr;
    int64_t n_items = 0;
    Config cfg{0, 1};
    int grid = 0;
    double tuned_ms = -1;
    bool from_cache = false;
    std::string key;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    // LINEAR batches: pair copies of the volumes read enough to amortise one, rebuilt by every run
    // (their make_pairs launches are part of the graph), so later changes to the volumes are seen.
    std::vector<std::pair<nb::ProjArgs, float4*>> pair_jobs;
    bool pairs_only = false;  // every request reads a pair copy: the pairs-only kernel
    // Requests over a pair copy with at least DIRECT_MIN_PIXELS output pixels leave the persistent
    // kernel: each runs the per-call pair kernel as a grid of its own on one of N_SIDE branches of the
    // graph, as soon as its volume's copy is written, while the copies of the next volumes are made on
    // a higher-priority branch. The per-call kernel's per-pixel cost is lower than the persistent
    // kernel's (no claims, request lookups or per-item tile setup), and with several branches the
    // grids' ramps and tails overlap. (The copies, HBM-bound, overlap the extractions only a little:
    // 0.62 ms of copies for 12 volumes of 128-384 saved 0.08 ms against copying first.)
    std::vector<BatchReq> direct;
    std::vector<size_t> direct_job;      // pair_jobs index of each direct request's copy
    int64_t n_requests = 0;              // persistent + direct
    cudaStream_t copy_stream = nullptr, side[N_SIDE] = {};
    cudaEvent_t ev_fork = nullptr, ev_join[N_SIDE + 1] = {};
    std::vector<cudaEvent_t> ev_pairs;   // one per pair job
};

namespace nb {
namespace {

int max_blocks_per_sm(KernelFn fn) {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, 256, 0) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    return n > 0 ? n : 1;
}

// Tile fields of one request for a variant; `first` is its first item and advances past its items.
void set_tiles(BatchReq& r, const Variant& vt, int64_t& first) {
    r.ppt = r.pairs ? PAIRS_PPT : 1;
    const int wp = r.a.slice_w / 2 + 1;
    const int th = vt.ty * r.ppt;
    r.ntx = (wp + vt.tx - 1) / vt.tx;
    r.tiles_per_slice = r.ntx * ((r.a.slice_h + th - 1) / th);
    r.first_item = first;
    first += static_cast<int64_t>(r.tiles_per_slice) * r.a.n_slices;
}

// Fills the per-variant tile fields and uploads the descriptors.
cudaError_t upload(nb_extract_batch_t* h, int variant, cudaStream_t stream) {
    const Variant vt = VARIANTS[variant];
    int64_t first = 0;
    for (BatchReq& r : h->host_reqs)
        set_tiles(r, vt, first);
    h->n_items = first;
    cudaError_t err = cudaMemcpyAsync(h->d_reqs, h->host_reqs.data(), h->host_reqs.size() * sizeof(BatchReq),
                                      cudaMemcpyHostToDevice, stream);
    if (err != cudaSuccess)
        return err;
    return cudaStreamSynchronize(stream);
}

KernelFn pairs_only_kernel(bool out_c) {
    return out_c ? batch_extract_kernel<I_LINEAR, true, true, 0, true> : batch_extract_kernel<I_LINEAR, true, false, 0, true>;
}

int param_blocks_per_sm(bool out_c) {
    int n = 0;
    const cudaError_t e = out_c ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_pairs_param_kernel<true>, 256, 0)
                                : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_pairs_param_kernel<false>, 256, 0);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    return n > 0 ? n : 1;
}

// The pairs-only kernel with the descriptors (tile fields set for variant 0) as its parameter.
cudaError_t launch_param(const std::vector<BatchReq>& reqs, int64_t n_items, bool out_c, int blocks_per_sm,
                         unsigned long long* counter, cudaStream_t s) {
    auto pack = std::make_unique<ReqPack>();
    std::memset(static_cast<void*>(pack.get()), 0, sizeof(ReqPack));
    std::copy(reqs.begin(), reqs.end(), pack->r);
    const int n = static_cast<int>(reqs.size());
    const int grid = sm_count() * blocks_per_sm;
    if (out_c)
        batch_pairs_param_kernel<true><<<grid, 256, 0, s>>>(*pack, n, n_items, counter);
    else
        batch_pairs_param_kernel<false><<<grid, 256, 0, s>>>(*pack, n, n_items, counter);
    return cudaGetLastError();
}

bool use_param(const nb_extract_batch_t* h) {
    return h->pairs_only && h->host_reqs.size() <= static_cast<size_t>(PACK);
}

// The counter reset and the persistent kernel over the requests left in host_reqs.
cudaError_t launch_persistent(nb_extract_batch_t* h, const Config& c, cudaStream_t stream) {
    if (h->n_items == 0)
        return cudaSuccess;
    const KernelFn fn = h->pairs_only ? pairs_only_kernel(h->out_cplx)
                                      : pick_kernel(h->interp, h->in_cplx, h->out_cplx, c.variant);
    const int grid = sm_count() * c.blocks_per_sm;
    const cudaError_t err = cudaMemsetAsync(h->d_counter, 0, sizeof(unsigned long long), stream);
    if (err != cudaSuccess)
        return err;
    if (use_param(h))
        return launch_param(h->host_reqs, h->n_items, h->out_cplx, c.blocks_per_sm, h->d_counter, stream);
    fn<<<grid, 256, 0, stream>>>(h->d_reqs, static_cast<int>(h->host_reqs.size()), h->n_items, h->d_counter);
    return cudaGetLastError();
}

cudaError_t launch(nb_extract_batch_t* h, const Config& c, cudaStream_t stream) {
    cudaError_t err = cudaSuccess;
    if (h->direct.empty()) {
        for (const auto& job : h->pair_jobs)
            if ((err = launch_make_pairs(job.first, job.second, stream)) != cudaSuccess)
                return err;
        return launch_persistent(h, c, stream);
    }
    // Fork: copies on copy_stream, direct grids in turn on the side streams, the persistent kernel
    // after the last copy on copy_stream; everything joins back into `stream`.
    if ((err = cudaEventRecord(h->ev_fork, stream)) != cudaSuccess)
        return err;
    cudaStream_t branch[N_SIDE + 1] = {h->copy_stream};
    for (int k = 0; k < N_SIDE; ++k)
        branch[k + 1] = h->side[k];
    for (cudaStream_t b : branch)
        if ((err = cudaStreamWaitEvent(b, h->ev_fork, 0)) != cudaSuccess)
            return err;
    int least = 0, greatest = 0;
    if ((err = cudaDeviceGetStreamPriorityRange(&least, &greatest)) != cudaSuccess)
        return err;
    for (size_t j = 0; j < h->pair_jobs.size(); ++j) {
        if ((err = launch_make_pairs(h->pair_jobs[j].first, h->pair_jobs[j].second, h->copy_stream, &greatest)) !=
            cudaSuccess)
            return err;
        if ((err = cudaEventRecord(h->ev_pairs[j], h->copy_stream)) != cudaSuccess)
            return err;
    }
    for (size_t k = 0; k < h->direct.size(); ++k) {
        const cudaStream_t s = h->side[k % N_SIDE];
        if ((err = cudaStreamWaitEvent(s, h->ev_pairs[h->direct_job[k]], 0)) != cudaSuccess)
            return err;
        if ((err = launch_extract_pairs(h->direct[k].a, h->direct[k].pairs, s)) != cudaSuccess)
            return err;
    }
    if ((err = launch_persistent(h, c, h->copy_stream)) != cudaSuccess)
        return err;
    for (int k = 0; k < N_SIDE + 1; ++k) {
        if ((err = cudaEventRecord(h->ev_join[k], branch[k])) != cudaSuccess)
            return err;
        if ((err = cudaStreamWaitEvent(stream, h->ev_join[k], 0)) != cudaSuccess)
            return err;
    }
    return cudaSuccess;
}

// Median of `reps` timed launches (after one warm-up), in milliseconds.
double time_config(nb_extract_batch_t* h, const Config& c, cudaStream_t stream, int reps) {
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    std::vector<float> t;
    double result = 1e30;
    if (launch(h, c, stream) == cudaSuccess && cudaStreamSynchronize(stream) == cudaSuccess) {
        for (int i = 0; i < reps; ++i) {
            cudaEventRecord(e0, stream);
            if (launch(h, c, stream) != cudaSuccess)
                break;
            cudaEventRecord(e1, stream);
            if (cudaEventSynchronize(e1) != cudaSuccess)
                break;
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            t.push_back(ms);
        }
        if (!t.empty()) {
            std::sort(t.begin(), t.end());
            result = t[t.size() / 2];
        }
    }
    cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return result;
}

// LINEAR over complex volumes: a pair copy per distinct volume whose requests read at least twice
// as many pixels as it has voxels (the per-call rule), allocated for the batch's lifetime. Without
// memory for a copy, its requests take the generic path.
void plan_pairs(nb_extract_batch_t* h, bool allow_direct) {
    if (h->interp != I_LINEAR || !h->in_cplx)
        return;
    struct Vol { const ProjArgs* a; int64_t pixels; std::vector<size_t> reqs; };
    std::vector<Vol> vols;
    for (size_t i = 0; i < h->host_reqs.size(); ++i) {
        const ProjArgs& a = h->host_reqs[i].a;
        if (!pairs_apply(a))
            continue;
        Vol* v = nullptr;
        for (Vol& c : vols)
            if (c.a->in.data == a.in.data && c.a->vol_d == a.vol_d && c.a->vol_h == a.vol_h &&
                c.a->vol_w == a.vol_w && c.a->in.s0 == a.in.s0 && c.a->in.s1 == a.in.s1 &&
                c.a->in.s2 == a.in.s2 && c.a->in_centered == a.in_centered)
                v = &c;
        if (!v) {
            vols.push_back({&a, 0, {}});
            v = &vols.back();
        }
        v->pixels += a.n_slices * a.slice_h * static_cast<int64_t>(a.slice_w / 2 + 1);
        v->reqs.push_back(i);
    }
    for (const Vol& v : vols) {
        const int64_t vox = static_cast<int64_t>(v.a->vol_d) * v.a->vol_h * (v.a->vol_w / 2 + 1);
        if (v.pixels < 2 * vox)
            continue;
        float4* buf = static_cast<float4*>(device_alloc(static_cast<size_t>(vox) * sizeof(float4)));
        if (!buf)
            continue;  // no memory for the copy: these requests read the volume itself
        h->pair_jobs.push_back({*v.a, buf});
        for (size_t i : v.reqs)
            h->host_reqs[i].pairs = buf;
    }
    // Copies in increasing size, so the first direct grids start early and the largest copies overlap
    // the extractions.
    std::stable_sort(h->pair_jobs.begin(), h->pair_jobs.end(), [](const auto& x, const auto& y) {
        return static_cast<int64_t>(x.first.vol_d) * x.first.vol_h * x.first.vol_w <
               static_cast<int64_t>(y.first.vol_d) * y.first.vol_h * y.first.vol_w;
    });
    std::vector<BatchReq> keep;
    for (size_t j = 0; j < h->pair_jobs.size(); ++j)
        for (const BatchReq& r : h->host_reqs)
            if (allow_direct && r.pairs == h->pair_jobs[j].second &&
                r.a.n_slices * r.a.slice_h * static_cast<int64_t>(r.a.slice_w / 2 + 1) >= DIRECT_MIN_PIXELS) {
                h->direct.push_back(r);
                h->direct_job.push_back(j);
            }
    for (const BatchReq& r : h->host_reqs)
        if (!(allow_direct && r.pairs &&
              r.a.n_slices * r.a.slice_h * static_cast<int64_t>(r.a.slice_w / 2 + 1) >= DIRECT_MIN_PIXELS))
            keep.push_back(r);
    h->host_reqs.swap(keep);
    bool all = true;
    for (const BatchReq& r : h->host_reqs)
        all = all && r.pairs != nullptr;
    h->pairs_only = all;
}

// Streams and events of a batch with direct requests (see nb_extract_batch_t::direct).
cudaError_t make_branches(nb_extract_batch_t* h) {
    if (h->direct.empty())
        return cudaSuccess;
    int least = 0, greatest = 0;
    cudaError_t err = cudaDeviceGetStreamPriorityRange(&least, &greatest);
    if (err == cudaSuccess)
        err = cudaStreamCreateWithPriority(&h->copy_stream, cudaStreamNonBlocking, greatest);
    for (int k = 0; k < N_SIDE && err == cudaSuccess; ++k)
        err = cudaStreamCreateWithPriority(&h->side[k], cudaStreamNonBlocking, least);
    if (err == cudaSuccess)
        err = cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming);
    for (int k = 0; k < N_SIDE + 1 && err == cudaSuccess; ++k)
        err = cudaEventCreateWithFlags(&h->ev_join[k], cudaEventDisableTiming);
    h->ev_pairs.assign(h->pair_jobs.size(), nullptr);
    for (size_t j = 0; j < h->ev_pairs.size() && err == cudaSuccess; ++j)
        err = cudaEventCreateWithFlags(&h->ev_pairs[j], cudaEventDisableTiming);
    return err;
}

std::string workload_key(const nb_extract_batch_t* h) {
    std::set<std::string> boxes;
    int64_t slices = 0;
    for (const BatchReq& r : h->host_reqs) {
        boxes.insert(std::to_string(r.a.vol_d) + "x" + std::to_string(r.a.vol_h) + "x" + std::to_string(r.a.vol_w));
        slices += r.a.n_slices;
    }
    std::ostringstream k;
    k << "extract/i" << h->interp << "/t" << h->in_cplx << h->out_cplx << "/sm" << sm_count() << "/b";
    for (const std::string& b : boxes)
        k << b << ',';
    int64_t bucket = 1;
    while (bucket < slices)
        bucket *= 2;
    k << "/s" << bucket;
    return k.str();
}

void release(nb_extract_batch_t* h) {
    if (!h)
        return;
    if (h->exec) cudaGraphExecDestroy(h->exec);
    if (h->graph) cudaGraphDestroy(h->graph);
    if (h->d_reqs) cudaFree(h->d_reqs);
    if (h->d_counter) cudaFree(h->d_counter);
    for (auto& job : h->pair_jobs)
        cudaFree(job.second);
    if (h->copy_stream) cudaStreamDestroy(h->copy_stream);
    for (cudaStream_t st : h->side)
        if (st) cudaStreamDestroy(st);
    if (h->ev_fork) cudaEventDestroy(h->ev_fork);
    for (cudaEvent_t e : h->ev_join)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : h->ev_pairs)
        if (e) cudaEventDestroy(e);
    delete h;
}

// Stages the descriptors of `h` in stream-ordered device memory and launches `fn` once on `s`.
int launch_once(nb_extract_batch_t& h, KernelFn fn, int variant, int blocks_per_sm, cudaStream_t s) {
    const Variant vt = VARIANTS[variant];
    int64_t first = 0;
    for (BatchReq& r : h.host_reqs)
        set_tiles(r, vt, first);
    if (first == 0)
        return finish_launch(cudaSuccess);
    // Descriptors then the work counter, in one stream-ordered allocation.
    const size_t desc_bytes = (h.host_reqs.size() * sizeof(BatchReq) + 255) / 256 * 256;
    void* dev = scratch_alloc(desc_bytes + sizeof(unsigned long long), s);
    if (!dev)
        return report_error(NB_ERROR_OOM, "cannot allocate the batch descriptors");
    auto* d_reqs = static_cast<BatchReq*>(dev);
    auto* d_counter = reinterpret_cast<unsigned long long*>(static_cast<char*>(dev) + desc_bytes);
    // The host vector goes when this returns: upload_async copies it in a form a capture keeps.
    cudaError_t err = upload_async(d_reqs, h.host_reqs.data(), h.host_reqs.size() * sizeof(BatchReq), s);
    if (err == cudaSuccess)
        err = cudaMemsetAsync(d_counter, 0, sizeof(unsigned long long), s);
    if (err == cudaSuccess) {
        fn<<<sm_count() * blocks_per_sm, 256, 0, s>>>(d_reqs, static_cast<int>(h.host_reqs.size()), first, d_counter);
        err = cudaGetLastError();
    }
    scratch_free(dev, s);
    return finish_launch(err);
}

} // namespace
} // namespace nb

extern "C" {

int nb_extract_batch_create(int32_t remap, const nb_extract_request* requests, int64_t n_requests,
                            const nb_options* options, int32_t flags, void* stream, nb_extract_batch* out) {
    if (!out)
        return report_error(NB_ERROR_INVALID, "out should not be NULL");
    *out = nullptr;
    if (!requests || n_requests <= 0)
        return report_error(NB_ERROR_INVALID, "a batch needs at least one request");
    if (n_requests > (int64_t(1) << 30))
        return report_error(NB_ERROR_INVALID, "too many requests");
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (stream_capturing(s))
        return report_error(NB_ERROR_INVALID, "a batch is created outside a stream capture (creation uploads, "
                                              "may autotune and synchronizes); its runs may be captured");
    auto* h = new nb_extract_batch_t();
    cudaGetDevice(&h->device);
    h->host_reqs.resize(static_cast<size_t>(n_requests));
    for (int64_t i = 0; i < n_requests; ++i) {
        const nb_extract_request& q = requests[i];
        ProjArgs a{};
        const int st = prepare_extract(remap, q.volume, q.volume_weight, q.volume_shape, q.slice, q.slice_weight,
                                       q.slice_shape, q.inv_scaling, q.fwd_rotation, options, a);
        if (st != NB_OK) {
            release(h);
            return st;
        }
        if (a.wide_in) {
            release(h);
            return report_error(NB_ERROR_INVALID, "batched volumes must span fewer than 2^31 elements");
        }
        if (i == 0) {
            h->interp = a.interp;
            h->in_cplx = a.in_cplx;
            h->out_cplx = a.out_cplx;
        } else if (a.in_cplx != h->in_cplx || a.out_cplx != h->out_cplx) {
            release(h);
            return report_error(NB_ERROR_INVALID, "all requests of a batch must have the same value types");
        }
        h->host_reqs[static_cast<size_t>(i)].a = a;
        h->host_reqs[static_cast<size_t>(i)].pairs = nullptr;
    }
    h->n_requests = n_requests;
    plan_pairs(h, !(flags & NB_BATCH_PERSISTENT_ONLY));
    if (const cudaError_t berr = make_branches(h); berr != cudaSuccess) {
        release(h);
        return finish_launch(berr);
    }
    h->d_reqs = static_cast<BatchReq*>(device_alloc(std::max<size_t>(1, h->host_reqs.size()) * sizeof(BatchReq)));
    h->d_counter = static_cast<unsigned long long*>(h->d_reqs ? device_alloc(sizeof(unsigned long long)) : nullptr);
    if (!h->d_reqs || !h->d_counter) {
        release(h);
        return report_error(NB_ERROR_OOM, "cannot allocate the batch descriptors");
    }

    // Configuration: autotuned (cached per workload key), or the default. With a pair copy for every
    // request, the pairs-only kernel at full occupancy (as the one-shot launch uses).
    h->key = workload_key(h);
    Config best{0, use_param(h) ? param_blocks_per_sm(h->out_cplx)
                                : max_blocks_per_sm(h->pairs_only ? pairs_only_kernel(h->out_cplx)
                                                                  : pick_kernel(h->interp, h->in_cplx, h->out_cplx, 0))};
    bool tuned = h->pairs_only;
    if ((flags & NB_BATCH_AUTOTUNE) && !tuned) {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        load_cache_locked();
        auto it = g_tuned.find(h->key);
        if (it != g_tuned.end()) {
            best = {it->second.first, it->second.second};
            h->from_cache = true;
            tuned = true;
        }
    }
    if ((flags & NB_BATCH_AUTOTUNE) && !tuned) {
        double best_ms = 1e30;
        for (int v = 0; v < N_VARIANTS; ++v) {
            if (upload(h, v, s) != cudaSuccess)
                continue;
            const int max_b = max_blocks_per_sm(pick_kernel(h->interp, h->in_cplx, h->out_cplx, v));
            const std::set<int> cands{1, 2, 4, max_b};
            for (int bps : cands) {
                if (bps > max_b)
                    continue;
                const double ms = time_config(h, Config{v, bps}, s, 3);
                if (ms < best_ms) {
                    best_ms = ms;
                    best = {v, bps};
                }
            }
        }
        h->tuned_ms = best_ms;
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        store_cache_locked(h->key, best.variant, best.blocks_per_sm, best_ms);
    }
    h->cfg = best;
    cudaError_t err = upload(h, best.variant, s);
    if (err != cudaSuccess) {
        release(h);
        return finish_launch(err);
    }
    h->grid = sm_count() * best.blocks_per_sm;

    // Capture counter reset + persistent kernel into a graph, on a private stream.
    cudaStream_t cap;
    if ((err = cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking)) == cudaSuccess) {
        err = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
        if (err == cudaSuccess) {
            const cudaError_t lerr = launch(h, best, cap);
            err = cudaStreamEndCapture(cap, &h->graph);
            if (err == cudaSuccess && lerr != cudaSuccess)
                err = lerr;
        }
        // Node priorities: the copies' branch was captured from a higher-priority stream.
        if (err == cudaSuccess)
            err = cudaGraphInstantiateWithFlags(&h->exec, h->graph, cudaGraphInstantiateFlagUseNodePriority);
        cudaStreamDestroy(cap);
    }
    if (err != cudaSuccess) {
        release(h);
        return finish_launch(err);
    }
    *out = h;
    return finish_launch(cudaSuccess);
}

int nb_extract_batch_run(nb_extract_batch batch, void* stream) {
    if (!batch || !batch->exec)
        return report_error(NB_ERROR_INVALID, "invalid batch handle");
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    // Inside a caller's stream capture the batch's launch sequence (the same copies, kernels and
    // branches its own graph holds) is issued into that capture instead of launching the graph.
    if (stream_capturing(s))
        return finish_launch(launch(batch, batch->cfg, s));
    return finish_launch(cudaGraphLaunch(batch->exec, s));
}

int nb_extract_batch_info(nb_extract_batch batch, nb_batch_info* info) {
    if (!batch || !info)
        return report_error(NB_ERROR_INVALID, "invalid batch handle");
    const Variant vt = VARIANTS[batch->cfg.variant];
    info->n_requests = batch->n_requests;
    info->n_items = batch->n_items;
    info->tile_h = vt.ty;
    info->tile_w = vt.tx;
    info->blocks_per_sm = batch->cfg.blocks_per_sm;
    info->grid = batch->grid;
    info->tuned_ms = batch->tuned_ms;
    info->from_cache = batch->from_cache;
    info->min_ctas = vt.min_ctas;
    info->n_direct = static_cast<int32_t>(batch->direct.size());
    return NB_OK;
}

int nb_extract_batch_destroy(nb_extract_batch batch) {
    release(batch);
    return NB_OK;
}

int nb_extract_batch_launch(int32_t remap, const nb_extract_request_ex* requests, int64_t n_requests,
                            const nb_options* options, void* stream) {
    return nb_extract_batch_launch_ex(remap, requests, n_requests, options, 0, stream);
}

int nb_extract_batch_launch_ex(int32_t remap, const nb_extract_request_ex* requests, int64_t n_requests,
                               const nb_options* options, int32_t flags, void* stream) {
    if (!requests || n_requests <= 0)
        return report_error(NB_ERROR_INVALID, "a batch needs at least one request");
    if (n_requests > (int64_t(1) << 30))
        return report_error(NB_ERROR_INVALID, "too many requests");
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    nb_extract_batch_t h;  // host-side description only: no graph, no device descriptors of its own
    h.host_reqs.resize(static_cast<size_t>(n_requests));
    for (int64_t i = 0; i < n_requests; ++i) {
        const nb_extract_request& q = requests[i].call;
        ProjArgs a{};
        int st = prepare_extract(remap, q.volume, q.volume_weight, q.volume_shape, q.slice, q.slice_weight,
                                 q.slice_shape, q.inv_scaling, q.fwd_rotation, options, a);
        if (st != NB_OK)
            return st;
        if (a.wide_in)
            return report_error(NB_ERROR_INVALID, "batched volumes must span fewer than 2^31 elements");
        if (i == 0) {
            h.interp = a.interp;
            h.in_cplx = a.in_cplx;
            h.out_cplx = a.out_cplx;
        } else if (a.in_cplx != h.in_cplx || a.out_cplx != h.out_cplx) {
            return report_error(NB_ERROR_INVALID, "all requests of a batch must have the same value types");
        }
        BatchReq& r = h.host_reqs[static_cast<size_t>(i)];
        r.a = a;
        r.pairs = nullptr;
        if (requests[i].volume_pairs && pairs_apply(a)) {
            if ((st = check_pairs(requests[i].volume_pairs, requests[i].volume_pairs_bytes, a, "volume_pairs")) != NB_OK)
                return st;
            r.pairs = static_cast<const float4*>(requests[i].volume_pairs);
        }
    }
    // Validated: from here on, requests large enough over a pair copy are launched as grids of their
    // own, in order, and leave the persistent launch.
    if (!(flags & NB_BATCH_PERSISTENT_ONLY)) {
        std::vector<BatchReq> keep;
        for (const BatchReq& r : h.host_reqs) {
            if (r.pairs &&
                r.a.n_slices * r.a.slice_h * static_cast<int64_t>(r.a.slice_w / 2 + 1) >= ONESHOT_DIRECT_MIN_PIXELS) {
                const cudaError_t err = launch_extract_pairs(r.a, r.pairs, s);
                if (err != cudaSuccess)
                    return finish_launch(err);
            } else {
                keep.push_back(r);
            }
        }
        h.host_reqs.swap(keep);
        if (h.host_reqs.empty())
            return finish_launch(cudaSuccess);
    }
    bool all_pairs = true;
    for (const BatchReq& r : h.host_reqs)
        all_pairs = all_pairs && r.pairs != nullptr;
    h.key = workload_key(&h);
    Config cfg{0, 0};
    if (all_pairs) {
        // Pair copies everywhere: the lean pairs-only kernel, tile 64 x 16, full occupancy. (The
        // parameter-descriptor kernel is for captured graphs only: launched one-shot from a serving
        // loop, its 28 KB of parameters per launch made the loop's tail latency 5x worse.)
        const KernelFn fn = pairs_only_kernel(h.out_cplx);
        return launch_once(h, fn, 0, max_blocks_per_sm(fn), s);
    }
    {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        load_cache_locked();
        auto it = g_tuned.find(h.key);
        if (it != g_tuned.end())
            cfg = {it->second.first, it->second.second};
    }
    if (cfg.blocks_per_sm <= 0)
        cfg.blocks_per_sm = max_blocks_per_sm(pick_kernel(h.interp, h.in_cplx, h.out_cplx, cfg.variant));
    return launch_once(h, pick_kernel(h.interp, h.in_cplx, h.out_cplx, cfg.variant), cfg.variant,
                       cfg.blocks_per_sm, s);
}

} // extern "C"
