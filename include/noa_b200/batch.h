/* noa_b200 — batched extraction (many extract_central_slices_3d calls in one captured graph or one
 * batched launch) and batched rasterization (many rasterize_central_slices_3d calls in one launch of
 * each kernel).
 *
 * No single function of the reference corresponds to this: it executes a list of
 * extract_central_slices_3d calls (noa/xform/FourierProject.hpp:1869-1914) — different volumes, box
 * sizes and slice counts — as ONE persistent kernel fed by a device work queue, except that large
 * LINEAR requests read through pair copies run as grids of their own beside it; captured once into a
 * CUDA graph and replayed. Every request is validated like nb_extract_central_slices_3d and produces
 * bit-identical results. All requests of a batch share `remap` and `options`; their value types
 * (c32->c32, c32->f32 or f32->f32) must agree; each volume must span fewer than 2^31 elements.
 */
#ifndef NOA_B200_BATCH_H
#define NOA_B200_BATCH_H

#include "noa_b200/fourier_project.h"

#ifdef __cplusplus
extern "C" {
#endif

/* One extraction: the arguments of nb_extract_central_slices_3d. The structs are read during
 * nb_extract_batch_create; the device buffers they point to must stay valid while the batch is used. */
typedef struct {
    const nb_array* volume;
    const nb_array* volume_weight;     /* nullable */
    int64_t volume_shape[4];
    const nb_array* slice;
    const nb_array* slice_weight;      /* nullable */
    int64_t slice_shape[4];
    const nb_transform* inv_scaling;   /* nullable */
    const nb_transform* fwd_rotation;
} nb_extract_request;

typedef struct nb_extract_batch_t* nb_extract_batch;

/* Launch configuration of a batch (tile of pixels per work item, CTAs per SM, grid). */
typedef struct {
    int64_t n_requests;
    int64_t n_items;       /* (slice, tile) work items */
    int32_t tile_h, tile_w;
    int32_t blocks_per_sm;
    int32_t grid;
    double tuned_ms;       /* time of the chosen configuration while autotuning, or -1 */
    int32_t from_cache;    /* 1 if the configuration came from the autotune cache */
    int32_t min_ctas;      /* CTAs per SM the kernel variant was compiled for (its register cap) */
    int32_t n_direct;      /* requests run as grids of their own (see nb_extract_batch_create) */
} nb_batch_info;

/* NB_BATCH_PERSISTENT_ONLY: every request goes through the persistent kernel (no direct grids). */
enum { NB_BATCH_AUTOTUNE = 1, NB_BATCH_PERSISTENT_ONLY = 2 };

/* Validates the requests, uploads their descriptors, chooses the launch configuration (with
 * NB_BATCH_AUTOTUNE: by timing the candidates on this batch, once per workload key, cached in memory and
 * in the text file $NB_AUTOTUNE_CACHE or $HOME/.cache/noa_b200/autotune.txt; autotuning runs the batch,
 * so it writes the outputs) and captures the launch into a CUDA graph. Synchronizes `stream`.
 * LINEAR batches over complex volumes (no scaling, EWS, input weights or w-window) hold a pair copy
 * (16 bytes per rfft voxel) of each volume whose requests read at least twice as many pixels as it
 * has voxels, like the per-call entry point; the graph rebuilds these copies at every run, so changes
 * to the volumes between runs are seen. A request read through a pair copy with at least 2^23 output
 * pixels runs, in the graph, as a grid of its own (the per-call pair kernel) on a parallel branch that
 * starts when its volume's copy is written; the copies of the other volumes are made meanwhile on a
 * higher-priority branch (NB_BATCH_PERSISTENT_ONLY keeps every request in the persistent kernel).
 * Results are bit-identical either way. */
NB_API int nb_extract_batch_create(int32_t remap, const nb_extract_request* requests, int64_t n_requests,
                                   const nb_options* options, int32_t flags, void* stream,
                                   nb_extract_batch* batch);

/* Replays the batch on `stream` (asynchronous). Calls on one batch must not overlap on the GPU. While
 * `stream` is being captured into a caller's graph, the batch's launch sequence is issued into that
 * capture. (nb_extract_batch_create itself synchronizes: inside a capture it returns NB_ERROR_INVALID.) */
NB_API int nb_extract_batch_run(nb_extract_batch batch, void* stream);

NB_API int nb_extract_batch_info(nb_extract_batch batch, nb_batch_info* info);

/* ---- Resident volumes and one-shot batched launches (used by serving loops) ----------------------- */

/* Pair copy of a volume for LINEAR extraction: element (z, y, x) holds the x-neighbours v[z][y][x] and
 * v[z][y][x+1] as 16 bytes, so a trilinear cell is four aligned loads. Results read through it are
 * bit-identical to reading the volume. nb_volume_pairs_bytes gives its size (-1 for a bad shape);
 * nb_volume_pairs writes it (`volume`: one c32 rfft volume, `volume_shape` {1, D, H, W}). */
NB_API int64_t nb_volume_pairs_bytes(const int64_t volume_shape[4]);
NB_API int nb_volume_pairs(const nb_array* volume, const int64_t volume_shape[4], void* pairs,
                           int64_t pairs_bytes, void* stream);

/* An extraction with, optionally, the pair copy of its volume. The copy is used where it applies
 * (LINEAR, complex volume, no volume weights, no EWS, no scaling, no w-window) and ignored otherwise. */
typedef struct {
    nb_extract_request call;
    const void* volume_pairs;          /* nullable */
    int64_t volume_pairs_bytes;
} nb_extract_request_ex;

/* Validates the requests and enqueues them on `stream` (no graph, no autotuning: the configuration
 * cached for the workload key is used when there is one, else a default): each request read through
 * its pair copy with at least 2^21 output pixels as a grid of its own (the per-call pair kernel), the
 * others as ONE persistent launch, its descriptors staged in stream-ordered device memory. The request
 * structs may be freed on return; the device buffers must stay valid until the launches complete.
 * Results are bit-identical to nb_extract_central_slices_3d on each request. */
NB_API int nb_extract_batch_launch(int32_t remap, const nb_extract_request_ex* requests, int64_t n_requests,
                                   const nb_options* options, void* stream);

/* nb_extract_batch_launch with flags: NB_BATCH_PERSISTENT_ONLY sends every request through the
 * persistent launch. */
NB_API int nb_extract_batch_launch_ex(int32_t remap, const nb_extract_request_ex* requests, int64_t n_requests,
                                      const nb_options* options, int32_t flags, void* stream);

NB_API int nb_extract_batch_destroy(nb_extract_batch batch);

/* ---- Batched rasterization (used by serving loops) ------------------------------------------------ */

/* One rasterization: the arguments of nb_rasterize_central_slices_3d. */
typedef struct {
    const nb_array* slice;
    const nb_array* slice_weight;      /* nullable */
    int64_t slice_shape[4];
    const nb_array* volume;
    const nb_array* volume_weight;     /* nullable */
    int64_t volume_shape[4];
    const nb_transform* inv_scaling;   /* nullable */
    const nb_transform* fwd_rotation;
} nb_rasterize_request;

/* No counterpart in the reference: a list of rasterize_central_slices_3d calls
 * (FourierProject.hpp:1653-1692), each into its own grids, enqueued on `stream` as ONE scatter launch and
 * ONE finalize launch instead of a launch sequence per call. Each request is validated like
 * nb_rasterize_central_slices_3d and sums the same terms (the order of the atomic additions may differ,
 * as between two per-call runs). All requests share `remap` and `options`, their value types and the
 * presence of output weights; their output grids must not overlap (NB_ERROR_INVALID otherwise). The
 * accumulators of all requests come from one stream-ordered allocation (NB_ERROR_OOM without it). The
 * request structs may be freed on return; the device buffers must stay valid until the work completes. */
NB_API int nb_rasterize_batch_launch(int32_t remap, const nb_rasterize_request* requests, int64_t n_requests,
                                     const nb_options* options, void* stream);

#ifdef __cplusplus
}
#endif
#endif
