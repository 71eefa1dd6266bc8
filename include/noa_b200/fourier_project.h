/* noa_b200 — B200-native (sm_100a) Fourier central-slice extraction and insertion.
 *
 * C ABI of the drop-in. Each entry point replaces the GPU branch of one noa function template in
 * noa/xform/FourierProject.hpp (the `details::launch_*<REMAP, i32, true>` call inside
 * `#ifdef NOA_ENABLE_GPU`), keeping its argument meaning, layouts and results:
 *
 *   nb_rasterize_central_slices_3d            <- rasterize_central_slices_3d            FourierProject.hpp:1653-1692 (GPU branch :1675-1685)
 *   nb_insert_central_slices_3d               <- insert_central_slices_3d               FourierProject.hpp:1770-1815 (GPU branch :1792-1808)
 *   nb_extract_central_slices_3d              <- extract_central_slices_3d              FourierProject.hpp:1869-1914 (GPU branch :1891-1907)
 *   nb_insert_and_extract_central_slices_3d   <- insert_and_extract_central_slices_3d   FourierProject.hpp:1987-2049 (GPU branch :2022-2041)
 *
 * All array and transform pointers are DEVICE pointers on the current CUDA device. Calls are
 * asynchronous on `stream` (a cudaStream_t; NULL = the legacy default stream). Return values are
 * NB_OK or a negative NB_ERROR_*; nb_last_error() then describes the failure (thread-local). No kernel
 * traps: invalid arguments are rejected on the host before any launch.
 */
#ifndef NOA_B200_FOURIER_PROJECT_H
#define NOA_B200_FOURIER_PROJECT_H

#include <stdint.h>

#if defined(__GNUC__)
#define NB_API __attribute__((visibility("default")))
#else
#define NB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

enum {
    NB_OK = 0,
    NB_ERROR_INVALID = -1,      /* bad argument (shape, stride, overlap, option): noa's check() failures */
    NB_ERROR_UNSUPPORTED = -2,  /* valid for noa but not provided here (f64/c64 values, textures) */
    NB_ERROR_CUDA = -3,         /* a CUDA runtime call failed */
    NB_ERROR_OOM = -4,          /* a scratch or device allocation failed */
    NB_ERROR_TIMEOUT = -5       /* reserved: no kernel of this library waits on the device, so none returns it */
};

/* noa::fft::Layout values of the four hx2hx remaps (fft/core/Layout.hpp:48-55). */
enum { NB_REMAP_H2H = 0, NB_REMAP_H2HC = 8, NB_REMAP_HC2H = 4, NB_REMAP_HC2HC = 12 };

/* noa::xform::Interp::Method values (xform/core/Interp.hpp:16-40). The _FAST variants (value + 100)
 * only differ from the accurate ones for texture inputs, which this library does not take. */
enum {
    NB_INTERP_NEAREST = 0, NB_INTERP_LINEAR = 1, NB_INTERP_CUBIC = 2, NB_INTERP_CUBIC_BSPLINE = 3,
    NB_INTERP_LANCZOS4 = 4, NB_INTERP_LANCZOS6 = 5, NB_INTERP_LANCZOS8 = 6
};

enum { NB_DTYPE_F32 = 1, NB_DTYPE_C32 = 2, NB_DTYPE_F64 = 3, NB_DTYPE_C64 = 4 };

/* Transform kinds, in noa's memory layout: Mat22<f32> is 4 floats (16 bytes), Mat33<f32> is 9 floats
 * row-major padded to 48 bytes (alignas 16), Quaternion<f32> is z,y,x,w (16 bytes). */
enum { NB_XFORM_NONE = 0, NB_XFORM_MAT22_F32 = 1, NB_XFORM_MAT33_F32 = 2, NB_XFORM_QUAT_F32 = 3 };

/* An array argument: noa's View/Array reduced to pointer, physical BDHW shape and element strides. */
typedef struct {
    void* data;             /* device pointer; NULL with is_value == 0 means "absent" (noa's Empty) */
    int32_t dtype;          /* NB_DTYPE_* */
    int32_t is_value;       /* 1: a single value (value[0] + i*value[1]) stands for every element */
    int64_t shape[4];       /* physical shape, i.e. the logical shape's .rfft() */
    int64_t strides[4];     /* strides in elements (any sign-free layout; 0 broadcasts) */
    double value[2];
} nb_array;

/* A per-slice transform argument: a single value (data == NULL, count == 1) or a contiguous array. */
typedef struct {
    const void* data;       /* device pointer to `count` transforms, or NULL to use value[] */
    int32_t kind;           /* NB_XFORM_*; NB_XFORM_NONE is only valid for scalings (noa's Empty) */
    int64_t count;          /* 1 = the same transform for every slice, else the number of slices */
    double value[9];        /* inline transform: Mat22 row-major (4), Mat33 row-major (9), quaternion z,y,x,w */
} nb_transform;

/* Union of noa's option structs (FourierProject.hpp:1602-1627, 1703-1739, 1817-1838, 1916-1951). */
typedef struct {
    int32_t interp;             /* NB_INTERP_* (+100 accepted); ignored by rasterize */
    double fftfreq_cutoff;      /* default 0.5 */
    int64_t target_shape[4];    /* BDHW; any zero element -> the grid shape (noa's default {}) */
    double ews_radius[2];       /* HW Ewald sphere radius; {0,0} -> no curvature */
    double fftfreq_sinc;        /* insert: windowed_sinc; insert_and_extract: input_windowed_sinc (default -1) */
    double fftfreq_blackman;    /* (default -1) */
    double w_fftfreq_sinc;      /* extract / insert_and_extract: w_windowed_sinc (default -1) */
    double w_fftfreq_blackman;  /* (default -1) */
    int32_t add_to_output;      /* insert_and_extract only */
    int32_t correct_weights;    /* insert_and_extract only */
} nb_options;

/* Fills `o` with noa's defaults (LINEAR, cutoff 0.5, no target, no EWS, windowed-sinc {-1,-1}). */
NB_API void nb_options_default(nb_options* o);

/* rasterize_central_slices_3d: trilinear scatter of 2-D rfft slices into a 3-D rfft volume (+=).
 * slice: B x 1 x H x W/2+1 (f32|c32, or a constant value); volume: 1 x D x H x W/2+1 (f32|c32);
 * weights are f32 or absent. inv_scaling: Mat22 or NONE; fwd_rotation: Mat33 or quaternion. */
NB_API int nb_rasterize_central_slices_3d(
    int32_t remap,
    const nb_array* slice, const nb_array* slice_weight, const int64_t slice_shape[4],
    const nb_array* volume, const nb_array* volume_weight, const int64_t volume_shape[4],
    const nb_transform* inv_scaling, const nb_transform* fwd_rotation,
    const nb_options* options, void* stream);

/* insert_central_slices_3d: windowed-sinc gather insertion, one output voxel at a time (+=).
 * fwd_scaling: Mat22 or NONE; inv_rotation: Mat33 or quaternion. Deterministic. */
NB_API int nb_insert_central_slices_3d(
    int32_t remap,
    const nb_array* slice, const nb_array* slice_weight, const int64_t slice_shape[4],
    const nb_array* volume, const nb_array* volume_weight, const int64_t volume_shape[4],
    const nb_transform* fwd_scaling, const nb_transform* inv_rotation,
    const nb_options* options, void* stream);

/* Slice-major scatter form of nb_insert_central_slices_3d (no counterpart in the reference): the same
 * per-(voxel, slice) terms — same windowed sinc, same 2-D interpolation, same cutoff — but each slice
 * visits the voxels of its slab |fz| <= fftfreq_blackman and adds its terms with atomics, so the sum
 * over slices is in an unspecified order (results match the gather form to float rounding, not
 * bit-exactly). Needs a dense accumulator of the volume (16 bytes per rfft voxel with weights) from the
 * library's stream-ordered pool; with an Ewald-sphere curvature, or without that memory, it runs the
 * gather form. Same arguments and errors as nb_insert_central_slices_3d. */
NB_API int nb_insert_central_slices_3d_scatter(
    int32_t remap,
    const nb_array* slice, const nb_array* slice_weight, const int64_t slice_shape[4],
    const nb_array* volume, const nb_array* volume_weight, const int64_t volume_shape[4],
    const nb_transform* fwd_scaling, const nb_transform* inv_rotation,
    const nb_options* options, void* stream);

/* fourier_interpolation_correction (FourierProject.hpp:2062-2087): real-space correction of the LINEAR
 * gridding kernel, output = input / sinc^2(pi r) (post_correction != 0) or input * sinc^2(pi r), r the
 * distance of each voxel from the center (shape / 2) in units of the shape. Real f32 arrays; the input
 * may broadcast (size-1 dimensions) or be a constant, and may be the output (in place). interp must be
 * NB_INTERP_LINEAR (or its _FAST alias), else NB_ERROR_INVALID, as in the reference. */
NB_API int nb_fourier_interpolation_correction(const nb_array* input, const nb_array* output, int32_t interp,
                                               int32_t post_correction, void* stream);

/* Reconstruction spectrum pass (no counterpart in the reference): output = values / max(weights,
 * weight_threshold) (no division when weights is NULL), remapped from the inserted layout (centered = 1:
 * "hc", 0: "h") to the non-centered layout a c2r FFT reads, times exp(-2 pi i k.c / n) with c = n / 2,
 * so that the c2r's real-space origin lands at the volume's center (where nb_fourier_interpolation_correction
 * puts it). One volume, `volume_shape` {1, D, H, W}; output contiguous c32 and not overlapping the inputs. */
NB_API int nb_reconstruction_spectrum(const nb_array* values, const nb_array* weights, const int64_t volume_shape[4],
                                      int32_t centered, double weight_threshold, const nb_array* output,
                                      void* stream);

/* extract_central_slices_3d: 3-D spectrum interpolation at every pixel of every output slice (=). */
NB_API int nb_extract_central_slices_3d(
    int32_t remap,
    const nb_array* volume, const nb_array* volume_weight, const int64_t volume_shape[4],
    const nb_array* slice, const nb_array* slice_weight, const int64_t slice_shape[4],
    const nb_transform* inv_scaling, const nb_transform* fwd_rotation,
    const nb_options* options, void* stream);

/* insert_and_extract_central_slices_3d: extraction from the virtual volume of the input slices. */
NB_API int nb_insert_and_extract_central_slices_3d(
    int32_t remap,
    const nb_array* input_slice, const nb_array* input_weight, const int64_t input_slice_shape[4],
    const nb_array* output_slice, const nb_array* output_weight, const int64_t output_slice_shape[4],
    const nb_transform* input_fwd_scaling, const nb_transform* input_inv_rotation,
    const nb_transform* output_inv_scaling, const nb_transform* output_fwd_rotation,
    const nb_options* options, void* stream);

/* No counterpart in the reference. Same arguments, checks and results as
 * nb_rasterize_central_slices_3d, but the call allocates no device memory: for callers that cannot let
 * a library allocate at call time (a fixed up-front memory budget, an allocator owned by someone else,
 * a steady state that must not enter the driver's allocator). With output weights, the (value, weight)
 * accumulator lives in a 64 MiB array of this library's device code. CUDA reserves it on a GPU when it
 * loads that code there: by default (lazy module loading) during the first call on that GPU, or when the
 * library loads under CUDA_MODULE_LOADING=EAGER; it is then held until exit. So make one warm-up call
 * per GPU while setting up a memory budget (and before any stream capture: the first call also looks
 * the array's address up); the calls after it allocate nothing. The rfft grid D*H*(W/2+1) may hold at
 * most 4,194,304 voxels for complex values (8,388,608 for real ones); larger volumes return
 * NB_ERROR_INVALID. All calls share the array and each clears the part it uses first: calls that
 * overlap on the GPU race, so order them. */
NB_API int nb_rasterize_central_slices_3d_static_scratch(
    int32_t remap,
    const nb_array* slice, const nb_array* slice_weight, const int64_t slice_shape[4],
    const nb_array* volume, const nb_array* volume_weight, const int64_t volume_shape[4],
    const nb_transform* inv_scaling, const nb_transform* fwd_rotation,
    const nb_options* options, void* stream);

/* No counterpart in the reference (noa's Array allocations are the caller's). Caps the size of any
 * ONE device allocation this library makes on its own behalf on CUDA device `device`: the per-call
 * scratch of the fast paths (the pair copy of a LINEAR extraction, 16 bytes per rfft voxel; the padded
 * accumulator of a rasterization or scatter insertion, up to 16 bytes per voxel of the grid padded to
 * the cutoff; a one-shot batched launch's descriptors) and a captured batch's descriptors and pair
 * copies. An allocation above the cap fails as if the device were out of memory, so calls take their
 * path without it, with the same results: extraction reads the volume directly, rasterization reduces
 * into an unpadded scratch or straight into the caller's grids, the scatter insertion runs the gather
 * form; a batch whose descriptors cannot be allocated returns NB_ERROR_OOM. bytes < 0 removes the cap
 * (the default); 0 makes every call take its path without scratch. Applies to calls made after it
 * returns, from any thread. NB_ERROR_INVALID for a device that does not exist. */
NB_API int nb_set_scratch_limit(int32_t device, int64_t bytes);

/* The cap set on `device` in bytes, -1 when there is none (or the device does not exist). */
NB_API int64_t nb_scratch_limit(int32_t device);

/* How many of the library's own allocations on `device` were refused since it loaded (above the cap,
 * or the device out of memory): each sent a call down its path without that memory (same results,
 * slower) or, for batch descriptors, to NB_ERROR_OOM. A caller that expects the fast paths reads it
 * before and after its calls. -1 for a bad device index. No counterpart in noa. */
NB_API int64_t nb_scratch_refusals(int32_t device);

/* Description of the last error on the calling thread ("" if none). */
NB_API const char* nb_last_error(void);

/* Library version, "major.minor.patch". */
NB_API const char* nb_version(void);

#ifdef __cplusplus
}
#endif
#endif
