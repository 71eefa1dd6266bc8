/* ORACLE TEST INFRASTRUCTURE — never part of the product path.
 *
 * Plain-C restatement of noa's Fourier central-slice algorithms (noa/xform/FourierProject.hpp and the
 * helpers it calls). It is the parity checker for the CUDA kernels in noa_b200/csrc: only the tests,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
 *
 * Each function has an f32 variant (coordinates, values and weights in float: the precision the
 * reference uses when given Mat33<f32>/Quaternion<f32> rotations) and an f64 variant (the FP64 oracle:
 * the same algorithm with every quantity in double). All pointers are HOST pointers.
 *
 * Parity is pinned against the reference's own CPU path, compiled from its sources into
 * oracle/_ref/libnoa_ref.so (see oracle/Makefile and tests/golden/make_golden.py).
 */
#ifndef NOA_B200_FP_ORACLE_H
#define NOA_B200_FP_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { FPO_REAL = 1, FPO_COMPLEX = 2 };
enum { FPO_NONE = 0, FPO_MAT22 = 1, FPO_MAT33 = 2, FPO_QUAT = 3 };

typedef struct {
    void* data;            /* host pointer; NULL (and is_value == 0) means "absent" (noa's Empty) */
    int32_t dtype;         /* FPO_REAL or FPO_COMPLEX; precision is given by the function suffix */
    int32_t is_value;      /* 1: a single value (value[0] + i value[1]) stands for every element */
    int64_t shape[4];      /* physical BDHW shape (rfft width) */
    int64_t strides[4];    /* strides, in elements */
    double value[2];
} fpo_array;

typedef struct {
    const void* data;      /* host pointer to `count` transforms in noa's layout (Mat33<f32> is 9 floats
                            * padded to 48 bytes, Mat33<f64> 80 bytes); NULL -> use value[] */
    int32_t kind;          /* FPO_NONE (scale only: Empty), FPO_MAT22, FPO_MAT33 or FPO_QUAT */
    int64_t count;         /* 1 = the same transform for every slice */
    double value[9];       /* inline transform when data == NULL (row-major matrix, or z,y,x,w) */
} fpo_transform;

typedef struct {
    int32_t interp;                 /* noa Interp::Method value (0..6, +100 for _FAST) */
    double fftfreq_cutoff;
    int64_t target_shape[4];        /* BDHW; any zero -> use the grid shape */
    double ews_radius[2];
    double fftfreq_sinc;            /* insert: windowed_sinc; insert_and_extract: input_windowed_sinc */
    double fftfreq_blackman;
    double w_fftfreq_sinc;          /* extract and insert_and_extract: w_windowed_sinc */
    double w_fftfreq_blackman;
    int32_t add_to_output;          /* insert_and_extract only */
    int32_t correct_weights;        /* insert_and_extract only */
} fpo_options;

/* remap: noa Layout value, 0=h2h, 8=h2hc, 4=hc2h, 12=hc2hc. Return 0 on success, <0 on bad input. */
#define FPO_DECLARE(NAME, SFX)                                                                     \
    int NAME##SFX(int32_t remap,                                                                   \
                  const fpo_array* input, const fpo_array* input_weight, const int64_t input_shape[4], \
                  const fpo_array* output, const fpo_array* output_weight, const int64_t output_shape[4], \
                  const fpo_transform* scale, const fpo_transform* rotation,                        \
                  const fpo_transform* scale2, const fpo_transform* rotation2,                      \
                  const fpo_options* options, int n_threads)

/* rasterize_central_slices_3d:          scale=inv_scaling, rotation=fwd_rotation (scale2/rotation2 unused)
 * insert_central_slices_3d:             scale=fwd_scaling, rotation=inv_rotation
 * extract_central_slices_3d:            scale=inv_scaling, rotation=fwd_rotation
 * insert_and_extract_central_slices_3d: scale/rotation = input fwd_scaling/inv_rotation,
 *                                       scale2/rotation2 = output inv_scaling/fwd_rotation */
FPO_DECLARE(fpo_rasterize, _f32);
FPO_DECLARE(fpo_rasterize, _f64);
FPO_DECLARE(fpo_insert, _f32);
FPO_DECLARE(fpo_insert, _f64);
FPO_DECLARE(fpo_extract, _f32);
FPO_DECLARE(fpo_extract, _f64);
FPO_DECLARE(fpo_insert_extract, _f32);
FPO_DECLARE(fpo_insert_extract, _f64);

/* fourier_interpolation_correction (FourierProject.hpp:2062-2087; GriddingCorrection :1009-1061):
 * real input and output arrays (`input` may broadcast with zero strides) of the output's BDHW shape;
 * interp must be LINEAR (1 or 101). post_correction != 0 divides by sinc^2(pi r), else multiplies.
 * PARITY UNPINNED: the reference's GriddingCorrection does not compile (FourierProject.hpp:1034 builds
 * `half` with Vec::from_vec(l_shape != 1), but Shape's != yields one bool), no test or caller of it
 * exists, so this restates its documented intent: half = shape / 2 (float), 0 where a size is 1. */
int fpo_gridding_correction_f32(const fpo_array* input, const fpo_array* output, int32_t interp,
                                int32_t post_correction, int n_threads);
int fpo_gridding_correction_f64(const fpo_array* input, const fpo_array* output, int32_t interp,
                                int32_t post_correction, int n_threads);

#ifdef __cplusplus
}
#endif
#endif
