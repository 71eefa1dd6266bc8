// Launch arguments shared by the central-slice kernels, and the launchers each .cu file provides.
// The host side (capi.cu) fills one ProjArgs per call with the per-call constants computed exactly as
// the reference's operator constructors do (FourierProject.hpp:199-231, 426-475, 577-609, 790-848).
#pragma once

#include "fp_common.cuh"
#include "noa_b200/fourier_project.h"

namespace nb {

struct ProjArgs {
    SrcView in, in_w;          // volume (extract) or input slices (the others)
    DstView out, out_w;        // slices (extract, insert_extract) or volume (rasterize, insert)
    XformView scale, rot;      // rasterize/extract: inv_scaling, fwd_rotation; insert: fwd_scaling, inv_rotation;
                               // insert_extract: input fwd_scaling, input inv_rotation
    XformView scale2, rot2;    // insert_extract: output inv_scaling, output fwd_rotation
    Ews ews;

    // Logical geometry. Slices: (count, h, w); volume: (d, h, w). rfft widths are w/2+1.
    int64_t n_slices;          // slices iterated per launch (input or output, depending on the op)
    int64_t n_in;              // insert_extract: number of input slices
    int slice_h, slice_w;      // logical slice size of the iterated slices
    int in_h, in_w_;           // insert_extract: logical size of the input slices
    int vol_d, vol_h, vol_w;   // logical volume size
    bool in_centered, out_centered;
    int interp;                // interpolation family, 0..6

    float f_slice0, f_slice1;  // float(slice_h), float(slice_w) of the iterated slices
    float f_in0, f_in1;        // insert_extract: float sizes of the input slices
    float target0, target1, target2;
    float cutoff_sqd;
    float fs, fb;              // windowed sinc (insert; insert_extract input)
    float pfs, pfb;            // pi / fs, pi / fb (for windowed_sinc_fast)
    float ifs;                 // 1 / fs (the sinc phase in units of pi, for sinpif)
    float efs, efb;            // w-windowed sinc (extract; insert_extract output)
    int wsize;                 // w-window size (1 = plain 3-D form)
    float vz;                  // insert_extract: the virtual volume's z size
    int add_to_output, correct_weights;

    int in_cplx, out_cplx;     // value kinds (input/output complex?)
    int wide_in;               // input offsets need 64 bits (an array spans >= 2^31 elements)
    int in_slice_narrow;       // offsets within one input slice fit 32 bits
};

cudaError_t launch_extract(const ProjArgs& a, cudaStream_t stream);
cudaError_t launch_rasterize(const ProjArgs& a, cudaStream_t stream);
cudaError_t launch_insert(const ProjArgs& a, cudaStream_t stream);
cudaError_t launch_insert_extract(const ProjArgs& a, cudaStream_t stream);
cudaError_t launch_insert_scatter(const ProjArgs& a, cudaStream_t stream);
// The reconstruction's spectrum pass (fp_reconstruct.cu) on checked arrays.
cudaError_t launch_reconstruction_spectrum(const nb_array* values, const nb_array* weights,
                                           const int64_t shape[4], bool centered, float threshold,
                                           const nb_array* out, cudaStream_t stream);
// fourier_interpolation_correction on checked real f32 arrays (capi.cu checks them).
cudaError_t launch_gridding_correction(const nb_array* input, const nb_array* output, bool post,
                                       cudaStream_t stream);

// Argument checks and per-call constants of nb_rasterize_central_slices_3d (capi.cu); fills `a` and
// returns NB_OK, or an NB_ERROR_* code with the thread's last-error message set.
int prepare_rasterize(int32_t remap,
                      const nb_array* slice, const nb_array* slice_weight, const int64_t slice_shape[4],
                      const nb_array* volume, const nb_array* volume_weight, const int64_t volume_shape[4],
                      const nb_transform* inv_scaling, const nb_transform* fwd_rotation,
                      const nb_options* options, ProjArgs& a);
// Same for nb_insert_central_slices_3d (and its scatter form).
int prepare_insert(int32_t remap,
                   const nb_array* slice, const nb_array* slice_weight, const int64_t slice_shape[4],
                   const nb_array* volume, const nb_array* volume_weight, const int64_t volume_shape[4],
                   const nb_transform* fwd_scaling, const nb_transform* inv_rotation,
                   const nb_options* options, ProjArgs& a);
// Same for nb_extract_central_slices_3d.
int prepare_extract(int32_t remap,
                    const nb_array* volume, const nb_array* volume_weight, const int64_t volume_shape[4],
                    const nb_array* slice, const nb_array* slice_weight, const int64_t slice_shape[4],
                    const nb_transform* inv_scaling, const nb_transform* fwd_rotation,
                    const nb_options* options, ProjArgs& a);
// Checks a caller's pair copy (nb_volume_pairs) of the volume of `a`: NB_OK or NB_ERROR_INVALID.
int check_pairs(const void* pairs, int64_t bytes, const ProjArgs& a, const char* name);
// NB_OK (clearing the thread's last error) or NB_ERROR_CUDA with the launch error's description.
int finish_launch(cudaError_t err);
// Sets the thread's last error and returns `code`.
int report_error(int code, const char* message);

// Number of SMs of the current device (cached per device).
int sm_count();

} // namespace nb
