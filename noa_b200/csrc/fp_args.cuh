// Launch arguments shared by the central-slice kernels, and the launchers each .cu file provides.
// The host side (capi.cu) fills one ProjArgs per call with the per-call constants computed exactly as
// the reference's operator constructors do (FourierProject.hpp:199-231, 426-475, 577-609, 790-848).
#pragma once

#include "fp_common.cuh"

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
    float efs, efb;            // w-windowed sinc (extract; insert_extract output)
    int wsize;                 // w-window size (1 = plain 3-D form)
    float vz;                  // insert_extract: the virtual volume's z size
    int add_to_output, correct_weights;

    int in_cplx, out_cplx;     // value kinds (input/output complex?)
    int wide_in;               // input offsets need 64 bits (an array spans >= 2^31 elements)
};

cudaError_t launch_extract(const ProjArgs& a, cudaStream_t stream);
cudaError_t launch_rasterize(const ProjArgs& a, cudaStream_t stream);
cudaError_t launch_insert(const ProjArgs& a, cudaStream_t stream);
cudaError_t launch_insert_extract(const ProjArgs& a, cudaStream_t stream);

// Number of SMs of the current device (cached per device).
int sm_count();

} // namespace nb
