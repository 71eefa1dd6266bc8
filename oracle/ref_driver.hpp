// ORACLE TEST INFRASTRUCTURE — not part of the product.
//
// C-ABI driver around the reference's own CPU implementation of the Fourier central-slice path
// (noa/xform/FourierProject.hpp). It is compiled, together with a few of the reference's .cpp files,
// into oracle/_ref/libnoa_ref.so by oracle/Makefile. Tests and the bench's reference arm use it to
// (1) pin the C restatement in oracle/fp_oracle.c and (2) time noa's CPU (OpenMP) path.
//
// Every entry point wraps plain host pointers into noa Views on the "cpu" device and calls the public
// templates unchanged:
//   rasterize_central_slices_3d           FourierProject.hpp:1653-1692
//   insert_central_slices_3d              FourierProject.hpp:1770-1815
//   extract_central_slices_3d             FourierProject.hpp:1869-1914
//   insert_and_extract_central_slices_3d  FourierProject.hpp:1987-2049
#pragma once

#include <cstdint>

extern "C" {
    // One array argument: host pointer (NULL = absent/Empty), physical BDHW shape, element strides.
    typedef struct {
        void* ptr;
        int64_t shape[4];
        int64_t strides[4];
    } noaref_array;

    typedef struct {
        int32_t remap;              // noa Layout: 0=h2h, 8=h2hc, 4=hc2h, 12=hc2hc
        int32_t interp;             // noa Interp::Method value
        double fftfreq_cutoff;
        int64_t target_shape[4];
        double ews_radius[2];
        double sinc[2];             // windowed_sinc (insert) or input_windowed_sinc (insert_and_extract)
        double w_sinc[2];           // w_windowed_sinc (extract and insert_and_extract)
        int32_t add_to_output;
        int32_t correct_weights;
    } noaref_options;

    // Value combinations: input→output element types.
    enum { NOAREF_C32C32 = 0, NOAREF_F32F32 = 1, NOAREF_C32F32 = 2, NOAREF_C64C64 = 3, NOAREF_F64F64 = 4 };
    // Rotation kinds: Mat33 (9 values, row-major DHW) or Quaternion (z,y,x,w). Precision follows the combo.
    enum { NOAREF_MAT33 = 0, NOAREF_QUAT = 1 };
}

#define NOAREF_DECLARE(NAME)                                                                        \
    extern "C" int NAME(                                                                            \
        const noaref_array* in, const noaref_array* in_w, const int64_t in_shape[4],                \
        const noaref_array* out, const noaref_array* out_w, const int64_t out_shape[4],             \
        const void* scale0, const void* rot0, const void* scale1, const void* rot1, int rot_kind,   \
        const noaref_options* opt, int n_threads, char* err, int errlen)
