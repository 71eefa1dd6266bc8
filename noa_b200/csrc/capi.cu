// C ABI of noa_b200 (include/noa_b200/fourier_project.h): argument checks, per-call constants and
// kernel dispatch.
//
// The checks restate noa's fourier_projection_check_parameters (noa/xform/FourierProject.hpp:1100-1185)
// and the correct_weights check of insert_and_extract_central_slices_3d (:2013-2020), so a call the
// reference rejects is rejected here with NB_ERROR_INVALID. The constants restate the operator
// constructors (FourierProject.hpp:199-231, 426-475, 577-609, 790-848), computed in float like the
// reference's f32 coordinate type.
#include "fp_args.cuh"
#include "fp_pairs.cuh"
#include "fp_pool.cuh"

#include "noa_b200/batch.h"
#include "noa_b200/fourier_project.h"

#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <string>

namespace nb {

int sm_count() {
    // Filled on first use per device; concurrent first calls store the same value.
    static std::atomic<int> counts[64];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64)
        dev = 0;
    int n = counts[dev].load(std::memory_order_relaxed);
    if (n == 0) {
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        n = n > 0 ? n : 148;
        counts[dev].store(n, std::memory_order_relaxed);
    }
    return n;
}

namespace {

thread_local std::string g_last_error;

int fail(int code, const char* fmt, ...) {
    char buf[1024];
    va_list args;
    va_start(args, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, args);
    va_end(args);
    g_last_error = buf;
    return code;
}

bool is_complex(int32_t dt) { return dt == NB_DTYPE_C32 || dt == NB_DTYPE_C64; }
bool is_f64(int32_t dt) { return dt == NB_DTYPE_F64 || dt == NB_DTYPE_C64; }
int64_t elem_size(int32_t dt) { return dt == NB_DTYPE_F32 ? 4 : dt == NB_DTYPE_C32 ? 8 : dt == NB_DTYPE_F64 ? 8 : 16; }

bool present(const nb_array* a) { return a && (a->data || a->is_value); }
bool is_array(const nb_array* a) { return a && a->data && !a->is_value; }

void rfft_shape(const int64_t logical[4], int64_t out[4]) {
    out[0] = logical[0];
    out[1] = logical[1];
    out[2] = logical[2];
    out[3] = logical[3] / 2 + 1;
}

bool shape_eq(const int64_t a[4], const int64_t b[4]) {
    return a[0] == b[0] && a[1] == b[1] && a[2] == b[2] && a[3] == b[3];
}

// Byte range [lo, hi) spanned by an array (noa's are_overlapped, runtime/Utils.hpp).
void byte_range(const nb_array* a, uintptr_t& lo, uintptr_t& hi) {
    int64_t lo_e = 0, hi_e = 0;
    for (int i = 0; i < 4; ++i) {
        const int64_t extent = (a->shape[i] - 1) * a->strides[i];
        if (extent < 0)
            lo_e += extent;
        else
            hi_e += extent;
    }
    const int64_t es = elem_size(a->dtype);
    lo = reinterpret_cast<uintptr_t>(a->data) + static_cast<uintptr_t>(lo_e * es);
    hi = reinterpret_cast<uintptr_t>(a->data) + static_cast<uintptr_t>((hi_e + 1) * es);
}

bool overlap(const nb_array* a, const nb_array* b) {
    if (!is_array(a) || !is_array(b))
        return false;
    uintptr_t alo, ahi, blo, bhi;
    byte_range(a, alo, ahi);
    byte_range(b, blo, bhi);
    return alo < bhi && blo < ahi;
}

int check_device_pointer(const void* p, const char* name, int device) {
    cudaPointerAttributes attr{};
    const cudaError_t err = cudaPointerGetAttributes(&attr, p);
    if (err != cudaSuccess) {
        cudaGetLastError();
        return fail(NB_ERROR_INVALID, "%s: not a CUDA pointer (%s)", name, cudaGetErrorString(err));
    }
    if (attr.type != cudaMemoryTypeDevice && attr.type != cudaMemoryTypeManaged)
        return fail(NB_ERROR_INVALID, "%s: expected device or managed memory", name);
    if (attr.type == cudaMemoryTypeDevice && attr.device != device)
        return fail(NB_ERROR_INVALID,
                    "The arrays should be on the same device, but got %s:device=gpu:%d and the compute device gpu:%d",
                    name, attr.device, device);
    return NB_OK;
}

int check_array(const nb_array* a, const int64_t logical[4], const char* name, bool weight, int device) {
    if (!present(a))
        return NB_OK;
    if (a->dtype < NB_DTYPE_F32 || a->dtype > NB_DTYPE_C64)
        return fail(NB_ERROR_INVALID, "%s: unknown dtype %d", name, a->dtype);
    if (weight && is_complex(a->dtype))
        return fail(NB_ERROR_INVALID, "%s: weights should be real", name);
    if (is_f64(a->dtype))
        return fail(NB_ERROR_UNSUPPORTED, "%s: f64/c64 values are not provided on the GPU by this library", name);
    if (a->is_value)
        return NB_OK;
    int64_t expected[4];
    rfft_shape(logical, expected);
    if (!shape_eq(a->shape, expected))
        return fail(NB_ERROR_INVALID,
                    "The shape of the rfft does not match the expected shape. Got %s:shape={%lld,%lld,%lld,%lld} "
                    "and shape={%lld,%lld,%lld,%lld}", name,
                    (long long) a->shape[0], (long long) a->shape[1], (long long) a->shape[2], (long long) a->shape[3],
                    (long long) expected[0], (long long) expected[1], (long long) expected[2], (long long) expected[3]);
    for (int i = 0; i < 4; ++i) {
        if (a->shape[i] <= 0)
            return fail(NB_ERROR_INVALID, "Empty array detected (%s)", name);
        if (a->strides[i] < 0)
            return fail(NB_ERROR_INVALID, "%s: negative strides are not supported", name);
    }
    if (reinterpret_cast<uintptr_t>(a->data) % static_cast<uintptr_t>(elem_size(a->dtype) == 8 ? 8 : 4))
        return fail(NB_ERROR_INVALID, "%s: misaligned data pointer", name);
    return check_device_pointer(a->data, name, device);
}

int check_transform(const nb_transform* t, int64_t required, bool rotation, const char* name, int device) {
    if (!t) {
        if (rotation)
            return fail(NB_ERROR_INVALID, "%s should not be empty", name);
        return NB_OK;
    }
    if (rotation && t->kind != NB_XFORM_MAT33_F32 && t->kind != NB_XFORM_QUAT_F32)
        return fail(NB_ERROR_INVALID, "%s: expected Mat33<f32> or Quaternion<f32>", name);
    if (!rotation && t->kind != NB_XFORM_NONE && t->kind != NB_XFORM_MAT22_F32)
        return fail(NB_ERROR_INVALID, "%s: expected Mat22<f32> or Empty", name);
    if (t->kind == NB_XFORM_NONE || !t->data)
        return NB_OK;
    if (t->count != required && t->count != 1)
        return fail(NB_ERROR_INVALID,
                    "%s should be a contiguous vector with n_slices=%lld elements, but got %lld",
                    name, (long long) required, (long long) t->count);
    if (reinterpret_cast<uintptr_t>(t->data) % 16)
        return fail(NB_ERROR_INVALID, "%s: transforms should be 16-byte aligned (noa's layout)", name);
    return check_device_pointer(t->data, name, device);
}

SrcView make_src(const nb_array* a, int dim0) {
    SrcView s{};
    if (!present(a))
        return s;
    s.present = 1;
    s.is_value = a->is_value;
    s.value = make_float2(static_cast<float>(a->value[0]), is_complex(a->dtype) ? static_cast<float>(a->value[1]) : 0.f);
    s.data = a->data;
    s.s0 = a->is_value ? 0 : a->strides[dim0];
    s.s1 = a->is_value ? 0 : a->strides[2];
    s.s2 = a->is_value ? 0 : a->strides[3];
    return s;
}

DstView make_dst(const nb_array* a, int dim0) {
    DstView d{};
    if (!is_array(a))
        return d;
    d.present = 1;
    d.data = a->data;
    d.s0 = a->strides[dim0];
    d.s1 = a->strides[2];
    d.s2 = a->strides[3];
    return d;
}

XformView make_xform(const nb_transform* t) {
    XformView x{};
    if (!t)
        return x;
    x.kind = t->kind == NB_XFORM_MAT22_F32 ? 1 : t->kind == NB_XFORM_MAT33_F32 ? 2 : t->kind == NB_XFORM_QUAT_F32 ? 3 : 0;
    x.data = static_cast<const float*>(t->data);
    x.count = t->data ? t->count : 1;
    for (int i = 0; i < 9; ++i)
        x.inline_value[i] = static_cast<float>(t->value[i]);
    return x;
}

Ews make_ews(const double r[2]) {
    Ews e{};
    e.on = r[0] != 0 || r[1] != 0;
    const float r0 = static_cast<float>(r[0]), r1 = static_cast<float>(r[1]);
    if (r0 != 0.f || r1 != 0.f) {
        e.d0 = 1.f / (2.f * r0);
        e.d1 = 1.f / (2.f * r1);
    }
    return e;
}

float fmax_ref(float a, float b) { return a < b ? b : a; }

// Whether offsets within one slice (dimensions 2 and 3) of an array fit 31 bits.
bool slice_narrow(const nb_array* a) {
    if (!is_array(a))
        return false;
    const int64_t extent = (a->shape[2] - 1) * a->strides[2] + (a->shape[3] - 1) * a->strides[3];
    return extent < (int64_t(1) << 31) - 1 && a->strides[2] < (int64_t(1) << 31) && a->strides[3] < (int64_t(1) << 31);
}

// Whether an array's largest element offset needs more than 31 bits.
bool needs_wide(const nb_array* a) {
    if (!is_array(a))
        return false;
    int64_t extent = 0;
    for (int i = 0; i < 4; ++i)
        extent += (a->shape[i] - 1) * a->strides[i];
    return extent >= (int64_t(1) << 31) - 1;
}

// blackman_window_size (FourierProject.hpp:114-137).
int blackman_window_size(float fftfreq_blackman, float spectrum_size) {
    double samples = static_cast<double>(spectrum_size) * static_cast<double>(fftfreq_blackman);
    const double diff = std::fabs(samples - 1.);
    const bool close = std::isfinite(diff) &&
                       (diff <= 1e-6 || diff <= std::fmax(std::fabs(samples), 1.) * (2.220446049250313e-16 * 2));
    samples = close ? std::round(samples) : std::ceil(samples);
    int64_t n = static_cast<int64_t>(samples);
    if (n < 1)
        n = 1;
    return static_cast<int>(2 * n + 1 - 2);
}

void target3(const nb_options* o, const int64_t grid4[4], float t[3]) {
    const int64_t* ts = o->target_shape;
    const bool any0 = ts[0] == 0 || ts[1] == 0 || ts[2] == 0 || ts[3] == 0;
    for (int i = 0; i < 3; ++i)
        t[i] = static_cast<float>(any0 ? grid4[i + 1] : ts[i + 1]);
}

float cutoff_sqd(const nb_options* o) {
    float c = static_cast<float>(o->fftfreq_cutoff);
    c = fmax_ref(c, 0.f);
    return c * c;
}

int interp_family(int32_t interp) {
    const int m = interp >= 100 ? interp - 100 : interp;
    return (m >= 0 && m <= 6) ? m : -1;
}

enum class Op { RASTERIZE, INSERT, EXTRACT, INSERT_EXTRACT };

int common_checks(Op op, int32_t remap, const nb_array* in, const nb_array* in_w, const int64_t in_shape[4],
                  const nb_array* out, const nb_array* out_w, const int64_t out_shape[4],
                  const nb_options* o, int& device) {
    if (!o)
        return fail(NB_ERROR_INVALID, "options should not be NULL");
    if (remap != NB_REMAP_H2H && remap != NB_REMAP_H2HC && remap != NB_REMAP_HC2H && remap != NB_REMAP_HC2HC)
        return fail(NB_ERROR_INVALID, "remap should be one of h2h, h2hc, hc2h, hc2hc (got %d)", remap);
    if (!in_shape || !out_shape)
        return fail(NB_ERROR_INVALID, "shapes should not be NULL");
    for (int i = 0; i < 4; ++i) {
        if (in_shape[i] <= 0 || out_shape[i] <= 0)
            return fail(NB_ERROR_INVALID, "Empty array detected (logical shapes should be positive)");
    }
    if (op != Op::RASTERIZE && interp_family(o->interp) < 0)
        return fail(NB_ERROR_INVALID, "unknown interpolation method %d", o->interp);
    if (cudaGetDevice(&device) != cudaSuccess)
        return fail(NB_ERROR_CUDA, "no CUDA device");
    if (!is_array(out))
        return fail(NB_ERROR_INVALID, "Empty array detected (output)");
    int st;
    if ((st = check_array(out, out_shape, "output", false, device)) != NB_OK) return st;
    if (!present(in))
        return fail(NB_ERROR_INVALID, "Empty array detected (input)");
    const bool value_ok = op == Op::RASTERIZE || op == Op::INSERT_EXTRACT;
    if (in->is_value && !value_ok)
        return fail(NB_ERROR_INVALID, "this function does not take a constant input");
    if (in_w && in_w->is_value && !value_ok)
        return fail(NB_ERROR_INVALID, "this function does not take a constant input weight");
    if ((st = check_array(in, in_shape, "input", false, device)) != NB_OK) return st;
    if ((st = check_array(in_w, in_shape, "input_weight", true, device)) != NB_OK) return st;
    if ((st = check_array(out_w, out_shape, "output_weight", true, device)) != NB_OK) return st;
    if (out_w && out_w->is_value)
        return fail(NB_ERROR_INVALID, "output_weight should be an array");
    if (!is_complex(in->dtype) && is_complex(out->dtype))
        return fail(NB_ERROR_INVALID, "real inputs cannot produce complex outputs");
    if (overlap(in, out) || overlap(in_w, out))
        return fail(NB_ERROR_INVALID, "Input and output arrays should not overlap");
    if (overlap(out_w, out))
        return fail(NB_ERROR_INVALID, "Output arrays should not overlap");

    const int64_t* ts = o->target_shape;
    if (op == Op::RASTERIZE || op == Op::INSERT) {
        if (in_shape[1] != 1)
            return fail(NB_ERROR_INVALID, "2d input slices are expected, but got shape={%lld,%lld,%lld,%lld}",
                        (long long) in_shape[0], (long long) in_shape[1], (long long) in_shape[2], (long long) in_shape[3]);
        if (out_shape[0] != 1 || ts[0] > 1)
            return fail(NB_ERROR_INVALID, "A single 3d volume is expected");
    } else if (op == Op::EXTRACT) {
        if (in_shape[0] != 1 || ts[0] > 1)
            return fail(NB_ERROR_INVALID, "A single 3d volume is expected");
        if (out_shape[1] != 1)
            return fail(NB_ERROR_INVALID, "2d input slices are expected");
    } else {
        if (in_shape[1] != 1 || out_shape[1] != 1)
            return fail(NB_ERROR_INVALID, "2d slices are expected");
    }
    return NB_OK;
}

int finish(cudaError_t err) {
    if (err != cudaSuccess)
        return fail(NB_ERROR_CUDA, "kernel launch failed: %s", cudaGetErrorString(err));
    g_last_error.clear();
    return NB_OK;
}

} // namespace

int prepare_rasterize(
    int32_t remap,
    const nb_array* slice, const nb_array* slice_weight, const int64_t slice_shape[4],
    const nb_array* volume, const nb_array* volume_weight, const int64_t volume_shape[4],
    const nb_transform* inv_scaling, const nb_transform* fwd_rotation,
    const nb_options* options, ProjArgs& a) {
    int device = 0;
    int st = common_checks(Op::RASTERIZE, remap, slice, slice_weight, slice_shape,
                           volume, volume_weight, volume_shape, options, device);
    if (st != NB_OK) return st;
    if ((st = check_transform(inv_scaling, slice_shape[0], false, "inv_scaling", device)) != NB_OK) return st;
    if ((st = check_transform(fwd_rotation, slice_shape[0], true, "fwd_rotation", device)) != NB_OK) return st;

    a = ProjArgs{};
    a.in = make_src(slice, 0);
    a.in_w = make_src(slice_weight, 0);
    a.out = make_dst(volume, 1);
    a.out_w = make_dst(volume_weight, 1);
    a.scale = make_xform(inv_scaling);
    a.rot = make_xform(fwd_rotation);
    a.ews = make_ews(options->ews_radius);
    a.n_slices = slice_shape[0];
    a.slice_h = static_cast<int>(slice_shape[2]);
    a.slice_w = static_cast<int>(slice_shape[3]);
    a.vol_d = static_cast<int>(volume_shape[1]);
    a.vol_h = static_cast<int>(volume_shape[2]);
    a.vol_w = static_cast<int>(volume_shape[3]);
    a.in_centered = (remap & 4) != 0;
    a.out_centered = (remap & 8) != 0;
    a.f_slice0 = static_cast<float>(slice_shape[2]);
    a.f_slice1 = static_cast<float>(slice_shape[3]);
    float t[3];
    target3(options, volume_shape, t);
    a.target0 = t[0]; a.target1 = t[1]; a.target2 = t[2];
    a.cutoff_sqd = cutoff_sqd(options);
    a.in_cplx = is_complex(slice->dtype);
    a.out_cplx = is_complex(volume->dtype);
    return NB_OK;
}

int prepare_extract(
    int32_t remap,
    const nb_array* volume, const nb_array* volume_weight, const int64_t volume_shape[4],
    const nb_array* slice, const nb_array* slice_weight, const int64_t slice_shape[4],
    const nb_transform* inv_scaling, const nb_transform* fwd_rotation,
    const nb_options* options, ProjArgs& a) {
    int device = 0;
    int st = common_checks(Op::EXTRACT, remap, volume, volume_weight, volume_shape,
                           slice, slice_weight, slice_shape, options, device);
    if (st != NB_OK) return st;
    if ((st = check_transform(inv_scaling, slice_shape[0], false, "inv_scaling", device)) != NB_OK) return st;
    if ((st = check_transform(fwd_rotation, slice_shape[0], true, "fwd_rotation", device)) != NB_OK) return st;

    a = ProjArgs{};
    a.in = make_src(volume, 1);
    a.in_w = make_src(volume_weight, 1);
    a.out = make_dst(slice, 0);
    a.out_w = make_dst(slice_weight, 0);
    a.scale = make_xform(inv_scaling);
    a.rot = make_xform(fwd_rotation);
    a.ews = make_ews(options->ews_radius);
    a.n_slices = slice_shape[0];
    a.slice_h = static_cast<int>(slice_shape[2]);
    a.slice_w = static_cast<int>(slice_shape[3]);
    a.vol_d = static_cast<int>(volume_shape[1]);
    a.vol_h = static_cast<int>(volume_shape[2]);
    a.vol_w = static_cast<int>(volume_shape[3]);
    a.in_centered = (remap & 4) != 0;
    a.out_centered = (remap & 8) != 0;
    a.interp = interp_family(options->interp);
    a.f_slice0 = static_cast<float>(slice_shape[2]);
    a.f_slice1 = static_cast<float>(slice_shape[3]);
    float t[3];
    target3(options, volume_shape, t);
    a.target0 = t[0]; a.target1 = t[1]; a.target2 = t[2];
    a.cutoff_sqd = cutoff_sqd(options);
    a.efs = fmax_ref(static_cast<float>(options->w_fftfreq_sinc), 1.f / t[0]);
    a.efb = fmax_ref(static_cast<float>(options->w_fftfreq_blackman), 1.f / t[0]);
    a.wsize = blackman_window_size(a.efb, t[0]);
    a.in_cplx = is_complex(volume->dtype);
    a.out_cplx = is_complex(slice->dtype);
    a.wide_in = needs_wide(volume) || needs_wide(volume_weight);
    return NB_OK;
}

int prepare_insert(
    int32_t remap,
    const nb_array* slice, const nb_array* slice_weight, const int64_t slice_shape[4],
    const nb_array* volume, const nb_array* volume_weight, const int64_t volume_shape[4],
    const nb_transform* fwd_scaling, const nb_transform* inv_rotation,
    const nb_options* options, ProjArgs& a) {
    int device = 0;
    int st = common_checks(Op::INSERT, remap, slice, slice_weight, slice_shape,
                           volume, volume_weight, volume_shape, options, device);
    if (st != NB_OK) return st;
    if ((st = check_transform(fwd_scaling, slice_shape[0], false, "fwd_scaling", device)) != NB_OK) return st;
    if ((st = check_transform(inv_rotation, slice_shape[0], true, "inv_rotation", device)) != NB_OK) return st;

    a = ProjArgs{};
    a.in = make_src(slice, 0);
    a.in_w = make_src(slice_weight, 0);
    a.out = make_dst(volume, 1);
    a.out_w = make_dst(volume_weight, 1);
    a.scale = make_xform(fwd_scaling);
    a.rot = make_xform(inv_rotation);
    a.ews = make_ews(options->ews_radius);
    a.n_slices = slice_shape[0];
    a.slice_h = static_cast<int>(slice_shape[2]);
    a.slice_w = static_cast<int>(slice_shape[3]);
    a.vol_d = static_cast<int>(volume_shape[1]);
    a.vol_h = static_cast<int>(volume_shape[2]);
    a.vol_w = static_cast<int>(volume_shape[3]);
    a.in_centered = (remap & 4) != 0;
    a.out_centered = (remap & 8) != 0;
    a.interp = interp_family(options->interp);
    a.f_slice0 = static_cast<float>(slice_shape[2]);
    a.f_slice1 = static_cast<float>(slice_shape[3]);
    float t[3];
    target3(options, volume_shape, t);
    a.target0 = t[0]; a.target1 = t[1]; a.target2 = t[2];
    a.cutoff_sqd = cutoff_sqd(options);
    float tmin = t[0];
    if (t[1] < tmin) tmin = t[1];
    if (t[2] < tmin) tmin = t[2];
    a.fs = fmax_ref(static_cast<float>(options->fftfreq_sinc), 1.f / tmin);
    a.fb = fmax_ref(static_cast<float>(options->fftfreq_blackman), 1.f / tmin);
    a.pfs = static_cast<float>(3.14159265358979323846 / static_cast<double>(a.fs));
    a.pfb = static_cast<float>(3.14159265358979323846 / static_cast<double>(a.fb));
    a.ifs = static_cast<float>(1.0 / static_cast<double>(a.fs));
    a.in_slice_narrow = slice_narrow(slice) && (!is_array(slice_weight) || slice_narrow(slice_weight));
    a.in_cplx = is_complex(slice->dtype);
    a.out_cplx = is_complex(volume->dtype);
    return NB_OK;
}

int finish_launch(cudaError_t err) { return finish(err); }

int report_error(int code, const char* message) { return fail(code, "%s", message); }

int check_pairs(const void* pairs, int64_t bytes, const ProjArgs& a, const char* name) {
    const int64_t need = static_cast<int64_t>(a.vol_d) * a.vol_h * (a.vol_w / 2 + 1) * 16;
    if (!pairs)
        return fail(NB_ERROR_INVALID, "%s should not be NULL", name);
    if (reinterpret_cast<uintptr_t>(pairs) % 16)
        return fail(NB_ERROR_INVALID, "%s: the pair copy should be 16-byte aligned", name);
    if (bytes < need)
        return fail(NB_ERROR_INVALID, "%s: %lld bytes given, the pair copy needs %lld", name,
                    static_cast<long long>(bytes), static_cast<long long>(need));
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) {
        cudaGetLastError();
        return fail(NB_ERROR_CUDA, "no CUDA device");
    }
    return check_device_pointer(pairs, name, device);
}

} // namespace nb

using namespace nb;

extern "C" {

int nb_fourier_interpolation_correction(const nb_array* input, const nb_array* output, int32_t interp,
                                        int32_t post_correction, void* stream) {
    if (interp_family(interp) != 1)
        return fail(NB_ERROR_INVALID, "interp=%d is currently not supported (LINEAR only)", interp);
    if (!is_array(output))
        return fail(NB_ERROR_INVALID, "output should be an array");
    if (!present(input))
        return fail(NB_ERROR_INVALID, "input should not be empty");
    if (input->dtype != NB_DTYPE_F32 || output->dtype != NB_DTYPE_F32) {
        if (is_f64(input->dtype) || is_f64(output->dtype))
            return fail(NB_ERROR_UNSUPPORTED, "f64 values are not provided on the GPU by this library");
        return fail(NB_ERROR_INVALID, "input and output should be real (f32)");
    }
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) {
        cudaGetLastError();
        return fail(NB_ERROR_CUDA, "no CUDA device");
    }
    for (int i = 0; i < 4; ++i) {
        if (output->shape[i] <= 0)
            return fail(NB_ERROR_INVALID, "Empty array detected (output)");
        if (output->strides[i] < 0 || (!input->is_value && input->strides[i] < 0))
            return fail(NB_ERROR_INVALID, "negative strides are not supported");
        if (!input->is_value && input->shape[i] != output->shape[i] && input->shape[i] != 1)
            return fail(NB_ERROR_INVALID,
                        "input of shape {%lld,%lld,%lld,%lld} cannot be broadcast to the output shape "
                        "{%lld,%lld,%lld,%lld}",
                        (long long) input->shape[0], (long long) input->shape[1], (long long) input->shape[2],
                        (long long) input->shape[3], (long long) output->shape[0], (long long) output->shape[1],
                        (long long) output->shape[2], (long long) output->shape[3]);
    }
    if (reinterpret_cast<uintptr_t>(output->data) % 4 || (!input->is_value && reinterpret_cast<uintptr_t>(input->data) % 4))
        return fail(NB_ERROR_INVALID, "misaligned data pointer");
    int st = check_device_pointer(output->data, "output", device);
    if (st == NB_OK && !input->is_value)
        st = check_device_pointer(input->data, "input", device);
    if (st != NB_OK)
        return st;
    return finish(launch_gridding_correction(input, output, post_correction != 0, static_cast<cudaStream_t>(stream)));
}

int nb_reconstruction_spectrum(const nb_array* values, const nb_array* weights, const int64_t volume_shape[4],
                               int32_t centered, double weight_threshold, const nb_array* output, void* stream) {
    if (!volume_shape)
        return fail(NB_ERROR_INVALID, "volume_shape should not be NULL");
    if (volume_shape[0] != 1)
        return fail(NB_ERROR_INVALID, "one volume at a time, got a batch of %lld", (long long) volume_shape[0]);
    if (!is_array(values) || values->dtype != NB_DTYPE_C32)
        return fail(NB_ERROR_INVALID, "values should be a complex (c32) array");
    if (!is_array(output) || output->dtype != NB_DTYPE_C32)
        return fail(NB_ERROR_INVALID, "output should be a complex (c32) array");
    if (present(weights) && (!is_array(weights) || weights->dtype != NB_DTYPE_F32))
        return fail(NB_ERROR_INVALID, "weights should be a real (f32) array or absent");
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) {
        cudaGetLastError();
        return fail(NB_ERROR_CUDA, "no CUDA device");
    }
    int st = check_array(values, volume_shape, "values", false, device);
    if (st == NB_OK)
        st = check_array(weights, volume_shape, "weights", true, device);
    if (st == NB_OK)
        st = check_array(output, volume_shape, "output", false, device);
    if (st != NB_OK)
        return st;
    const int64_t wp = volume_shape[3] / 2 + 1;
    if (output->strides[3] != 1 || output->strides[2] != wp || output->strides[1] != wp * volume_shape[2])
        return fail(NB_ERROR_INVALID, "output should be contiguous");
    if (overlap(output, values) || overlap(output, weights))
        return fail(NB_ERROR_INVALID, "output should not overlap the inputs");
    if (static_cast<int64_t>(volume_shape[1]) * volume_shape[2] * wp >= (int64_t(1) << 31))
        return fail(NB_ERROR_INVALID, "the volume must span fewer than 2^31 elements");
    return finish(launch_reconstruction_spectrum(values, present(weights) ? weights : nullptr, volume_shape,
                                                 centered != 0, static_cast<float>(weight_threshold), output,
                                                 static_cast<cudaStream_t>(stream)));
}

int64_t nb_volume_pairs_bytes(const int64_t volume_shape[4]) {
    if (!volume_shape || volume_shape[1] <= 0 || volume_shape[2] <= 0 || volume_shape[3] <= 0)
        return -1;
    return volume_shape[1] * volume_shape[2] * (volume_shape[3] / 2 + 1) * 16;
}

int nb_volume_pairs(const nb_array* volume, const int64_t volume_shape[4], void* pairs, int64_t pairs_bytes,
                    void* stream) {
    if (!volume_shape)
        return fail(NB_ERROR_INVALID, "volume_shape should not be NULL");
    if (volume_shape[0] != 1)
        return fail(NB_ERROR_INVALID, "the pair copy is made of one volume, got a batch of %lld",
                    static_cast<long long>(volume_shape[0]));
    if (!is_array(volume) || volume->dtype != NB_DTYPE_C32)
        return fail(NB_ERROR_INVALID, "the pair copy needs a complex (c32) volume array");
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) {
        cudaGetLastError();
        return fail(NB_ERROR_CUDA, "no CUDA device");
    }
    int st = check_array(volume, volume_shape, "volume", false, device);
    if (st != NB_OK)
        return st;
    ProjArgs a{};
    a.in = make_src(volume, 1);
    a.vol_d = static_cast<int>(volume_shape[1]);
    a.vol_h = static_cast<int>(volume_shape[2]);
    a.vol_w = static_cast<int>(volume_shape[3]);
    a.in_cplx = 1;
    a.interp = I_LINEAR;
    a.wsize = 1;
    if (!pairs_apply(a))
        return fail(NB_ERROR_INVALID, "the pair copy must span fewer than 2^31 voxels");
    if ((st = check_pairs(pairs, pairs_bytes, a, "pairs")) != NB_OK)
        return st;
    return finish(launch_make_pairs(a, static_cast<float4*>(pairs), static_cast<cudaStream_t>(stream)));
}

void nb_options_default(nb_options* o) {
    if (!o)
        return;
    *o = nb_options{};
    o->interp = NB_INTERP_LINEAR;
    o->fftfreq_cutoff = 0.5;
    o->fftfreq_sinc = -1;
    o->fftfreq_blackman = -1;
    o->w_fftfreq_sinc = -1;
    o->w_fftfreq_blackman = -1;
}

const char* nb_last_error(void) { return g_last_error.c_str(); }

const char* nb_version(void) { return "0.1.0"; }

int nb_set_scratch_limit(int32_t device, int64_t bytes) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess) {
        cudaGetLastError();
        count = 0;
    }
    if (device < 0 || device >= count || !nb::set_scratch_limit(device, bytes))
        return nb::report_error(NB_ERROR_INVALID, "no such device");
    return NB_OK;
}

int64_t nb_scratch_limit(int32_t device) { return nb::scratch_limit(device); }

int64_t nb_scratch_refusals(int32_t device) { return nb::refused_allocations(device); }

int nb_rasterize_central_slices_3d(
    int32_t remap,
    const nb_array* slice, const nb_array* slice_weight, const int64_t slice_shape[4],
    const nb_array* volume, const nb_array* volume_weight, const int64_t volume_shape[4],
    const nb_transform* inv_scaling, const nb_transform* fwd_rotation,
    const nb_options* options, void* stream) {
    ProjArgs a{};
    const int st = prepare_rasterize(remap, slice, slice_weight, slice_shape, volume, volume_weight, volume_shape,
                                     inv_scaling, fwd_rotation, options, a);
    if (st != NB_OK) return st;
    return finish(launch_rasterize(a, static_cast<cudaStream_t>(stream)));
}

int nb_insert_central_slices_3d(
    int32_t remap,
    const nb_array* slice, const nb_array* slice_weight, const int64_t slice_shape[4],
    const nb_array* volume, const nb_array* volume_weight, const int64_t volume_shape[4],
    const nb_transform* fwd_scaling, const nb_transform* inv_rotation,
    const nb_options* options, void* stream) {
    ProjArgs a{};
    const int st = prepare_insert(remap, slice, slice_weight, slice_shape, volume, volume_weight, volume_shape,
                                  fwd_scaling, inv_rotation, options, a);
    if (st != NB_OK) return st;
    return finish(launch_insert(a, static_cast<cudaStream_t>(stream)));
}

int nb_insert_central_slices_3d_scatter(
    int32_t remap,
    const nb_array* slice, const nb_array* slice_weight, const int64_t slice_shape[4],
    const nb_array* volume, const nb_array* volume_weight, const int64_t volume_shape[4],
    const nb_transform* fwd_scaling, const nb_transform* inv_rotation,
    const nb_options* options, void* stream) {
    ProjArgs a{};
    const int st = prepare_insert(remap, slice, slice_weight, slice_shape, volume, volume_weight, volume_shape,
                                  fwd_scaling, inv_rotation, options, a);
    if (st != NB_OK) return st;
    return finish(launch_insert_scatter(a, static_cast<cudaStream_t>(stream)));
}

int nb_extract_central_slices_3d(
    int32_t remap,
    const nb_array* volume, const nb_array* volume_weight, const int64_t volume_shape[4],
    const nb_array* slice, const nb_array* slice_weight, const int64_t slice_shape[4],
    const nb_transform* inv_scaling, const nb_transform* fwd_rotation,
    const nb_options* options, void* stream) {
    ProjArgs a{};
    const int st = prepare_extract(remap, volume, volume_weight, volume_shape, slice, slice_weight, slice_shape,
                                   inv_scaling, fwd_rotation, options, a);
    if (st != NB_OK) return st;
    return finish(launch_extract(a, static_cast<cudaStream_t>(stream)));
}

int nb_insert_and_extract_central_slices_3d(
    int32_t remap,
    const nb_array* input_slice, const nb_array* input_weight, const int64_t input_slice_shape[4],
    const nb_array* output_slice, const nb_array* output_weight, const int64_t output_slice_shape[4],
    const nb_transform* input_fwd_scaling, const nb_transform* input_inv_rotation,
    const nb_transform* output_inv_scaling, const nb_transform* output_fwd_rotation,
    const nb_options* options, void* stream) {
    int device = 0;
    int st = common_checks(Op::INSERT_EXTRACT, remap, input_slice, input_weight, input_slice_shape,
                           output_slice, output_weight, output_slice_shape, options, device);
    if (st != NB_OK) return st;
    if ((st = check_transform(input_fwd_scaling, input_slice_shape[0], false, "input_scaling", device)) != NB_OK) return st;
    if ((st = check_transform(input_inv_rotation, input_slice_shape[0], true, "input_rotation", device)) != NB_OK) return st;
    if ((st = check_transform(output_inv_scaling, output_slice_shape[0], false, "output_scaling", device)) != NB_OK) return st;
    if ((st = check_transform(output_fwd_rotation, output_slice_shape[0], true, "output_rotation", device)) != NB_OK) return st;

    // correct_weights compatibility (FourierProject.hpp:2013-2020): the window size of the raw option.
    const float vz = static_cast<float>(output_slice_shape[2] < output_slice_shape[3] ? output_slice_shape[2]
                                                                                      : output_slice_shape[3]);
    const int raw_w = blackman_window_size(static_cast<float>(options->w_fftfreq_blackman), vz);
    if (options->correct_weights && (options->add_to_output || raw_w != 1))
        return fail(NB_ERROR_INVALID,
                    "options.correct_weights=true is not compatible with options.add_to_output=true and "
                    "options.w_windowed_sinc.fftfreq_blackman=%g (=%d pixels)", options->w_fftfreq_blackman, raw_w);

    ProjArgs a{};
    a.in = make_src(input_slice, 0);
    a.in_w = make_src(input_weight, 0);
    a.out = make_dst(output_slice, 0);
    a.out_w = make_dst(output_weight, 0);
    a.scale = make_xform(input_fwd_scaling);
    a.rot = make_xform(input_inv_rotation);
    a.scale2 = make_xform(output_inv_scaling);
    a.rot2 = make_xform(output_fwd_rotation);
    a.ews = make_ews(options->ews_radius);
    a.n_slices = output_slice_shape[0];
    a.n_in = input_slice_shape[0];
    a.slice_h = static_cast<int>(output_slice_shape[2]);
    a.slice_w = static_cast<int>(output_slice_shape[3]);
    a.in_h = static_cast<int>(input_slice_shape[2]);
    a.in_w_ = static_cast<int>(input_slice_shape[3]);
    a.in_centered = (remap & 4) != 0;
    a.out_centered = (remap & 8) != 0;
    a.interp = interp_family(options->interp);
    a.f_slice0 = static_cast<float>(output_slice_shape[2]);
    a.f_slice1 = static_cast<float>(output_slice_shape[3]);
    a.f_in0 = static_cast<float>(input_slice_shape[2]);
    a.f_in1 = static_cast<float>(input_slice_shape[3]);
    a.cutoff_sqd = cutoff_sqd(options);
    a.vz = vz;
    a.fs = fmax_ref(static_cast<float>(options->fftfreq_sinc), 1.f / vz);
    a.fb = fmax_ref(static_cast<float>(options->fftfreq_blackman), 1.f / vz);
    a.pfs = static_cast<float>(3.14159265358979323846 / static_cast<double>(a.fs));
    a.pfb = static_cast<float>(3.14159265358979323846 / static_cast<double>(a.fb));
    a.ifs = static_cast<float>(1.0 / static_cast<double>(a.fs));
    a.efs = fmax_ref(static_cast<float>(options->w_fftfreq_sinc), 1.f / vz);
    a.efb = fmax_ref(static_cast<float>(options->w_fftfreq_blackman), 1.f / vz);
    a.wsize = blackman_window_size(a.efb, vz);
    a.add_to_output = options->add_to_output != 0;
    a.correct_weights = options->correct_weights != 0;
    a.in_slice_narrow = slice_narrow(input_slice) && (!is_array(input_weight) || slice_narrow(input_weight));
    a.in_cplx = is_complex(input_slice->dtype);
    a.out_cplx = is_complex(output_slice->dtype);
    return finish(launch_insert_extract(a, static_cast<cudaStream_t>(stream)));
}

} // extern "C"
