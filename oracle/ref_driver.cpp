// ORACLE TEST INFRASTRUCTURE — not part of the product.
//
// One translation unit per (function, value combination); oracle/Makefile compiles this file with
// -DREF_FUNC=<0..3> -DREF_COMBO=<0..4>. See ref_driver.hpp for the entry points.
#include "ref_driver.hpp"

#include <noa/xform/FourierProject.hpp>

#include <cstdio>
#include <exception>
#include <utility>
#include <vector>

using namespace ::noa::types;
namespace nx = ::noa::xform;
namespace nf = ::noa::fft;

#if REF_COMBO == 0
using vin_t = c32; using vout_t = c32; using real_t = f32;
#define REF_ALL_WEIGHTS 1
#define REF_QUAT 1
#define REF_SUFFIX c32c32
#elif REF_COMBO == 1
using vin_t = f32; using vout_t = f32; using real_t = f32;
#define REF_ALL_WEIGHTS 0
#define REF_QUAT 0
#define REF_SUFFIX f32f32
#elif REF_COMBO == 2
using vin_t = c32; using vout_t = f32; using real_t = f32;
#define REF_ALL_WEIGHTS 0
#define REF_QUAT 0
#define REF_SUFFIX c32f32
#elif REF_COMBO == 3
using vin_t = c64; using vout_t = c64; using real_t = f64;
#define REF_ALL_WEIGHTS 1
#define REF_QUAT 0
#define REF_SUFFIX c64c64
#elif REF_COMBO == 4
using vin_t = f64; using vout_t = f64; using real_t = f64;
#define REF_ALL_WEIGHTS 0
#define REF_QUAT 0
#define REF_SUFFIX f64f64
#else
#error "REF_COMBO"
#endif

#if REF_FUNC == 0
#define REF_NAME_BASE noaref_rasterize_
#elif REF_FUNC == 1
#define REF_NAME_BASE noaref_insert_
#elif REF_FUNC == 2
#define REF_NAME_BASE noaref_extract_
#elif REF_FUNC == 3
#define REF_NAME_BASE noaref_insert_extract_
#else
#error "REF_FUNC"
#endif

#define REF_CAT2(a, b) a##b
#define REF_CAT(a, b) REF_CAT2(a, b)
#define REF_NAME REF_CAT(REF_NAME_BASE, REF_SUFFIX)

namespace {
    using w_t = real_t;
    using mat22_t = Mat22<real_t>;
    using mat33_t = Mat33<real_t>;
    using quat_t = nx::Quaternion<real_t>;

    Shape4 shape4(const int64_t* s) { return Shape4{s[0], s[1], s[2], s[3]}; }
    Strides4 strides4(const int64_t* s) { return Strides4{s[0], s[1], s[2], s[3]}; }
    const ArrayOption CPU{Device("cpu"), Allocator::DEFAULT};

    template<typename T>
    View<T> view(const noaref_array* a) {
        return View<T>(static_cast<T*>(a->ptr), shape4(a->shape), strides4(a->strides), CPU);
    }

    Vec<f64, 2> vec2(const double* v) { return Vec<f64, 2>{v[0], v[1]}; }

    // Scales are always passed as per-slice arrays (identity when the caller has none); the reference
    // treats an identity transform exactly like Empty (FourierProject.hpp:1234-1244, transform_vector).
    struct Transforms {
        std::vector<mat22_t> scale;
        View<const mat22_t> scale_view;
        View<const mat33_t> mat_view;
        View<const quat_t> quat_view;
    };

    Transforms make_transforms(const void* scale, const void* rot, isize n) {
        Transforms t;
        if (scale) {
            t.scale_view = View<const mat22_t>(static_cast<const mat22_t*>(scale), n, CPU);
        } else {
            t.scale.assign(static_cast<size_t>(n), mat22_t::eye(1));
            t.scale_view = View<const mat22_t>(t.scale.data(), n, CPU);
        }
        t.mat_view = View<const mat33_t>(static_cast<const mat33_t*>(rot), n, CPU);
        t.quat_view = View<const quat_t>(static_cast<const quat_t*>(rot), n, CPU);
        return t;
    }

    template<nf::Layout REMAP, typename InW, typename OutW, typename Rot>
    void call(const noaref_array* in, InW in_w, const int64_t* in_shape,
              const noaref_array* out, OutW out_w, const int64_t* out_shape,
              const Transforms& t0, const Transforms& t1, const Rot& rot0, const Rot& rot1,
              const noaref_options* o) {
        const Shape4 ishape = shape4(in_shape);
        const Shape4 oshape = shape4(out_shape);
#if REF_FUNC == 0
        (void) t1; (void) rot1;
        nx::rasterize_central_slices_3d<REMAP>(
            view<const vin_t>(in), std::move(in_w), ishape, view<vout_t>(out), std::move(out_w), oshape,
            t0.scale_view, rot0,
            {.fftfreq_cutoff = o->fftfreq_cutoff, .target_shape = shape4(o->target_shape),
             .ews_radius = vec2(o->ews_radius)});
#elif REF_FUNC == 1
        (void) t1; (void) rot1;
        nx::insert_central_slices_3d<REMAP>(
            view<const vin_t>(in), std::move(in_w), ishape, view<vout_t>(out), std::move(out_w), oshape,
            t0.scale_view, rot0,
            {.interp = static_cast<nx::Interp::Method>(o->interp),
             .windowed_sinc = {o->sinc[0], o->sinc[1]},
             .fftfreq_cutoff = o->fftfreq_cutoff, .target_shape = shape4(o->target_shape),
             .ews_radius = vec2(o->ews_radius)});
#elif REF_FUNC == 2
        (void) t1; (void) rot1;
        nx::extract_central_slices_3d<REMAP>(
            view<const vin_t>(in), std::move(in_w), ishape, view<vout_t>(out), std::move(out_w), oshape,
            t0.scale_view, rot0,
            {.interp = static_cast<nx::Interp::Method>(o->interp),
             .w_windowed_sinc = {o->w_sinc[0], o->w_sinc[1]},
             .fftfreq_cutoff = o->fftfreq_cutoff, .target_shape = shape4(o->target_shape),
             .ews_radius = vec2(o->ews_radius)});
#else
        nx::insert_and_extract_central_slices_3d<REMAP>(
            view<const vin_t>(in), std::move(in_w), ishape, view<vout_t>(out), std::move(out_w), oshape,
            t0.scale_view, rot0, t1.scale_view, rot1,
            {.interp = static_cast<nx::Interp::Method>(o->interp),
             .input_windowed_sinc = {o->sinc[0], o->sinc[1]},
             .w_windowed_sinc = {o->w_sinc[0], o->w_sinc[1]},
             .add_to_output = o->add_to_output != 0,
             .correct_weights = o->correct_weights != 0,
             .fftfreq_cutoff = o->fftfreq_cutoff,
             .ews_radius = vec2(o->ews_radius)});
#endif
    }

    template<nf::Layout REMAP, typename Rot>
    int dispatch_weights(const noaref_array* in, const noaref_array* in_w, const int64_t* in_shape,
                         const noaref_array* out, const noaref_array* out_w, const int64_t* out_shape,
                         const Transforms& t0, const Transforms& t1, const Rot& rot0, const Rot& rot1,
                         const noaref_options* o) {
        const bool has_in = in_w && in_w->ptr;
        const bool has_out = out_w && out_w->ptr;
        if (!has_in && !has_out) {
            call<REMAP>(in, Empty{}, in_shape, out, Empty{}, out_shape, t0, t1, rot0, rot1, o);
            return 0;
        }
        if (has_in && has_out) {
            call<REMAP>(in, view<const w_t>(in_w), in_shape, out, view<w_t>(out_w), out_shape,
                        t0, t1, rot0, rot1, o);
            return 0;
        }
#if REF_ALL_WEIGHTS
        if (!has_in && has_out) {
            call<REMAP>(in, Empty{}, in_shape, out, view<w_t>(out_w), out_shape, t0, t1, rot0, rot1, o);
            return 0;
        }
#endif
        return -2;
    }

    template<nf::Layout REMAP>
    int dispatch_rotation(const noaref_array* in, const noaref_array* in_w, const int64_t* in_shape,
                          const noaref_array* out, const noaref_array* out_w, const int64_t* out_shape,
                          const Transforms& t0, const Transforms& t1, int rot_kind, const noaref_options* o) {
        if (rot_kind == NOAREF_MAT33)
            return dispatch_weights<REMAP>(in, in_w, in_shape, out, out_w, out_shape,
                                           t0, t1, t0.mat_view, t1.mat_view, o);
#if REF_QUAT
        if (rot_kind == NOAREF_QUAT)
            return dispatch_weights<REMAP>(in, in_w, in_shape, out, out_w, out_shape,
                                           t0, t1, t0.quat_view, t1.quat_view, o);
#endif
        return -2;
    }
}

NOAREF_DECLARE(REF_NAME) {
    try {
        ::noa::Stream::current(Device("cpu")).set_thread_limit(n_threads > 0 ? n_threads : 1);
#if REF_FUNC == 2
        const isize n0 = out_shape[0];
#else
        const isize n0 = in_shape[0];
#endif
        const isize n1 = out_shape[0];
        const Transforms t0 = make_transforms(scale0, rot0, n0);
        const Transforms t1 = make_transforms(scale1, rot1 ? rot1 : rot0, rot1 ? n1 : n0);
        int status = -3;
        switch (opt->remap) {
            case 0:  status = dispatch_rotation<nf::Layout::H2H>(in, in_w, in_shape, out, out_w, out_shape, t0, t1, rot_kind, opt); break;
            case 8:  status = dispatch_rotation<nf::Layout::H2HC>(in, in_w, in_shape, out, out_w, out_shape, t0, t1, rot_kind, opt); break;
            case 4:  status = dispatch_rotation<nf::Layout::HC2H>(in, in_w, in_shape, out, out_w, out_shape, t0, t1, rot_kind, opt); break;
            case 12: status = dispatch_rotation<nf::Layout::HC2HC>(in, in_w, in_shape, out, out_w, out_shape, t0, t1, rot_kind, opt); break;
            default: break;
        }
        if (status != 0 && err)
            std::snprintf(err, static_cast<size_t>(errlen), "variant not instantiated in the driver (status %d)", status);
        return status;
    } catch (const std::exception& e) {
        if (err)
            std::snprintf(err, static_cast<size_t>(errlen), "%s", e.what());
        return -1;
    }
}
