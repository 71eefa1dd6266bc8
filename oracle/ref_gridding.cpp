// ORACLE TEST INFRASTRUCTURE — not part of the product.
//
// C-ABI driver around the reference's own fourier_interpolation_correction (noa/xform/FourierProject.hpp
// :2062-2087, class GriddingCorrection :1009-1061) on the CPU. As published, GriddingCorrection does not
// compile when instantiated: its constructor (:1034) passes `l_shape != 1` to Vec::from_vec, but
// Vec's operator!= returns one bool (noa/base/Vec.hpp:493), not a per-element vector. oracle/Makefile
// therefore compiles this file against a copy of FourierProject.hpp, generated under oracle/_ref/ at
// build time, in which that single expression is spelled per element:
//     coord3_type::from_vec(l_shape != 1)
//  -> coord3_type::from_values(l_shape[0] != 1, l_shape[1] != 1, l_shape[2] != 1)
// which is what its comment says ("if size == 1, half should be 0"). Nothing else changes, and the
// other reference entry points are built from the unmodified header.
#include "ref_driver.hpp"

#include <noa/xform/FourierProject.hpp>

#include <cstdio>
#include <exception>

using namespace ::noa::types;
namespace nx = ::noa::xform;

namespace {
    const ArrayOption CPU{Device("cpu"), Allocator::DEFAULT};

    template<typename T>
    View<T> view(const noaref_array* a) {
        return View<T>(static_cast<T*>(a->ptr), Shape4{a->shape[0], a->shape[1], a->shape[2], a->shape[3]},
                       Strides4{a->strides[0], a->strides[1], a->strides[2], a->strides[3]}, CPU);
    }

    template<typename T>
    int run(const noaref_array* in, const noaref_array* out, int32_t post, int n_threads, char* err, int errlen) {
        try {
            ::noa::Stream::current(Device("cpu")).set_thread_limit(n_threads > 0 ? n_threads : 1);
            nx::fourier_interpolation_correction(view<const T>(in), view<T>(out), nx::Interp::LINEAR, post != 0);
            ::noa::Stream::current(Device("cpu")).synchronize();
            return 0;
        } catch (const std::exception& e) {
            if (err)
                std::snprintf(err, static_cast<size_t>(errlen), "%s", e.what());
            return -1;
        }
    }
}

extern "C" int noaref_gridding_correction_f32(const noaref_array* in, const noaref_array* out, int32_t post,
                                              int n_threads, char* err, int errlen) {
    return run<f32>(in, out, post, n_threads, err, errlen);
}

extern "C" int noaref_gridding_correction_f64(const noaref_array* in, const noaref_array* out, int32_t post,
                                              int n_threads, char* err, int errlen) {
    return run<f64>(in, out, post, n_threads, err, errlen);
}
