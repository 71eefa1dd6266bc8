// Reference-side binding: what a noa maintainer adds so that noa's GPU branch of the Fourier
// central-slice functions calls noa_b200 instead of `details::launch_*<REMAP, i32, true>`.
//
// Header-only C++20; include it from noa/xform/FourierProject.hpp (it needs noa's types). Each
// function below converts noa's arguments — Views/Arrays of c32/f32, constant values, Empty weights,
// Mat22/Mat33/Quaternion values or arrays, and noa's option structs — into the plain C structs of
// noa_b200/fourier_project.h, and turns a non-zero status into noa's exception, carrying
// nb_last_error(). The checks noa runs before its GPU branch (fourier_projection_check_parameters,
// FourierProject.hpp:1100-1185) stay where they are; noa_b200 repeats them.
//
// Replaced calls (all in noa/xform/FourierProject.hpp):
//   rasterize_central_slices_3d           :1679  details::launch_rasterize_central_slices_3d<REMAP, i32>
//   insert_central_slices_3d              :1801  details::launch_insert_central_slices_3d<REMAP, i32, true>
//   extract_central_slices_3d             :1900  details::launch_extract_central_slices_3d<REMAP, i32, true>
//   insert_and_extract_central_slices_3d  :2031  details::launch_insert_and_extract_central_slices_3d<REMAP, i32, true>
#pragma once

#include <noa/xform/FourierProject.hpp>
#include <noa/xform/Texture.hpp>

#include "noa_b200/fourier_project.h"

#include <type_traits>

namespace noa_b200::binding {
    namespace nt = ::noa::traits;
    namespace nx = ::noa::xform;
    namespace nf = ::noa::fft;

    template<typename T>
    constexpr int32_t dtype_of() {
        using v = std::remove_cv_t<T>;
        if constexpr (std::is_same_v<v, ::noa::f32>) return NB_DTYPE_F32;
        else if constexpr (std::is_same_v<v, ::noa::c32>) return NB_DTYPE_C32;
        else if constexpr (std::is_same_v<v, ::noa::f64>) return NB_DTYPE_F64;
        else if constexpr (std::is_same_v<v, ::noa::c64>) return NB_DTYPE_C64;
        else return 0;
    }

    // An array argument: a noa View/Array, a constant value (AllowValue inputs) or Empty.
    template<typename T>
    nb_array to_array(const T& a) {
        nb_array r{};
        using d = std::decay_t<T>;
        if constexpr (nt::empty<d>) {
            return r;
        } else if constexpr (nt::varray<d>) {
            r.data = const_cast<void*>(static_cast<const void*>(a.get()));
            r.dtype = dtype_of<nt::value_type_t<d>>();
            for (int i = 0; i < 4; ++i) {
                r.shape[i] = a.shape()[i];
                r.strides[i] = a.strides()[i];
            }
        } else {  // a value standing for every element
            r.is_value = 1;
            r.dtype = dtype_of<d>();
            if constexpr (nt::complex<d>) {
                r.value[0] = static_cast<double>(a.real);
                r.value[1] = static_cast<double>(a.imag);
            } else {
                r.value[0] = static_cast<double>(a);
            }
        }
        return r;
    }

    // A per-slice transform: Empty, one Mat22/Mat33/Quaternion value (passed inline), or an array of
    // them (noa's memory layout is kept: Mat33<f32> is 48 bytes).
    template<typename T>
    nb_transform to_transform(const T& x) {
        nb_transform t{};
        using d = std::decay_t<T>;
        if constexpr (nt::empty<d>) {
            t.kind = NB_XFORM_NONE;
        } else if constexpr (nt::varray<d>) {
            using v = std::remove_cv_t<nt::value_type_t<d>>;
            t.data = static_cast<const void*>(x.get());
            t.count = x.n_elements();
            if constexpr (std::is_same_v<v, ::noa::Mat22<::noa::f32>>) t.kind = NB_XFORM_MAT22_F32;
            else if constexpr (std::is_same_v<v, ::noa::Mat33<::noa::f32>>) t.kind = NB_XFORM_MAT33_F32;
            else if constexpr (std::is_same_v<v, nx::Quaternion<::noa::f32>>) t.kind = NB_XFORM_QUAT_F32;
            else t.kind = -1;  // f64 transforms: rejected as invalid by the library
        } else {
            t.count = 1;
            if constexpr (std::is_same_v<d, ::noa::Mat22<::noa::f32>>) {
                t.kind = NB_XFORM_MAT22_F32;
                for (int i = 0; i < 2; ++i)
                    for (int j = 0; j < 2; ++j)
                        t.value[i * 2 + j] = static_cast<double>(x[i][j]);
            } else if constexpr (std::is_same_v<d, ::noa::Mat33<::noa::f32>>) {
                t.kind = NB_XFORM_MAT33_F32;
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j)
                        t.value[i * 3 + j] = static_cast<double>(x[i][j]);
            } else if constexpr (std::is_same_v<d, nx::Quaternion<::noa::f32>>) {
                t.kind = NB_XFORM_QUAT_F32;
                t.value[0] = x.z; t.value[1] = x.y; t.value[2] = x.x; t.value[3] = x.w;
            } else {
                t.kind = -1;
            }
        }
        return t;
    }

    // An input that may be a Texture (Texture.hpp). noa keeps a GPU texture's values in a CUDA array
    // (Texture.hpp:147-170); the binding copies them into linear device memory with one
    // cudaMemcpy3DAsync on the call's stream (a 3-D array for a volume, a layered 2-D array for a stack
    // of slices: extent W x H x (B*D) either way), keeps that buffer alive on the stream, and passes it
    // as an array. Views, values and Empty pass through unchanged.
    template<typename T>
    struct Staged {
        using d = std::decay_t<T>;
        static constexpr bool TEXTURE = nt::texture<d>;
        nb_array array{};
        std::conditional_t<TEXTURE, ::noa::Array<nt::mutable_value_type_t<d>>, int> keep{};
    };

    template<typename T>
    Staged<T> stage(const T& a, void* stream) {
        Staged<T> s;
        if constexpr (Staged<T>::TEXTURE) {
#ifdef NOA_ENABLE_CUDA
            using V = nt::mutable_value_type_t<std::decay_t<T>>;
            const ::noa::Shape4 shape = a.shape();
            s.keep = ::noa::Array<V>(shape, ::noa::ArrayOption{a.device(), ::noa::Allocator::DEFAULT});
            cudaMemcpy3DParms p{};
            p.srcArray = a.cuda().handle->array.get();
            p.dstPtr = make_cudaPitchedPtr(s.keep.get(), static_cast<size_t>(shape[3]) * sizeof(V),
                                           static_cast<size_t>(shape[3]), static_cast<size_t>(shape[2]));
            p.extent = make_cudaExtent(static_cast<size_t>(shape[3]), static_cast<size_t>(shape[2]),
                                       static_cast<size_t>(shape[0] * shape[1]));
            p.kind = cudaMemcpyDeviceToDevice;
            const cudaError_t err = cudaMemcpy3DAsync(&p, static_cast<cudaStream_t>(stream));
            if (err != cudaSuccess)
                ::noa::panic("noa_b200: staging a texture failed: {}", cudaGetErrorString(err));
            ::noa::Stream::current(a.device()).cuda().enqueue_attach(s.keep);
            s.array = to_array(s.keep.view());
#else
            (void) stream;
            ::noa::panic("noa_b200: texture inputs need noa's CUDA backend");
#endif
        } else {
            (void) stream;
            s.array = to_array(a);
        }
        return s;
    }

    inline void fill_common(nb_options& o, double cutoff, const ::noa::Shape4& target, const ::noa::Vec<double, 2>& ews) {
        nb_options_default(&o);
        o.fftfreq_cutoff = cutoff;
        for (int i = 0; i < 4; ++i)
            o.target_shape[i] = target[i];
        o.ews_radius[0] = ews[0];
        o.ews_radius[1] = ews[1];
    }

    inline void check(int status) {
        if (status != NB_OK)
            ::noa::panic("noa_b200: {}", nb_last_error());
    }

    inline const int64_t* shape_ptr(const ::noa::Shape4& s) {
        static_assert(sizeof(s[0]) == sizeof(int64_t));
        return reinterpret_cast<const int64_t*>(&s[0]);
    }

    template<nf::Layout REMAP, typename Input, typename InputWeight, typename Output, typename OutputWeight,
             typename Scale, typename Rotate>
    void rasterize(const Input& slice, const InputWeight& slice_weight, const ::noa::Shape4& slice_shape,
                   const Output& volume, const OutputWeight& volume_weight, const ::noa::Shape4& volume_shape,
                   const Scale& inv_scaling, const Rotate& fwd_rotation,
                   const nx::RasterizeCentralSlicesOptions& options, void* stream) {
        nb_options o;
        fill_common(o, options.fftfreq_cutoff, options.target_shape, options.ews_radius);
        const nb_array s = to_array(slice), sw = to_array(slice_weight), v = to_array(volume), vw = to_array(volume_weight);
        const nb_transform sc = to_transform(inv_scaling), rot = to_transform(fwd_rotation);
        check(nb_rasterize_central_slices_3d(static_cast<int32_t>(REMAP.value), &s, &sw, shape_ptr(slice_shape),
                                             &v, &vw, shape_ptr(volume_shape), &sc, &rot, &o, stream));
    }

    template<nf::Layout REMAP, typename Input, typename InputWeight, typename Output, typename OutputWeight,
             typename Scale, typename Rotate>
    void insert(const Input& slice, const InputWeight& slice_weight, const ::noa::Shape4& slice_shape,
                const Output& volume, const OutputWeight& volume_weight, const ::noa::Shape4& volume_shape,
                const Scale& fwd_scaling, const Rotate& inv_rotation,
                const nx::InsertCentralSlicesOptions& options, void* stream) {
        nb_options o;
        fill_common(o, options.fftfreq_cutoff, options.target_shape, options.ews_radius);
        // With textures, the interpolation method is the textures' (FourierProject.hpp:1203-1217).
        o.interp = static_cast<int32_t>(
            nx::details::fourier_insert_extract_interp_mode(slice, slice_weight, options.interp).value);
        o.fftfreq_sinc = options.windowed_sinc.fftfreq_sinc;
        o.fftfreq_blackman = options.windowed_sinc.fftfreq_blackman;
        const auto s = stage(slice, stream);
        const auto sw = stage(slice_weight, stream);
        const nb_array v = to_array(volume), vw = to_array(volume_weight);
        const nb_transform sc = to_transform(fwd_scaling), rot = to_transform(inv_rotation);
        check(nb_insert_central_slices_3d(static_cast<int32_t>(REMAP.value), &s.array, &sw.array,
                                          shape_ptr(slice_shape), &v, &vw, shape_ptr(volume_shape), &sc, &rot, &o,
                                          stream));
    }

    template<nf::Layout REMAP, typename Input, typename InputWeight, typename Output, typename OutputWeight,
             typename Scale, typename Rotate>
    void extract(const Input& volume, const InputWeight& volume_weight, const ::noa::Shape4& volume_shape,
                 const Output& slice, const OutputWeight& slice_weight, const ::noa::Shape4& slice_shape,
                 const Scale& inv_scaling, const Rotate& fwd_rotation,
                 const nx::ExtractCentralSlicesOptions& options, void* stream) {
        nb_options o;
        fill_common(o, options.fftfreq_cutoff, options.target_shape, options.ews_radius);
        o.interp = static_cast<int32_t>(
            nx::details::fourier_insert_extract_interp_mode(volume, volume_weight, options.interp).value);
        o.w_fftfreq_sinc = options.w_windowed_sinc.fftfreq_sinc;
        o.w_fftfreq_blackman = options.w_windowed_sinc.fftfreq_blackman;
        const auto v = stage(volume, stream);
        const auto vw = stage(volume_weight, stream);
        const nb_array s = to_array(slice), sw = to_array(slice_weight);
        const nb_transform sc = to_transform(inv_scaling), rot = to_transform(fwd_rotation);
        check(nb_extract_central_slices_3d(static_cast<int32_t>(REMAP.value), &v.array, &vw.array,
                                           shape_ptr(volume_shape), &s, &sw, shape_ptr(slice_shape), &sc, &rot, &o,
                                           stream));
    }

    template<nf::Layout REMAP, typename Input, typename InputWeight, typename Output, typename OutputWeight,
             typename InputScale, typename InputRotate, typename OutputScale, typename OutputRotate>
    void insert_and_extract(const Input& input_slice, const InputWeight& input_weight, const ::noa::Shape4& input_shape,
                            const Output& output_slice, const OutputWeight& output_weight, const ::noa::Shape4& output_shape,
                            const InputScale& input_fwd_scaling, const InputRotate& input_inv_rotation,
                            const OutputScale& output_inv_scaling, const OutputRotate& output_fwd_rotation,
                            const nx::InsertAndExtractCentralSlicesOptions& options, void* stream) {
        nb_options o;
        fill_common(o, options.fftfreq_cutoff, ::noa::Shape4{}, options.ews_radius);
        o.interp = static_cast<int32_t>(
            nx::details::fourier_insert_extract_interp_mode(input_slice, input_weight, options.interp).value);
        o.fftfreq_sinc = options.input_windowed_sinc.fftfreq_sinc;
        o.fftfreq_blackman = options.input_windowed_sinc.fftfreq_blackman;
        o.w_fftfreq_sinc = options.w_windowed_sinc.fftfreq_sinc;
        o.w_fftfreq_blackman = options.w_windowed_sinc.fftfreq_blackman;
        o.add_to_output = options.add_to_output;
        o.correct_weights = options.correct_weights;
        const auto i = stage(input_slice, stream);
        const auto iw = stage(input_weight, stream);
        const nb_array out = to_array(output_slice), ow = to_array(output_weight);
        const nb_transform isc = to_transform(input_fwd_scaling), irot = to_transform(input_inv_rotation);
        const nb_transform osc = to_transform(output_inv_scaling), orot = to_transform(output_fwd_rotation);
        check(nb_insert_and_extract_central_slices_3d(static_cast<int32_t>(REMAP.value), &i.array, &iw.array,
                                                      shape_ptr(input_shape),
                                                      &out, &ow, shape_ptr(output_shape), &isc, &irot, &osc, &orot,
                                                      &o, stream));
    }
}
