// TEST INFRASTRUCTURE — not part of the product.
//
// Runs the reference-side binding (include/noa_b200/noa_binding.hpp) on a GPU with noa's own CUDA
// backend, compiled from the reference sources by oracle/Makefile (target ref-cuda) into
// oracle/_ref/libnoa_ref_cuda.so. noa builds a Texture<c32> of a volume the way its users do
// (xform/Texture.hpp:63-170: a CUDA array and a texture object), and the binding's extract() is called
// twice: with that texture, and with the plain device array it was made from. The binding stages the
// texture's CUDA array into linear memory and takes the interpolation method from the texture
// (FourierProject.hpp:1203-1217), so both calls must give the same slices.
#include "noa_b200/noa_binding.hpp"

#include <cstdio>
#include <cstring>
#include <exception>

using namespace ::noa::types;
namespace nx = ::noa::xform;
namespace nf = ::noa::fft;

extern "C" int noaref_texture_extract(const void* volume, int64_t n, const void* rotations, int64_t count,
                                      int32_t interp, void* out_texture, void* out_array, char* err, int errlen) {
    try {
        const Device gpu("gpu:0");
        const ArrayOption on_gpu{gpu, Allocator::DEFAULT};
        const Shape4 vshape{1, n, n, n / 2 + 1}, sshape{count, 1, n, n / 2 + 1};
        const Shape4 vlogical{1, n, n, n}, slogical{count, 1, n, n};

        const View<const c32> h_volume(static_cast<const c32*>(volume), vshape);
        const View<const Mat33<f32>> h_rot(static_cast<const Mat33<f32>*>(rotations), Shape4{1, 1, 1, count});
        Array<c32> d_volume = h_volume.to(on_gpu);
        Array<Mat33<f32>> d_rot = h_rot.to(on_gpu);
        const nx::Interp method = interp == 0 ? nx::Interp::NEAREST
                                : interp == 2 ? nx::Interp::CUBIC : nx::Interp::LINEAR;
        nx::Texture<c32> texture(d_volume, gpu, method);

        Array<c32> a(sshape, on_gpu), b(sshape, on_gpu);
        auto& stream = ::noa::Stream::current(gpu);
        void* handle = static_cast<void*>(stream.cuda().get());
        nx::ExtractCentralSlicesOptions options{};
        options.interp = method;
        noa_b200::binding::extract<nf::Layout::HC2H>(texture, Empty{}, vlogical, a.view(), Empty{}, slogical,
                                                     Empty{}, d_rot.view(), options, handle);
        noa_b200::binding::extract<nf::Layout::HC2H>(d_volume.view(), Empty{}, vlogical, b.view(), Empty{},
                                                     slogical, Empty{}, d_rot.view(), options, handle);
        stream.synchronize();
        const Array<c32> ha = a.to_cpu(), hb = b.to_cpu();
        ::noa::Stream::current(Device("cpu")).synchronize();
        std::memcpy(out_texture, ha.get(), static_cast<size_t>(sshape.n_elements()) * sizeof(c32));
        std::memcpy(out_array, hb.get(), static_cast<size_t>(sshape.n_elements()) * sizeof(c32));
        return 0;
    } catch (const std::exception& e) {
        if (err)
            std::snprintf(err, static_cast<size_t>(errlen), "%s", e.what());
        return -1;
    }
}
