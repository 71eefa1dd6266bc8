// fourier_interpolation_correction on sm_100a (noa/xform/FourierProject.hpp:2062-2087, operator
// GriddingCorrection :1009-1061): the real-space correction of the trilinear gridding kernel. Per
// voxel (b, j, k, l): dist = ((j, k, l) - half) / shape, half = shape / 2 (0 where a size is 1),
// r = |dist|, sinc2 = sinc(pi r)^2 (noa::sinc is 1 at 0, base/Math.hpp:28-29); the output is
// value / sinc2 (post-correction) or value * sinc2. Memory-bound elementwise: one read and one write
// per voxel, coalesced along l; in place is allowed. The coordinates are rounded like the reference's
// f32 operator (no contraction), so the factors differ from it only through sinf.
#include "fp_args.cuh"

namespace nb {
namespace {

struct Grid4 {
    const float* in;
    float* out;
    int64_t is[4], os[4];     // strides in elements (input strides are 0 along broadcast dimensions)
    int64_t n[4];             // output shape
    float f[3], half[3];
    float value;              // constant input when in == nullptr
    int post;
};

__global__ void gridding_correction_kernel(const __grid_constant__ Grid4 g) {
    constexpr float PI = 3.1415926535897932384626433832795f;
    const int64_t total = g.n[0] * g.n[1] * g.n[2] * g.n[3];
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t l = i % g.n[3];
        const int64_t t = i / g.n[3];
        const int64_t k = t % g.n[2];
        const int64_t t2 = t / g.n[2];
        const int64_t j = t2 % g.n[1];
        const int64_t b = t2 / g.n[1];
        const float d0 = div(sub(static_cast<float>(j), g.half[0]), g.f[0]);
        const float d1 = div(sub(static_cast<float>(k), g.half[1]), g.f[1]);
        const float d2 = div(sub(static_cast<float>(l), g.half[2]), g.f[2]);
        const float radius = __fsqrt_rn(dot3(d0, d1, d2, d0, d1, d2));
        const float x = mul(PI, radius);
        const float sinc = x == 0.f ? 1.f : div(sinf(x), x);
        const float sinc2 = mul(sinc, sinc);
        const float v = g.in ? g.in[b * g.is[0] + j * g.is[1] + k * g.is[2] + l * g.is[3]] : g.value;
        g.out[b * g.os[0] + j * g.os[1] + k * g.os[2] + l * g.os[3]] = g.post ? div(v, sinc2) : mul(v, sinc2);
    }
}

} // namespace

cudaError_t launch_gridding_correction(const nb_array* input, const nb_array* output, bool post,
                                       cudaStream_t stream) {
    Grid4 g{};
    g.in = input->is_value ? nullptr : static_cast<const float*>(input->data);
    g.out = static_cast<float*>(output->data);
    g.value = static_cast<float>(input->value[0]);
    for (int d = 0; d < 4; ++d) {
        g.n[d] = output->shape[d];
        g.os[d] = output->strides[d];
        g.is[d] = input->is_value || input->shape[d] == 1 ? 0 : input->strides[d];
    }
    for (int d = 0; d < 3; ++d) {
        g.f[d] = static_cast<float>(output->shape[d + 1]);
        g.half[d] = output->shape[d + 1] == 1 ? 0.f : g.f[d] / 2.f;
    }
    g.post = post ? 1 : 0;
    const int64_t total = g.n[0] * g.n[1] * g.n[2] * g.n[3];
    if (total == 0)
        return cudaSuccess;
    const int64_t blocks = (total + 255) / 256;
    const int grid = static_cast<int>(blocks < static_cast<int64_t>(sm_count()) * 16 ? blocks : sm_count() * 16);
    gridding_correction_kernel<<<grid, 256, 0, stream>>>(g);
    return cudaGetLastError();
}

} // namespace nb
