// The step between insertion and the inverse FFT of a reconstruction, in one pass over the spectrum:
// value / max(weight, threshold), the remap from the inserted layout (centered "hc" or not "h") to the
// non-centered layout a c2r FFT reads, and the phase exp(-2 pi i k.c / n) with c = n / 2 per axis that
// puts the real-space origin at the volume's center (for even sizes, the factor (-1)^(kz+ky+kx)). After
// the c2r, fourier_interpolation_correction (fp_gridding.cu) finishes the reconstruction in real space.
// No function of the reference does this step; it replaces the elementwise ops, remap and fftshift a
// noa user would chain (fft/Remap.hpp).
#include "fp_args.cuh"

namespace nb {
namespace {

struct SpecArgs {
    const float2* values;
    const float* weights;      // may be null: no division
    float2* out;
    int64_t vs[3], ws[3];      // strides (d, h, w) of the inputs, in elements
    int d, h, wp, n_w;         // logical sizes; wp = n_w / 2 + 1
    bool centered;             // inputs are centered (hc)
    float threshold;
    float cz, cy, cx;          // phase centers (n / 2), as fractions of the sizes: c / n
};

__global__ void spectrum_kernel(const __grid_constant__ SpecArgs a) {
    const int64_t total = static_cast<int64_t>(a.d) * a.h * a.wp;
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int x = static_cast<int>(i % a.wp);
        const int64_t zy = i / a.wp;
        const int y = static_cast<int>(zy % a.h), z = static_cast<int>(zy / a.h);
        // Output element (z, y, x) is non-centered: its frequencies, then where they sit in the input.
        const int fz = index2frequency(false, z, a.d), fy = index2frequency(false, y, a.h);
        const int iz = frequency2index(a.centered, fz, a.d), iy = frequency2index(a.centered, fy, a.h);
        float2 v = __ldcs(a.values + iz * a.vs[0] + iy * a.vs[1] + x * a.vs[2]);
        if (a.weights) {
            const float w = fmaxf(__ldcs(a.weights + iz * a.ws[0] + iy * a.ws[1] + x * a.ws[2]), a.threshold);
            v = make_float2(v.x / w, v.y / w);
        }
        // exp(-2 pi i (fz cz + fy cy + fx cx)), the turns reduced to [-0.5, 0.5) before sincospi.
        float turns = fz * a.cz + fy * a.cy + x * a.cx;
        turns -= rintf(turns);
        float s, c;
        sincospif(-2.f * turns, &s, &c);
        __stcs(a.out + i, make_float2(v.x * c - v.y * s, v.x * s + v.y * c));
    }
}

} // namespace

cudaError_t launch_reconstruction_spectrum(const nb_array* values, const nb_array* weights,
                                           const int64_t shape[4], bool centered, float threshold,
                                           const nb_array* out, cudaStream_t stream) {
    SpecArgs a{};
    a.values = static_cast<const float2*>(values->data);
    a.weights = weights && weights->data ? static_cast<const float*>(weights->data) : nullptr;
    a.out = static_cast<float2*>(out->data);
    for (int k = 0; k < 3; ++k) {
        a.vs[k] = values->strides[k + 1];
        a.ws[k] = a.weights ? weights->strides[k + 1] : 0;
    }
    a.d = static_cast<int>(shape[1]);
    a.h = static_cast<int>(shape[2]);
    a.n_w = static_cast<int>(shape[3]);
    a.wp = a.n_w / 2 + 1;
    a.centered = centered;
    a.threshold = threshold;
    a.cz = static_cast<float>(a.d / 2) / static_cast<float>(a.d);
    a.cy = static_cast<float>(a.h / 2) / static_cast<float>(a.h);
    a.cx = static_cast<float>(a.n_w / 2) / static_cast<float>(a.n_w);
    const int64_t total = static_cast<int64_t>(a.d) * a.h * a.wp;
    const int64_t blocks = (total + 255) / 256;
    const int grid = static_cast<int>(blocks < static_cast<int64_t>(sm_count()) * 16 ? blocks : sm_count() * 16);
    if (total > 0)
        spectrum_kernel<<<grid, 256, 0, stream>>>(a);
    return cudaGetLastError();
}

} // namespace nb
