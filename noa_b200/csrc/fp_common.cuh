// Device-side building blocks of the Fourier central-slice kernels (sm_100a).
//
// Restates, for the GPU, the per-element mathematics of noa's Fourier-projection operators:
//   index <-> frequency on rfft layouts        noa/fft/core/Frequency.hpp:80-145, 258-288
//   slice <-> grid transforms                   noa/xform/FourierProject.hpp:41-95
//   windowed sinc                               noa/xform/FourierProject.hpp:99-110, 114-145
//   interpolation weights                       noa/xform/core/Interpolation.hpp:64-146
//   Friedel-aware spectrum interpolation        noa/xform/core/Interpolation.hpp:440-526
//
// Coordinates are computed with explicitly rounded single-precision operations (__fmul_rn/__fadd_rn),
// in the reference's operand order, so no multiply-add is fused: every cutoff test, window test and
// interpolation tap is then decided on exactly the value the reference's CPU path computes. The
// interpolation sums themselves are free to use FMA.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace nb {

// Interpolation families (noa Interp::Method with the _FAST bit erased).
enum InterpFamily : int { I_NEAREST = 0, I_LINEAR = 1, I_CUBIC = 2, I_BSPLINE = 3,
                          I_LANCZOS4 = 4, I_LANCZOS6 = 5, I_LANCZOS8 = 6 };

template<int I> struct InterpTraits;
template<> struct InterpTraits<I_NEAREST> { static constexpr int SIZE = 2; };
template<> struct InterpTraits<I_LINEAR> { static constexpr int SIZE = 2; };
template<> struct InterpTraits<I_CUBIC> { static constexpr int SIZE = 4; };
template<> struct InterpTraits<I_BSPLINE> { static constexpr int SIZE = 4; };
template<> struct InterpTraits<I_LANCZOS4> { static constexpr int SIZE = 4; };
template<> struct InterpTraits<I_LANCZOS6> { static constexpr int SIZE = 6; };
template<> struct InterpTraits<I_LANCZOS8> { static constexpr int SIZE = 8; };

// ---------------------------------------------------------------------------------------------------
// Kernel-argument views.
// ---------------------------------------------------------------------------------------------------

// A read-only input addressed by 3 indices (batch-or-depth, height, width). `value` replaces the data
// for constant inputs. Complex values are float2 (noa's Complex<f32> layout).
struct SrcView {
    const void* data;
    int64_t s0, s1, s2;
    float2 value;
    int is_value;
    int present;
};

struct DstView {
    void* data;
    int64_t s0, s1, s2;
    int present;
};

// Per-slice transforms in noa's layout (see fourier_project.h). count == 1 broadcasts.
struct XformView {
    const float* data;     // nullptr -> inline
    int64_t count;
    int kind;              // 0 none, 1 mat22, 2 mat33 (48-byte stride), 3 quaternion
    float inline_value[9];
};

template<bool CPLX>
__device__ __forceinline__ float2 src_read(const SrcView& s, int64_t i0, int64_t i1, int64_t i2) {
    if (s.is_value)
        return s.value;
    const int64_t off = i0 * s.s0 + i1 * s.s1 + i2 * s.s2;
    if constexpr (CPLX) {
        return __ldg(static_cast<const float2*>(s.data) + off);
    } else {
        return make_float2(__ldg(static_cast<const float*>(s.data) + off), 0.f);
    }
}

__device__ __forceinline__ float src_read_real(const SrcView& s, int64_t i0, int64_t i1, int64_t i2) {
    if (s.is_value)
        return s.value.x;
    return __ldg(static_cast<const float*>(s.data) + (i0 * s.s0 + i1 * s.s1 + i2 * s.s2));
}

// ---------------------------------------------------------------------------------------------------
// Exactly rounded arithmetic helpers (no contraction).
// ---------------------------------------------------------------------------------------------------
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
// ((a0*b0) + (a1*b1)) + (a2*b2): noa's left-folded dot product.
__device__ __forceinline__ float dot3(float a0, float a1, float a2, float b0, float b1, float b2) {
    return add(add(mul(a0, b0), mul(a1, b1)), mul(a2, b2));
}
__device__ __forceinline__ float dot2(float a0, float a1, float b0, float b1) {
    return add(mul(a0, b0), mul(a1, b1));
}

// ---------------------------------------------------------------------------------------------------
// Frequencies (Frequency.hpp).
// ---------------------------------------------------------------------------------------------------
__device__ __forceinline__ int index2frequency(bool centered, int i, int n) {
    return centered ? i - n / 2 : (i < (n + 1) / 2 ? i : i - n);
}
__device__ __forceinline__ int frequency2index(bool centered, int f, int n) {
    return centered ? f + n / 2 : (f < 0 ? f + n : f);
}

// ---------------------------------------------------------------------------------------------------
// Transforms (Transform.hpp:201-218, Mat.hpp:420-424, Quaternion.hpp:167-181).
// ---------------------------------------------------------------------------------------------------
struct Mat33 { float m[9]; };
struct Quat { float z, y, x, w; };

__device__ __forceinline__ const float* xform_ptr(const XformView& x, int64_t batch, int stride) {
    if (!x.data)
        return x.inline_value;
    return x.data + (x.count == 1 ? 0 : batch) * stride;
}

// Rotation of the (z, y, x) vector v by slice `batch`'s matrix or quaternion, in place.
__device__ __forceinline__ void rotate(const XformView& r, int64_t batch, float& v0, float& v1, float& v2) {
    if (r.kind == 3) {
        const float* q = xform_ptr(r, batch, 4);
        const float z = q[0], y = q[1], x = q[2], w = q[3];
        const float s0 = sub(add(mul(w, v2), mul(y, v0)), mul(z, v1));
        const float s1 = sub(add(mul(w, v1), mul(z, v2)), mul(x, v0));
        const float s2 = sub(add(mul(w, v0), mul(x, v1)), mul(y, v2));
        const float r0 = add(v0, mul(2.f, sub(mul(x, s1), mul(y, s0))));
        const float r1 = add(v1, mul(2.f, sub(mul(z, s0), mul(x, s2))));
        const float r2 = add(v2, mul(2.f, sub(mul(y, s2), mul(z, s1))));
        v0 = r0; v1 = r1; v2 = r2;
    } else {
        const float* m = xform_ptr(r, batch, 12);
        const float r0 = dot3(m[0], m[1], m[2], v0, v1, v2);
        const float r1 = dot3(m[3], m[4], m[5], v0, v1, v2);
        const float r2 = dot3(m[6], m[7], m[8], v0, v1, v2);
        v0 = r0; v1 = r1; v2 = r2;
    }
}

__device__ __forceinline__ void scale2(const XformView& s, int64_t batch, float& f0, float& f1) {
    if (s.kind != 1)
        return;
    const float* m = xform_ptr(s, batch, 4);
    const float a = dot2(m[0], m[1], f0, f1);
    const float b = dot2(m[2], m[3], f0, f1);
    f0 = a;
    f1 = b;
}

struct Ews { int on; float d0, d1; };

// fourier_slice2grid (FourierProject.hpp:41-68).
__device__ __forceinline__ void slice2grid(float f0, float f1, const XformView& scale, const XformView& rot,
                                           int64_t batch, const Ews& ews, float& z, float& y, float& x) {
    scale2(scale, batch, f0, f1);
    z = 0.f;
    if (ews.on)
        z = add(mul(mul(ews.d0, f0), f0), mul(mul(ews.d1, f1), f1));
    y = f0;
    x = f1;
    rotate(rot, batch, z, y, x);
}

// Row 0 of the (inverse) rotation of slice i, so that grid2slice's fz = row . f.
__device__ __forceinline__ float3 rotation_row0(const XformView& r, int64_t i) {
    if (r.kind == 3) {
        float a0 = 1.f, a1 = 0.f, a2 = 0.f;
        float b0 = 0.f, b1 = 1.f, b2 = 0.f;
        float c0 = 0.f, c1 = 0.f, c2 = 1.f;
        rotate(r, i, a0, a1, a2);
        rotate(r, i, b0, b1, b2);
        rotate(r, i, c0, c1, c2);
        return make_float3(a0, b0, c0);
    }
    const float* m = xform_ptr(r, i, 12);
    return make_float3(m[0], m[1], m[2]);
}

// fourier_grid2slice (FourierProject.hpp:71-95): returns fz, and the 2-D frequency in (f0, f1).
__device__ __forceinline__ float grid2slice(float z, float y, float x, const XformView& scale,
                                            const XformView& rot, int64_t batch, const Ews& ews,
                                            float& f0, float& f1) {
    rotate(rot, batch, z, y, x);
    f0 = y;
    f1 = x;
    if (ews.on)
        z = sub(z, add(mul(mul(ews.d0, f0), f0), mul(mul(ews.d1, f1), f1)));
    scale2(scale, batch, f0, f1);
    return z;
}

// windowed_sinc (FourierProject.hpp:99-110).
__device__ __forceinline__ float windowed_sinc(float fftfreq, float fftfreq_sinc, float fftfreq_blackman) {
    constexpr float PI = 3.1415926535897932384626433832795f;
    fftfreq = mul(fftfreq, PI);
    const float xs = div(fftfreq, fftfreq_sinc);
    const float sinc = xs == 0.f ? 1.f : div(sinf(xs), xs);
    const float bc = div(fftfreq, fftfreq_blackman);
    const float blackman = add(add(0.42f, mul(0.5f, cosf(bc))), mul(0.08f, cosf(mul(2.f, bc))));
    return mul(sinc, blackman);
}

// The same window for the hot loops of the windowed-sinc insertions, where it only scales a term (the
// |fftfreq| <= fftfreq_blackman decision is taken before, on exactly rounded coordinates, and the window
// is 0 at that bound, so nothing discontinuous depends on it): the divisions by fftfreq_sinc and
// fftfreq_blackman become products with pi / fftfreq_sinc and pi / fftfreq_blackman, the sinc's
// division an approximate one, cos(2 b) is 2 cos(b)^2 - 1, and the Blackman cosine, whose argument
// stays within [-pi, pi], is the hardware approximation __cosf (6-10 % faster insertions). The sinc's
// sine is not __sinf: its argument reaches several pi, where __sinf's error grew the insertions' error
// to 1e-4. Relative difference from windowed_sinc: a few 1e-7.
// SINPI: the sinc's sine as sinpif(fftfreq * (1 / fftfreq_sinc)) rather than sinf(xs): 8.5 % faster in
// the gather insertion and 5.5 % in insert_and_extract, 11 % slower in the scatter form (each measured
// in one call), so those two use it; the two forms differ by 2e-7 (relative L2). sinpif's argument is
// the sinc's phase in units of pi, rounded twice (the reciprocal, then the product), and xs only feeds
// the division.
template<bool SINPI = false>
__device__ __forceinline__ float windowed_sinc_fast(float fftfreq, float pi_over_sinc, float inv_sinc,
                                                    float pi_over_blackman) {
    const float xs = fftfreq * pi_over_sinc;
    const float sn = SINPI ? sinpif(fftfreq * inv_sinc) : sinf(xs);
    const float sinc = xs == 0.f ? 1.f : __fdividef(sn, xs);
    const float c = __cosf(fftfreq * pi_over_blackman);
    const float blackman = 0.42f + 0.5f * c + 0.08f * (2.f * c * c - 1.f);
    return sinc * blackman;
}

// ---------------------------------------------------------------------------------------------------
// Interpolation weights (Interpolation.hpp:64-146), per axis. Rounded like the reference; they feed
// only the (continuous) interpolation sums.
// ---------------------------------------------------------------------------------------------------
template<int I>
__device__ __forceinline__ void interp_weights(float f, float* w) {
    if constexpr (I == I_LINEAR) {
        w[0] = sub(1.f, f);
        w[1] = f;
    } else if constexpr (I == I_CUBIC) {
        constexpr float A = -0.5f;
        const float f1 = add(f, 1.f);
        w[0] = sub(mul(add(mul(sub(mul(A, f1), 5 * A), f1), 8 * A), f1), 4 * A);
        w[1] = add(mul(mul(sub(mul(A + 2, f), A + 3), f), f), 1.f);
        const float g = sub(1.f, f);
        w[2] = add(mul(mul(sub(mul(A + 2, g), A + 3), g), g), 1.f);
        w[3] = sub(sub(sub(1.f, w[0]), w[1]), w[2]);
    } else if constexpr (I == I_BSPLINE) {
        const float ONE_SIXTH = 1.f / 6.f;
        const float TWO_THIRD = 2.f / 3.f;
        const float one_minus = sub(1.f, f);
        const float one_squared = mul(one_minus, one_minus);
        const float squared = mul(f, f);
        w[0] = mul(mul(ONE_SIXTH, one_squared), one_minus);
        w[1] = sub(TWO_THIRD, mul(mul(0.5f, squared), sub(2.f, f)));
        w[2] = sub(TWO_THIRD, mul(mul(0.5f, one_squared), sub(2.f, one_minus)));
        w[3] = mul(mul(ONE_SIXTH, squared), f);
    } else {
        constexpr int SIZE = InterpTraits<I>::SIZE;
        constexpr int CENTER = SIZE / 2 - 1;
        constexpr float PI = 3.1415926535897932384626433832795f;
        constexpr float S45 = 0.7071067811865475f;
        constexpr float CS[8][2] = {{1, 0}, {-S45, -S45}, {0, 1}, {S45, -S45},
                                    {-1, 0}, {S45, S45}, {0, -1}, {-S45, S45}};
        constexpr float EPS = 1.1920928955078125e-07f;
#pragma unroll
        for (int i = 0; i < SIZE; ++i)
            w[i] = 0.f;
        float sum = 0.f;
        if (f <= EPS) {
            w[CENTER] = 1.f;
            sum = 1.f;
        } else if (f >= sub(1.f, EPS)) {
            w[CENTER + 1] = 1.f;
            sum = 1.f;
        } else {
            const float x0 = -add(f, static_cast<float>(CENTER));
            const float y0 = mul(mul(x0, PI), 0.25f);
            float s, c;
            sincosf(y0, &s, &c);
#pragma unroll
            for (int i = 0; i < SIZE; ++i) {
                const float fij = -sub(add(f, static_cast<float>(CENTER)), static_cast<float>(i));
                const float yj = mul(mul(fij, PI), 0.25f);
                w[i] = div(add(mul(CS[i][0], s), mul(CS[i][1], c)), mul(yj, yj));
                sum = add(sum, w[i]);
            }
        }
        const float inv = div(1.f, sum);
#pragma unroll
        for (int i = 0; i < SIZE; ++i)
            w[i] = mul(w[i], inv);
    }
}

__device__ __forceinline__ float2 cmul(float2 a, float s) { return make_float2(s * a.x, s * a.y); }
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 cfma(float2 a, float s, float2 acc) {
    return make_float2(fmaf(s, a.x, acc.x), fmaf(s, a.y, acc.y));
}

// Spectrum geometry of one rfft input: logical sizes (last one is the full width) and centering.
struct Spectrum3 { int n0, n1, n2; bool centered; };
struct Spectrum2 { int n0, n1; bool centered; bool narrow = false; };  // narrow: in-slice offsets fit 32 bits

// Reads elements of one slice of a stack: with `narrow`, from the slice's base pointer with 32-bit
// in-slice offsets (the stack itself may span more than 2^31 elements); else through src_read.
template<bool CPLX>
struct SliceReader {
    const SrcView& src;
    int64_t batch;
    const void* base;
    int s1, s2;
    bool narrow;

    __device__ __forceinline__ SliceReader(const SrcView& s, int64_t b, bool n)
        : src(s), batch(b), narrow(n && !s.is_value) {
        base = narrow ? static_cast<const void*>(static_cast<const char*>(s.data) +
                                                 b * s.s0 * static_cast<int64_t>(CPLX ? sizeof(float2) : sizeof(float)))
                      : nullptr;
        s1 = static_cast<int>(s.s1);
        s2 = static_cast<int>(s.s2);
    }
    __device__ __forceinline__ float2 operator()(int i1, int i2) const {
        if (narrow) {
            const int off = i1 * s1 + i2 * s2;
            if constexpr (CPLX)
                return __ldg(static_cast<const float2*>(base) + off);
            else
                return make_float2(__ldg(static_cast<const float*>(base) + off), 0.f);
        }
        return src_read<CPLX>(src, batch, i1, i2);
    }
};

// ---------------------------------------------------------------------------------------------------
// interpolate_spectrum, 3-D (volume) form. `freq` is in samples, centered on DC.
// ---------------------------------------------------------------------------------------------------
template<int I, bool CPLX>
__device__ __forceinline__ float2 interp_spectrum_3d(const SrcView& src, const Spectrum3& sp,
                                                     float f0, float f1, float f2) {
    constexpr int SIZE = InterpTraits<I>::SIZE;
    constexpr bool FLIP_EARLY = SIZE <= 2;
    const int lo0 = -sp.n0 / 2, hi0 = (sp.n0 - 1) / 2;
    const int lo1 = -sp.n1 / 2, hi1 = (sp.n1 - 1) / 2;
    const int hi2 = sp.n2 / 2;
    float conjugate = 1.f;
    if (FLIP_EARLY && f2 < 0.f) {
        f0 = -f0; f1 = -f1; f2 = -f2;
        conjugate = -1.f;
    }
    if constexpr (I == I_NEAREST) {
        // NEAREST returns before the early-flip conjugation (Interpolation.hpp:480-485).
        const int i0 = static_cast<int>(roundf(f0));
        const int i1 = static_cast<int>(roundf(f1));
        const int i2 = static_cast<int>(roundf(f2));
        float2 v = make_float2(0.f, 0.f);
        if (i0 >= lo0 && i0 <= hi0 && i1 >= lo1 && i1 <= hi1 && i2 >= 0 && i2 <= hi2)
            v = src_read<CPLX>(src, frequency2index(sp.centered, i0, sp.n0),
                               frequency2index(sp.centered, i1, sp.n1), i2);
        return v;
    } else {
        constexpr int START = -(SIZE - 1) / 2;
        const float fl0 = floorf(f0), fl1 = floorf(f1), fl2 = floorf(f2);
        const int b0 = static_cast<int>(fl0), b1 = static_cast<int>(fl1), b2 = static_cast<int>(fl2);
        float w0[SIZE], w1[SIZE], w2[SIZE];
        interp_weights<I>(sub(f0, fl0), w0);
        interp_weights<I>(sub(f1, fl1), w1);
        interp_weights<I>(sub(f2, fl2), w2);
        float2 value = make_float2(0.f, 0.f);
        // Windows of 6 and 8 taps keep the z loop rolled: 216/512 unrolled taps only cost registers
        // and compile time, these modes are arithmetic-bound either way.
#pragma unroll (SIZE <= 4 ? SIZE : 1)
        for (int z = 0; z < SIZE; ++z) {
            float2 vz = make_float2(0.f, 0.f);
#pragma unroll
            for (int y = 0; y < SIZE; ++y) {
                float2 vy = make_float2(0.f, 0.f);
#pragma unroll
                for (int x = 0; x < SIZE; ++x) {
                    int t0 = b0 + START + z, t1 = b1 + START + y, t2 = b2 + START + x;
                    float conj = 1.f;
                    if (!FLIP_EARLY && t2 < 0) {
                        t0 = -t0; t1 = -t1; t2 = -t2;
                        conj = -1.f;
                    }
                    if (t0 >= lo0 && t0 <= hi0 && t1 >= lo1 && t1 <= hi1 && t2 >= 0 && t2 <= hi2) {
                        float2 v = src_read<CPLX>(src, frequency2index(sp.centered, t0, sp.n0),
                                                  frequency2index(sp.centered, t1, sp.n1), t2);
                        if (!FLIP_EARLY)
                            v.y *= conj;
                        vy = cfma(v, w2[x], vy);
                    }
                }
                vz = cfma(vy, w1[y], vz);
            }
            value = cfma(vz, w0[z], value);
        }
        if (FLIP_EARLY)
            value.y *= conjugate;
        return value;
    }
}

// interpolate_spectrum, 2-D (slice) form; `batch` selects the slice.
template<int I, bool CPLX>
__device__ __forceinline__ float2 interp_spectrum_2d(const SrcView& src, const Spectrum2& sp, int64_t batch,
                                                     float f0, float f1) {
    constexpr int SIZE = InterpTraits<I>::SIZE;
    constexpr bool FLIP_EARLY = SIZE <= 2;
    const int lo0 = -sp.n0 / 2, hi0 = (sp.n0 - 1) / 2;
    const int hi1 = sp.n1 / 2;
    const SliceReader<CPLX> read(src, batch, sp.narrow);
    float conjugate = 1.f;
    if (FLIP_EARLY && f1 < 0.f) {
        f0 = -f0; f1 = -f1;
        conjugate = -1.f;
    }
    if constexpr (I == I_NEAREST) {
        const int i0 = static_cast<int>(roundf(f0));
        const int i1 = static_cast<int>(roundf(f1));
        float2 v = make_float2(0.f, 0.f);
        if (i0 >= lo0 && i0 <= hi0 && i1 >= 0 && i1 <= hi1)
            v = read(frequency2index(sp.centered, i0, sp.n0), i1);
        return v;
    } else {
        constexpr int START = -(SIZE - 1) / 2;
        const float fl0 = floorf(f0), fl1 = floorf(f1);
        const int b0 = static_cast<int>(fl0), b1 = static_cast<int>(fl1);
        float w0[SIZE], w1[SIZE];
        interp_weights<I>(sub(f0, fl0), w0);
        interp_weights<I>(sub(f1, fl1), w1);
        float2 value = make_float2(0.f, 0.f);
        {
            // Interior fast path (all taps in bounds, none flipped per tap): same terms, same order.
            constexpr int END = SIZE / 2;
            if (b0 + START >= lo0 && b0 + END <= hi0 && b1 + START >= 0 && b1 + END <= hi1) {
#pragma unroll
                for (int y = 0; y < SIZE; ++y) {
                    const int iy = frequency2index(sp.centered, b0 + START + y, sp.n0);
                    float2 vy = make_float2(0.f, 0.f);
#pragma unroll
                    for (int x = 0; x < SIZE; ++x)
                        vy = cfma(read(iy, b1 + START + x), w1[x], vy);
                    value = cfma(vy, w0[y], value);
                }
                if (FLIP_EARLY)
                    value.y *= conjugate;
                return value;
            }
        }
#pragma unroll
        for (int y = 0; y < SIZE; ++y) {
            float2 vy = make_float2(0.f, 0.f);
#pragma unroll
            for (int x = 0; x < SIZE; ++x) {
                int t0 = b0 + START + y, t1 = b1 + START + x;
                float conj = 1.f;
                if (!FLIP_EARLY && t1 < 0) {
                    t0 = -t0; t1 = -t1;
                    conj = -1.f;
                }
                if (t0 >= lo0 && t0 <= hi0 && t1 >= 0 && t1 <= hi1) {
                    float2 v = read(frequency2index(sp.centered, t0, sp.n0), t1);
                    if (!FLIP_EARLY)
                        v.y *= conj;
                    vy = cfma(v, w1[x], vy);
                }
            }
            value = cfma(vy, w0[y], value);
        }
        if (FLIP_EARLY)
            value.y *= conjugate;
        return value;
    }
}

// ---------------------------------------------------------------------------------------------------
// Lean 3-D reads: offsets in Idx (int32 when the array fits, else int64), no constant-value branch.
// ---------------------------------------------------------------------------------------------------
template<typename Idx>
struct View3 {
    const void* data;
    Idx s0, s1, s2;
};

// Read-only 16-byte load whose line is kept in L2 with evict_last priority for half of the lines.
// Volumes (and their pair copies) are about the size of the L2 or larger while the output slices
// stream past them; keeping part of them resident saves re-reads (bit-identical; 1 % per extraction
// call, 7 % for batched launches over pair copies).
__device__ __forceinline__ float4 ldg_evict_last_half(const float4* p) {
    unsigned long long pol;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 0.5;" : "=l"(pol));
    // The policy touches no memory and may be hoisted; the load is volatile so that it is never
    // speculated above the bounds tests that guard it (a tap's address is only valid when they pass).
    float4 v;
    asm volatile("ld.global.nc.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(p), "l"(pol));
    return v;
}

template<bool CPLX, typename Idx>
__device__ __forceinline__ float2 view_read(const View3<Idx>& v, Idx off) {
    if constexpr (CPLX)
        return __ldg(static_cast<const float2*>(v.data) + off);
    else
        return make_float2(__ldg(static_cast<const float*>(v.data) + off), 0.f);
}

// interpolate_spectrum<LINEAR>, 3-D, rfft input (Interpolation.hpp:440-526): early Friedel flip, 2x2x2
// taps with per-axis bounds and frequency2index done once per axis, sums in the reference's order.
template<bool CPLX, typename Idx>
__device__ __forceinline__ float2 interp_linear_3d(const View3<Idx>& v, const Spectrum3& sp,
                                                   float q0, float q1, float q2) {
    float conjugate = 1.f;
    if (q2 < 0.f) {
        q0 = -q0; q1 = -q1; q2 = -q2;
        conjugate = -1.f;
    }
    const float fl0 = floorf(q0), fl1 = floorf(q1), fl2 = floorf(q2);
    const int b0 = static_cast<int>(fl0), b1 = static_cast<int>(fl1), b2 = static_cast<int>(fl2);
    const float t0 = sub(q0, fl0), t1 = sub(q1, fl1), t2 = sub(q2, fl2);
    const float w0[2] = {sub(1.f, t0), t0};
    const float w1[2] = {sub(1.f, t1), t1};
    const float w2[2] = {sub(1.f, t2), t2};
    const int lo0 = -sp.n0 / 2, hi0 = (sp.n0 - 1) / 2;
    const int lo1 = -sp.n1 / 2, hi1 = (sp.n1 - 1) / 2;
    const int hi2 = sp.n2 / 2;
    bool ok0[2], ok1[2], ok2[2];
    Idx o0[2], o1[2], o2[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const int z = b0 + k, y = b1 + k, x = b2 + k;
        ok0[k] = z >= lo0 && z <= hi0;
        ok1[k] = y >= lo1 && y <= hi1;
        ok2[k] = x >= 0 && x <= hi2;
        o0[k] = static_cast<Idx>(frequency2index(sp.centered, z, sp.n0)) * v.s0;
        o1[k] = static_cast<Idx>(frequency2index(sp.centered, y, sp.n1)) * v.s1;
        o2[k] = static_cast<Idx>(x) * v.s2;
    }
    float2 value = make_float2(0.f, 0.f);
#pragma unroll
    for (int z = 0; z < 2; ++z) {
        float2 vz = make_float2(0.f, 0.f);
#pragma unroll
        for (int y = 0; y < 2; ++y) {
            float2 vy = make_float2(0.f, 0.f);
#pragma unroll
            for (int x = 0; x < 2; ++x) {
                if (ok0[z] && ok1[y] && ok2[x])
                    vy = cfma(view_read<CPLX>(v, o0[z] + o1[y] + o2[x]), w2[x], vy);
            }
            vz = cfma(vy, w1[y], vz);
        }
        value = cfma(vz, w0[z], value);
    }
    value.y *= conjugate;
    return value;
}

// Generic interpolate_spectrum, 3-D, on a View3 (any window).
template<int I, bool CPLX, typename Idx>
__device__ __forceinline__ float2 interp_3d(const View3<Idx>& v, const Spectrum3& sp, float f0, float f1, float f2) {
    if constexpr (I == I_LINEAR) {
        return interp_linear_3d<CPLX>(v, sp, f0, f1, f2);
    } else {
        constexpr int SIZE = InterpTraits<I>::SIZE;
        constexpr bool FLIP_EARLY = SIZE <= 2;
        const int lo0 = -sp.n0 / 2, hi0 = (sp.n0 - 1) / 2;
        const int lo1 = -sp.n1 / 2, hi1 = (sp.n1 - 1) / 2;
        const int hi2 = sp.n2 / 2;
        float conjugate = 1.f;
        if (FLIP_EARLY && f2 < 0.f) {
            f0 = -f0; f1 = -f1; f2 = -f2;
            conjugate = -1.f;
        }
        if constexpr (I == I_NEAREST) {
            // NEAREST returns before the early-flip conjugation (Interpolation.hpp:480-485).
            const int i0 = static_cast<int>(roundf(f0));
            const int i1 = static_cast<int>(roundf(f1));
            const int i2 = static_cast<int>(roundf(f2));
            float2 r = make_float2(0.f, 0.f);
            if (i0 >= lo0 && i0 <= hi0 && i1 >= lo1 && i1 <= hi1 && i2 >= 0 && i2 <= hi2)
                r = view_read<CPLX>(v, static_cast<Idx>(frequency2index(sp.centered, i0, sp.n0)) * v.s0 +
                                       static_cast<Idx>(frequency2index(sp.centered, i1, sp.n1)) * v.s1 +
                                       static_cast<Idx>(i2) * v.s2);
            return r;
        } else {
            constexpr int START = -(SIZE - 1) / 2;
            const float fl0 = floorf(f0), fl1 = floorf(f1), fl2 = floorf(f2);
            const int b0 = static_cast<int>(fl0), b1 = static_cast<int>(fl1), b2 = static_cast<int>(fl2);
            float w0[SIZE], w1[SIZE], w2[SIZE];
            interp_weights<I>(sub(f0, fl0), w0);
            interp_weights<I>(sub(f1, fl1), w1);
            interp_weights<I>(sub(f2, fl2), w2);
            float2 value = make_float2(0.f, 0.f);
            constexpr int END = SIZE / 2;
            // Interior fast path: every tap in bounds and on the stored half (no per-tap Friedel
            // flip), so each (z, y) row of the window is SIZE consecutive x elements. Same terms in the
            // same order as the general loop below, hence the same bits.
            if (b0 + START >= lo0 && b0 + END <= hi0 && b1 + START >= lo1 && b1 + END <= hi1 &&
                b2 + START >= 0 && b2 + END <= hi2) {
                const Idx x0 = static_cast<Idx>(b2 + START) * v.s2;
                // With contiguous x and a 16-byte aligned volume, a row of SIZE complex values is read
                // as SIZE/2 aligned 16-byte loads from the even element at or before its start, plus
                // one 8-byte load when the start is odd: fewer, wider loads than SIZE 8-byte ones.
                constexpr bool WIDE = CPLX && SIZE % 2 == 0;
                const bool wide = WIDE && v.s2 == 1 && (reinterpret_cast<uintptr_t>(v.data) & 15) == 0;
#pragma unroll (SIZE <= 4 ? SIZE : 1)
                for (int z = 0; z < SIZE; ++z) {
                    const Idx oz = static_cast<Idx>(frequency2index(sp.centered, b0 + START + z, sp.n0)) * v.s0 + x0;
                    float2 vz = make_float2(0.f, 0.f);
#pragma unroll
                    for (int y = 0; y < SIZE; ++y) {
                        const Idx row = oz + static_cast<Idx>(frequency2index(sp.centered, b1 + START + y, sp.n1)) * v.s1;
                        float2 vy = make_float2(0.f, 0.f);
                        if constexpr (WIDE) {
                            if (wide) {
                                const bool odd = (row & 1) != 0;
                                const float2* e = static_cast<const float2*>(v.data) + (row - (odd ? 1 : 0));
                                float4 q[SIZE / 2];
#pragma unroll
                                for (int j = 0; j < SIZE / 2; ++j)
                                    q[j] = ldg_evict_last_half(reinterpret_cast<const float4*>(e) + j);
                                const float2 last = odd ? __ldg(e + SIZE) : make_float2(0.f, 0.f);
#pragma unroll
                                for (int x = 0; x < SIZE; ++x) {
                                    // element x of the row: element x + odd of the loaded run
                                    const int i0 = x, i1 = x + 1;
                                    const float2 even = (i0 & 1) ? make_float2(q[i0 / 2].z, q[i0 / 2].w)
                                                                 : make_float2(q[i0 / 2].x, q[i0 / 2].y);
                                    const float2 shifted = i1 == SIZE ? last
                                        : ((i1 & 1) ? make_float2(q[i1 / 2].z, q[i1 / 2].w)
                                                    : make_float2(q[i1 / 2].x, q[i1 / 2].y));
                                    vy = cfma(odd ? shifted : even, w2[x], vy);
                                }
                                vz = cfma(vy, w1[y], vz);
                                continue;
                            }
                        }
#pragma unroll
                        for (int x = 0; x < SIZE; ++x)
                            vy = cfma(view_read<CPLX>(v, row + static_cast<Idx>(x) * v.s2), w2[x], vy);
                        vz = cfma(vy, w1[y], vz);
                    }
                    value = cfma(vz, w0[z], value);
                }
                return value;
            }
#pragma unroll 1
            for (int z = 0; z < SIZE; ++z) {
                float2 vz = make_float2(0.f, 0.f);
#pragma unroll (SIZE <= 4 ? SIZE : 1)
                for (int y = 0; y < SIZE; ++y) {
                    float2 vy = make_float2(0.f, 0.f);
#pragma unroll
                    for (int x = 0; x < SIZE; ++x) {
                        int t0 = b0 + START + z, t1 = b1 + START + y, t2 = b2 + START + x;
                        float conj = 1.f;
                        if (!FLIP_EARLY && t2 < 0) {
                            t0 = -t0; t1 = -t1; t2 = -t2;
                            conj = -1.f;
                        }
                        if (t0 >= lo0 && t0 <= hi0 && t1 >= lo1 && t1 <= hi1 && t2 >= 0 && t2 <= hi2) {
                            float2 val = view_read<CPLX>(
                                v, static_cast<Idx>(frequency2index(sp.centered, t0, sp.n0)) * v.s0 +
                                   static_cast<Idx>(frequency2index(sp.centered, t1, sp.n1)) * v.s1 +
                                   static_cast<Idx>(t2) * v.s2);
                            if (!FLIP_EARLY)
                                val.y *= conj;
                            vy = cfma(val, w2[x], vy);
                        }
                    }
                    vz = cfma(vy, w1[y], vz);
                }
                value = cfma(vz, w0[z], value);
            }
            if (FLIP_EARLY)
                value.y *= conjugate;
            return value;
        }
    }
}

// cast_or_abs_squared (base/Math.hpp:220-225): complex -> real stores |z|^2.
template<bool IN_CPLX, bool OUT_CPLX>
__device__ __forceinline__ float2 to_output(float2 v) {
    if constexpr (IN_CPLX && !OUT_CPLX)
        return make_float2(v.x * v.x + v.y * v.y, 0.f);
    else
        return v;
}

template<bool CPLX>
__device__ __forceinline__ void dst_store(const DstView& d, int64_t i0, int64_t i1, int64_t i2, float2 v) {
    const int64_t off = i0 * d.s0 + i1 * d.s1 + i2 * d.s2;
    if constexpr (CPLX)
        static_cast<float2*>(d.data)[off] = v;
    else
        static_cast<float*>(d.data)[off] = v.x;
}

template<bool CPLX>
__device__ __forceinline__ float2 dst_load(const DstView& d, int64_t i0, int64_t i1, int64_t i2) {
    const int64_t off = i0 * d.s0 + i1 * d.s1 + i2 * d.s2;
    if constexpr (CPLX)
        return static_cast<const float2*>(d.data)[off];
    else
        return make_float2(static_cast<const float*>(d.data)[off], 0.f);
}

// Streaming (evict-first) variants, for data touched once per launch (output slices, input slices),
// so that it does not push the reused working set (volume, accumulator) out of L2.
template<bool CPLX>
__device__ __forceinline__ void dst_store_stream(const DstView& d, int64_t i0, int64_t i1, int64_t i2, float2 v) {
    const int64_t off = i0 * d.s0 + i1 * d.s1 + i2 * d.s2;
    if constexpr (CPLX)
        __stcs(static_cast<float2*>(d.data) + off, v);
    else
        __stcs(static_cast<float*>(d.data) + off, v.x);
}

__device__ __forceinline__ void store_real_stream(const DstView& d, int64_t i0, int64_t i1, int64_t i2, float v) {
    __stcs(static_cast<float*>(d.data) + (i0 * d.s0 + i1 * d.s1 + i2 * d.s2), v);
}

template<bool CPLX>
__device__ __forceinline__ float2 src_read_stream(const SrcView& s, int64_t i0, int64_t i1, int64_t i2) {
    if (s.is_value)
        return s.value;
    const int64_t off = i0 * s.s0 + i1 * s.s1 + i2 * s.s2;
    if constexpr (CPLX)
        return __ldcs(static_cast<const float2*>(s.data) + off);
    else
        return make_float2(__ldcs(static_cast<const float*>(s.data) + off), 0.f);
}

__device__ __forceinline__ void store_real(const DstView& d, int64_t i0, int64_t i1, int64_t i2, float v) {
    static_cast<float*>(d.data)[i0 * d.s0 + i1 * d.s1 + i2 * d.s2] = v;
}

__device__ __forceinline__ float load_real(const DstView& d, int64_t i0, int64_t i1, int64_t i2) {
    return static_cast<const float*>(d.data)[i0 * d.s0 + i1 * d.s1 + i2 * d.s2];
}

} // namespace nb
