/* ORACLE TEST INFRASTRUCTURE — included twice by fp_oracle.c, once per precision.
 *
 * Before inclusion: R (float|double), SFX (_f32|_f64), and the math names R_FLOOR, R_ROUND, R_SIN,
 * R_COS, R_FABS, R_EPS. Every floating-point expression below keeps the operand order of the reference
 * so that, compiled with -ffp-contract=off, it rounds exactly like noa's CPU path. The reference lines
 * each block restates are cited next to it (paths relative to the noa source tree, src/noa/).
 */

#define CAT2_(a, b) a##b
#define CAT_(a, b) CAT2_(a, b)
#define F_(name) CAT_(name, SFX)

typedef struct { R re, im; } F_(cpx);
#define cpx_t F_(cpx)
#define FPO_DECLARE_X(N, S) FPO_DECLARE(N, S)

static inline cpx_t F_(c_make)(R re, R im) { cpx_t c; c.re = re; c.im = im; return c; }
static inline cpx_t F_(c_add)(cpx_t a, cpx_t b) { return F_(c_make)(a.re + b.re, a.im + b.im); }
/* Complex * real: base/Complex.hpp:203-216 ({s*re, s*im}). */
static inline cpx_t F_(c_scale)(cpx_t a, R s) { return F_(c_make)(s * a.re, s * a.im); }

/* ---------------------------------------------------------------------------------------------------
 * Reading an input (array, constant value, or absent).
 * ------------------------------------------------------------------------------------------------- */
typedef struct {
    const R* data;
    int is_complex, is_value, present;
    int64_t s0, s1, s2;       /* strides of the 3 addressed dims (batch-or-depth, height, width) */
    cpx_t value;
} F_(src);

static F_(src) F_(make_src)(const fpo_array* a, int dim0) {
    /* dim0: which BDHW dim is the first addressed one (0 for slices: b,h,w; 1 for volumes: d,h,w). */
    F_(src) s;
    memset(&s, 0, sizeof(s));
    if (!a || (!a->data && !a->is_value))
        return s;
    s.present = 1;
    s.is_complex = a->dtype == FPO_COMPLEX;
    s.is_value = a->is_value;
    s.value = F_(c_make)((R) a->value[0], s.is_complex ? (R) a->value[1] : (R) 0);
    s.data = (const R*) a->data;
    s.s0 = a->strides[dim0];
    s.s1 = a->strides[2];
    s.s2 = a->strides[3];
    return s;
}

static inline cpx_t F_(src_read)(const F_(src)* s, int64_t i0, int64_t i1, int64_t i2) {
    if (s->is_value)
        return s->value;
    const int64_t off = i0 * s->s0 + i1 * s->s1 + i2 * s->s2;
    if (s->is_complex)
        return F_(c_make)(s->data[2 * off], s->data[2 * off + 1]);
    return F_(c_make)(s->data[off], (R) 0);
}

typedef struct { R* data; int is_complex, present; int64_t s0, s1, s2; } F_(dst);

static F_(dst) F_(make_dst)(const fpo_array* a, int dim0) {
    F_(dst) d;
    memset(&d, 0, sizeof(d));
    if (!a || !a->data)
        return d;
    d.present = 1;
    d.is_complex = a->dtype == FPO_COMPLEX;
    d.data = (R*) a->data;
    d.s0 = a->strides[dim0];
    d.s1 = a->strides[2];
    d.s2 = a->strides[3];
    return d;
}

/* cast_or_abs_squared (base/Math.hpp:220-225, base/Complex.hpp:398-402): complex->real stores |z|^2. */
static inline cpx_t F_(to_output)(cpx_t v, int in_complex, int out_complex) {
    if (in_complex && !out_complex)
        return F_(c_make)(v.re * v.re + v.im * v.im, (R) 0);
    return v;
}

static inline void F_(dst_store)(const F_(dst)* d, int64_t i0, int64_t i1, int64_t i2, cpx_t v) {
    const int64_t off = i0 * d->s0 + i1 * d->s1 + i2 * d->s2;
    if (d->is_complex) { d->data[2 * off] = v.re; d->data[2 * off + 1] = v.im; }
    else d->data[off] = v.re;
}

static inline void F_(dst_add)(const F_(dst)* d, int64_t i0, int64_t i1, int64_t i2, cpx_t v) {
    const int64_t off = i0 * d->s0 + i1 * d->s1 + i2 * d->s2;
    if (d->is_complex) { d->data[2 * off] += v.re; d->data[2 * off + 1] += v.im; }
    else d->data[off] += v.re;
}

static inline cpx_t F_(dst_load)(const F_(dst)* d, int64_t i0, int64_t i1, int64_t i2) {
    const int64_t off = i0 * d->s0 + i1 * d->s1 + i2 * d->s2;
    if (d->is_complex) return F_(c_make)(d->data[2 * off], d->data[2 * off + 1]);
    return F_(c_make)(d->data[off], (R) 0);
}

/* ---------------------------------------------------------------------------------------------------
 * Transforms: Mat22 scaling, Mat33 / quaternion rotation (xform/core/Transform.hpp:201-218,
 * base/Mat.hpp:420-424 with the left-folded dot of base/Vec.hpp:846-855, xform/core/Quaternion.hpp:167-181).
 * ------------------------------------------------------------------------------------------------- */
typedef struct { int kind; const R* data; int64_t count; R value[9]; } F_(xform);

static F_(xform) F_(make_xform)(const fpo_transform* t) {
    F_(xform) x;
    memset(&x, 0, sizeof(x));
    if (!t)
        return x;
    x.kind = t->kind;
    x.data = (const R*) t->data;
    x.count = t->count;
    for (int i = 0; i < 9; ++i)
        x.value[i] = (R) t->value[i];
    return x;
}

static inline const R* F_(xform_at)(const F_(xform)* x, int64_t batch) {
    /* Element strides of noa's types: Mat22 4 values, Quaternion 4, Mat33 9 values padded to its
     * 16-byte alignment (Mat33<f32>: 48 bytes, Mat33<f64>: 80 bytes). */
    const int n = x->kind == FPO_MAT33 ? R_MAT33_STRIDE : 4;
    if (!x->data)
        return x->value;
    return x->data + (x->count == 1 ? 0 : batch) * n;
}

static inline void F_(apply_scale)(const F_(xform)* s, int64_t b, R f[2]) {
    if (s->kind != FPO_MAT22)
        return;
    const R* m = F_(xform_at)(s, b);
    const R f0 = f[0], f1 = f[1];
    f[0] = m[0] * f0 + m[1] * f1;
    f[1] = m[2] * f0 + m[3] * f1;
}

static inline void F_(apply_rotation)(const F_(xform)* r, int64_t b, R v[3]) {
    const R* m = F_(xform_at)(r, b);
    const R v0 = v[0], v1 = v[1], v2 = v[2];
    if (r->kind == FPO_MAT33) {
        v[0] = m[0] * v0 + m[1] * v1 + m[2] * v2;
        v[1] = m[3] * v0 + m[4] * v1 + m[5] * v2;
        v[2] = m[6] * v0 + m[7] * v1 + m[8] * v2;
    } else { /* quaternion, stored z, y, x, w */
        const R z = m[0], y = m[1], x = m[2], w = m[3];
        const R s0 = w * v2 + y * v0 - z * v1;
        const R s1 = w * v1 + z * v2 - x * v0;
        const R s2 = w * v0 + x * v1 - y * v2;
        const R two = 2;
        v[0] = v0 + two * (x * s1 - y * s0);
        v[1] = v1 + two * (z * s0 - x * s2);
        v[2] = v2 + two * (y * s2 - z * s1);
    }
}

/* EWS curvature coefficient 1/(2*radius) in the coordinate type (FourierProject.hpp:227-228,459-460). */
typedef struct { int on; R d[2]; } F_(ews);

static F_(ews) F_(make_ews)(const double radius[2]) {
    F_(ews) e;
    e.on = radius[0] != 0 || radius[1] != 0;
    const R r0 = (R) radius[0], r1 = (R) radius[1];
    if (r0 != 0 || r1 != 0) {
        e.d[0] = 1 / (2 * r0);
        e.d[1] = 1 / (2 * r1);
    } else {
        e.d[0] = 0;
        e.d[1] = 0;
    }
    return e;
}

/* fourier_slice2grid (FourierProject.hpp:41-68). With neither scale nor EWS, both are Empty. */
static inline void F_(slice2grid)(R f2_0, R f2_1, const F_(xform)* scale, const F_(xform)* rot,
                                  int64_t b, const F_(ews)* ews, R out[3]) {
    R f2[2] = {f2_0, f2_1};
    F_(apply_scale)(scale, b, f2);
    out[0] = 0;
    out[1] = f2[0];
    out[2] = f2[1];
    if (ews->on)
        out[0] = ews->d[0] * f2[0] * f2[0] + ews->d[1] * f2[1] * f2[1];
    F_(apply_rotation)(rot, b, out);
}

/* fourier_grid2slice (FourierProject.hpp:71-95). */
static inline void F_(grid2slice)(const R f3_in[3], const F_(xform)* scale, const F_(xform)* rot,
                                  int64_t b, const F_(ews)* ews, R* fz, R f2[2]) {
    R f3[3] = {f3_in[0], f3_in[1], f3_in[2]};
    F_(apply_rotation)(rot, b, f3);
    f2[0] = f3[1];
    f2[1] = f3[2];
    R z = f3[0];
    if (ews->on)
        z -= ews->d[0] * f2[0] * f2[0] + ews->d[1] * f2[1] * f2[1];
    F_(apply_scale)(scale, b, f2);
    *fz = z;
}

/* windowed_sinc (FourierProject.hpp:99-110) with noa::sinc (base/Math.hpp:28-29). */
static inline R F_(windowed_sinc)(R fftfreq, R fftfreq_sinc, R fftfreq_blackman) {
    const R PI = (R) 3.1415926535897932384626433832795;
    fftfreq *= PI;
    const R xs = fftfreq / fftfreq_sinc;
    const R sinc = xs == 0 ? (R) 1 : R_SIN(xs) / xs;
    const R bc = fftfreq / fftfreq_blackman;
    const R blackman = (R) 0.42 + (R) 0.5 * R_COS(bc) + (R) 0.08 * R_COS(2 * bc);
    return sinc * blackman;
}

/* ---------------------------------------------------------------------------------------------------
 * Spectrum interpolation on rfft layouts (xform/core/Interpolation.hpp:64-146, 440-526;
 * fft/core/Frequency.hpp:80-145, 258-288).
 * ------------------------------------------------------------------------------------------------- */
static inline int64_t F_(i2f)(int centered, int64_t i, int64_t n) {
    if (centered)
        return i - n / 2;
    return i < (n + 1) / 2 ? i : i - n;
}

static inline int64_t F_(f2i)(int centered, int64_t f, int64_t n) {
    if (centered)
        return f + n / 2;
    return f < 0 ? f + n : f;
}

static int F_(window_size)(int interp) {
    const int m = interp >= 100 ? interp - 100 : interp;
    switch (m) {
        case 0: case 1: return 2;
        case 2: case 3: case 4: return 4;
        case 5: return 6;
        case 6: return 8;
        default: return 0;
    }
}

/* interpolation_weights: w[k] for tap k = START..END of one axis, given the fraction f. */
static void F_(interp_weights)(int interp, R f, R* w) {
    const int m = interp >= 100 ? interp - 100 : interp;
    if (m == 1) {
        w[0] = 1 - f;
        w[1] = f;
    } else if (m == 2) {
        const R A = (R) -0.5;
        w[0] = ((A * (f + 1) - 5 * A) * (f + 1) + 8 * A) * (f + 1) - 4 * A;
        w[1] = ((A + 2) * f - (A + 3)) * f * f + 1;
        w[2] = ((A + 2) * (1 - f) - (A + 3)) * (1 - f) * (1 - f) + 1;
        w[3] = 1 - w[0] - w[1] - w[2];
    } else if (m == 3) {
        const R ONE_SIXTH = (R) 1 / (R) 6;
        const R TWO_THIRD = (R) 2 / (R) 3;
        const R one_minus = 1 - f;
        const R one_squared = one_minus * one_minus;
        const R squared = f * f;
        w[0] = ONE_SIXTH * one_squared * one_minus;
        w[1] = TWO_THIRD - (R) 0.5 * squared * (2 - f);
        w[2] = TWO_THIRD - (R) 0.5 * one_squared * (2 - one_minus);
        w[3] = ONE_SIXTH * squared * f;
    } else {
        /* Lanczos windows: one sincos per axis and the rotation table of the reference
         * (Interpolation.hpp:102-141). */
        const int size = F_(window_size)(interp);
        const int center = size / 2 - 1;
        const R PI = (R) 3.1415926535897932384626433832795;
        const R s45 = (R) 0.7071067811865475;
        const R cs[8][2] = {{1, 0}, {-s45, -s45}, {0, 1}, {s45, -s45}, {-1, 0}, {s45, s45}, {0, -1}, {-s45, s45}};
        for (int i = 0; i < size; ++i)
            w[i] = 0;
        R sum = 0;
        if (f <= R_EPS) {
            w[center] = 1;
            sum = 1;
        } else if (f >= 1 - R_EPS) {
            w[center + 1] = 1;
            sum = 1;
        } else {
            const R x0 = -(f + (R) center);
            const R y0 = x0 * PI * (R) 0.25;
            const R s = R_SIN(y0), c = R_COS(y0);
            for (int i = 0; i < size; ++i) {
                const R fij = -(f + (R) center - (R) i);
                const R yj = fij * PI * (R) 0.25;
                w[i] = (cs[i][0] * s + cs[i][1] * c) / (yj * yj);
                sum += w[i];
            }
        }
        const R inv = 1 / sum;
        for (int i = 0; i < size; ++i)
            w[i] *= inv;
    }
}

/* One tap of interpolate_spectrum::update_at: per-index Friedel flip for windows > 2, bound test,
 * frequency2index, conj, accumulate. `ndim` is 2 or 3; the last dim is the rfft half-width. */
static inline void F_(tap)(const F_(src)* in, int64_t batch, int ndim, const int64_t shape[3], int centered,
                           int flip_per_index, int64_t f0, int64_t f1, int64_t f2, R weight, cpx_t* out) {
    int64_t f[3] = {f0, f1, f2};
    R conj = 1;
    if (flip_per_index && f[ndim - 1] < 0) {
        for (int i = 0; i < ndim; ++i)
            f[i] = -f[i];
        conj = -1;
    }
    for (int i = 0; i < ndim - 1; ++i) {
        if (f[i] < -shape[i] / 2 || f[i] > (shape[i] - 1) / 2)
            return;
    }
    if (f[ndim - 1] < 0 || f[ndim - 1] > shape[ndim - 1] / 2)
        return;
    cpx_t v;
    if (ndim == 3)
        v = F_(src_read)(in, F_(f2i)(centered, f[0], shape[0]), F_(f2i)(centered, f[1], shape[1]), f[2]);
    else
        v = F_(src_read)(in, batch, F_(f2i)(centered, f[0], shape[0]), f[1]);
    if (flip_per_index)
        v.im *= conj;
    *out = F_(c_add)(*out, F_(c_scale)(v, weight));
}

/* interpolate_spectrum<REMAP, INTERP, N> (Interpolation.hpp:440-526). `freq` is in samples, centered.
 * For N=2 the batch selects the slice; for N=3 it is ignored. */
static cpx_t F_(interp_spectrum)(const F_(src)* in, int64_t batch, int ndim, const int64_t shape[3],
                                 int centered, int interp, const R freq_in[3]) {
    const int size = F_(window_size)(interp);
    const int flip_early = size <= 2;
    const int m = interp >= 100 ? interp - 100 : interp;
    R freq[3] = {freq_in[0], freq_in[1], ndim == 3 ? freq_in[2] : 0};
    R conjugate = 1;
    if (flip_early && freq[ndim - 1] < 0) {
        for (int i = 0; i < ndim; ++i)
            freq[i] *= -1;
        conjugate = -1;
    }
    cpx_t value = F_(c_make)(0, 0);
    if (m == 0) {
        /* NEAREST returns before the early-flip conjugation (Interpolation.hpp:480-485). */
        int64_t idx[3];
        for (int i = 0; i < ndim; ++i)
            idx[i] = (int64_t) R_ROUND(freq[i]);
        F_(tap)(in, batch, ndim, shape, centered, 0, idx[0], idx[1], ndim == 3 ? idx[2] : 0, 1, &value);
        return value;
    }
    const int start = -(size - 1) / 2;
    const int end = size / 2;
    int64_t base[3];
    R w[3][8];
    for (int i = 0; i < ndim; ++i) {
        const R fl = R_FLOOR(freq[i]);
        base[i] = (int64_t) fl;
        F_(interp_weights)(interp, freq[i] - fl, w[i]);
    }
    const int flip_per_index = size > 2;
    if (ndim == 3) {
        for (int z = start; z <= end; ++z) {
            cpx_t vz = F_(c_make)(0, 0);
            for (int y = start; y <= end; ++y) {
                cpx_t vy = F_(c_make)(0, 0);
                for (int x = start; x <= end; ++x)
                    F_(tap)(in, batch, 3, shape, centered, flip_per_index,
                            base[0] + z, base[1] + y, base[2] + x, w[2][x - start], &vy);
                vz = F_(c_add)(vz, F_(c_scale)(vy, w[1][y - start]));
            }
            value = F_(c_add)(value, F_(c_scale)(vz, w[0][z - start]));
        }
    } else {
        for (int y = start; y <= end; ++y) {
            cpx_t vy = F_(c_make)(0, 0);
            for (int x = start; x <= end; ++x)
                F_(tap)(in, batch, 2, shape, centered, flip_per_index,
                        base[0] + y, base[1] + x, 0, w[1][x - start], &vy);
            value = F_(c_add)(value, F_(c_scale)(vy, w[0][y - start]));
        }
    }
    if (flip_early)
        value.im *= conjugate;
    return value;
}

/* blackman_window_size (FourierProject.hpp:114-137), computed in double. */
static int64_t F_(blackman_window_size)(R fftfreq_blackman, R spectrum_size) {
    double samples = (double) spectrum_size * (double) fftfreq_blackman;
    const double diff = fabs(samples - 1.);
    const int close = isfinite(diff) && (diff <= 1e-6 || diff <= fmax(fabs(samples), 1.) * (DBL_EPSILON * 2));
    samples = close ? round(samples) : ceil(samples);
    int64_t n = (int64_t) samples;
    if (n < 1)
        n = 1;
    return 2 * n + 1 - 2;
}

static inline R F_(w_offset)(int64_t w, int64_t window_size, R spectrum_size) {
    return (R) (w - window_size / 2) / spectrum_size;
}

static inline void F_(target3)(const fpo_options* o, const int64_t grid_shape4[4], R t[3]) {
    const int64_t* ts = o->target_shape;
    const int any0 = ts[0] == 0 || ts[1] == 0 || ts[2] == 0 || ts[3] == 0;
    for (int i = 0; i < 3; ++i)
        t[i] = (R) (any0 ? grid_shape4[i + 1] : ts[i + 1]);
}

static inline R F_(cutoff_sqd)(const fpo_options* o) {
    R c = (R) o->fftfreq_cutoff;
    c = c > 0 ? c : 0;
    return c * c;
}

static inline R F_(rmax)(R a, R b) { return a < b ? b : a; }

/* ---------------------------------------------------------------------------------------------------
 * rasterize_central_slices_3d: FourierInsertRasterize (FourierProject.hpp:238-373).
 * Serial, in the reference's single-thread order (batch, y, u) so that sums round identically.
 * Deviation: the reference bounds the u tap by the LOGICAL width, so taps at u = W/2+1 (zero weight for
 * even W at cutoff <= 0.5) land in the next row or past the end; here (and on the GPU) they are dropped.
 * ------------------------------------------------------------------------------------------------- */
FPO_DECLARE_X(fpo_rasterize, SFX) {
    (void) scale2; (void) rotation2; (void) n_threads;
    if (!input || !output || !output->data || !rotation)
        return -1;
    const int slices_centered = (remap & 4) != 0;
    const int volume_centered = (remap & 8) != 0;
    const F_(src) in = F_(make_src)(input, 0);
    const F_(src) in_w = F_(make_src)(input_weight, 0);
    const F_(dst) vol = F_(make_dst)(output, 1);
    const F_(dst) vol_w = F_(make_dst)(output_weight, 1);
    const F_(xform) sc = F_(make_xform)(scale);
    const F_(xform) rot = F_(make_xform)(rotation);
    const int any_scale = sc.kind == FPO_MAT22;
    const F_(ews) ews = F_(make_ews)(options->ews_radius);
    const F_(xform) sc_eff = (any_scale || ews.on) ? sc : F_(make_xform)(NULL);
    const F_(ews) ews_eff = ews;
    const int64_t D = output_shape[1], H = output_shape[2], W = output_shape[3];
    const int64_t B = input_shape[0], Hs = input_shape[2], Ws = input_shape[3];
    const int64_t Wp = W / 2 + 1;
    R target[3];
    F_(target3)(options, output_shape, target);
    const R fs0 = (R) Hs, fs1 = (R) Ws;
    const R cutoff_sqd = F_(cutoff_sqd)(options);
    const int in_complex = in.is_complex, out_complex = vol.is_complex;

    for (int64_t b = 0; b < B; ++b) {
        for (int64_t y = 0; y < Hs; ++y) {
            for (int64_t u = 0; u < Ws / 2 + 1; ++u) {
                const int64_t v = F_(i2f)(slices_centered, y, Hs);
                R f3[3];
                F_(slice2grid)((R) v / fs0, (R) u / fs1, &sc_eff, &rot, b, &ews_eff, f3);
                if (f3[0] * f3[0] + f3[1] * f3[1] + f3[2] * f3[2] > cutoff_sqd)
                    continue;
                R conjugate = 1;
                if (f3[2] < 0) {
                    f3[0] = -f3[0]; f3[1] = -f3[1]; f3[2] = -f3[2];
                    if (in_complex)
                        conjugate = -1;
                }
                R freq[3] = {f3[0] * target[0], f3[1] * target[1], f3[2] * target[2]};
                cpx_t value = F_(src_read)(&in, b, y, u);
                if (in_complex && out_complex)
                    value = F_(c_scale)(value, conjugate);
                else
                    value = F_(to_output)(value, in_complex, out_complex);
                R weight = 0;
                if (vol_w.present)
                    weight = in_w.present ? F_(src_read)(&in_w, b, y, u).re : (R) 1;

                int64_t base0[3];
                R frac[2][3];
                for (int i = 0; i < 3; ++i) {
                    base0[i] = (int64_t) R_FLOOR(freq[i]);
                    frac[1][i] = freq[i] - (R) base0[i];
                    frac[0][i] = 1 - frac[1][i];
                }
                R kernel[2][2][2];
                for (int w = 0; w < 2; ++w)
                    for (int vv = 0; vv < 2; ++vv)
                        for (int uu = 0; uu < 2; ++uu)
                            kernel[w][vv][uu] = frac[w][0] * frac[vv][1] * frac[uu][2];
                for (int w = 0; w < 2; ++w) {
                    for (int vv = 0; vv < 2; ++vv) {
                        for (int uu = 0; uu < 2; ++uu) {
                            const int64_t iw = F_(f2i)(volume_centered, base0[0] + w, D);
                            const int64_t iv = F_(f2i)(volume_centered, base0[1] + vv, H);
                            const int64_t iu = base0[2] + uu;
                            if (iw >= 0 && iw < D && iv >= 0 && iv < H && iu >= 0 && iu < Wp) {
                                const R k = kernel[w][vv][uu];
                                F_(dst_add)(&vol, iw, iv, iu, F_(c_scale)(value, k));
                                if (vol_w.present)
                                    F_(dst_add)(&vol_w, iw, iv, iu, F_(c_make)(weight * k, 0));
                            }
                        }
                    }
                }
                if (base0[2] == 0) {
                    cpx_t cv = value;
                    if (out_complex)
                        cv.im = -cv.im;
                    for (int w = 0; w < 2; ++w) {
                        for (int vv = 0; vv < 2; ++vv) {
                            const int64_t iw = F_(f2i)(volume_centered, -(base0[0] + w), D);
                            const int64_t iv = F_(f2i)(volume_centered, -(base0[1] + vv), H);
                            if (iw >= 0 && iw < D && iv >= 0 && iv < H) {
                                const R k = kernel[w][vv][0];
                                F_(dst_add)(&vol, iw, iv, 0, F_(c_scale)(cv, k));
                                if (vol_w.present)
                                    F_(dst_add)(&vol_w, iw, iv, 0, F_(c_make)(weight * k, 0));
                            }
                        }
                    }
                }
            }
        }
    }
    return 0;
}

/* ---------------------------------------------------------------------------------------------------
 * insert_central_slices_3d: FourierInsertInterpolate (FourierProject.hpp:445-519). Gather per voxel.
 * ------------------------------------------------------------------------------------------------- */
FPO_DECLARE_X(fpo_insert, SFX) {
    if (F_(window_size)(options->interp) == 0)
        return -1;
    (void) scale2; (void) rotation2;
    if (!input || !output || !output->data || !rotation)
        return -1;
    const int slices_centered = (remap & 4) != 0;
    const int volume_centered = (remap & 8) != 0;
    const F_(src) in = F_(make_src)(input, 0);
    const F_(src) in_w = F_(make_src)(input_weight, 0);
    const F_(dst) vol = F_(make_dst)(output, 1);
    const F_(dst) vol_w = F_(make_dst)(output_weight, 1);
    const F_(xform) sc = F_(make_xform)(scale);
    const F_(xform) rot = F_(make_xform)(rotation);
    const F_(ews) ews = F_(make_ews)(options->ews_radius);
    const F_(xform) sc_eff = (sc.kind == FPO_MAT22 || ews.on) ? sc : F_(make_xform)(NULL);
    const int64_t D = output_shape[1], H = output_shape[2], W = output_shape[3];
    const int64_t B = input_shape[0];
    const int64_t slice_shape[3] = {input_shape[2], input_shape[3], 0};
    R target[3];
    F_(target3)(options, output_shape, target);
    const R fsl0 = (R) input_shape[2], fsl1 = (R) input_shape[3];
    const R cutoff_sqd = F_(cutoff_sqd)(options);
    R tmin = target[0];
    if (target[1] < tmin) tmin = target[1];
    if (target[2] < tmin) tmin = target[2];
    const R fsinc = F_(rmax)((R) options->fftfreq_sinc, 1 / tmin);
    const R fblack = F_(rmax)((R) options->fftfreq_blackman, 1 / tmin);
    const int in_complex = in.is_complex, out_complex = vol.is_complex;
    const int64_t Wp = W / 2 + 1;

    #pragma omp parallel for collapse(2) schedule(static) num_threads(n_threads > 0 ? n_threads : 1)
    for (int64_t z = 0; z < D; ++z) {
        for (int64_t y = 0; y < H; ++y) {
            for (int64_t x = 0; x < Wp; ++x) {
                const R f[3] = {(R) F_(i2f)(volume_centered, z, D) / target[0],
                                (R) F_(i2f)(volume_centered, y, H) / target[1],
                                (R) x / target[2]};
                if (f[0] * f[0] + f[1] * f[1] + f[2] * f[2] > cutoff_sqd)
                    continue;
                cpx_t value = F_(c_make)(0, 0);
                R weights = 0;
                for (int64_t i = 0; i < B; ++i) {
                    R fz, f2[2];
                    F_(grid2slice)(f, &sc_eff, &rot, i, &ews, &fz, f2);
                    cpx_t iv = F_(c_make)(0, 0);
                    R iw = 0;
                    if (R_FABS(fz) <= fblack) {
                        const R window = F_(windowed_sinc)(fz, fsinc, fblack);
                        const R fr[3] = {f2[0] * fsl0, f2[1] * fsl1, 0};
                        iv = F_(c_scale)(F_(interp_spectrum)(&in, i, 2, slice_shape, slices_centered,
                                                             options->interp, fr), window);
                        if (vol_w.present) {
                            if (in_w.present)
                                iw = F_(interp_spectrum)(&in_w, i, 2, slice_shape, slices_centered,
                                                         options->interp, fr).re * window;
                            else
                                iw = window;
                        }
                    }
                    value = F_(c_add)(value, iv);
                    if (vol_w.present)
                        weights += iw;
                }
                const cpx_t outv = F_(to_output)(value, in_complex, out_complex);
                const cpx_t old = F_(dst_load)(&vol, z, y, x);
                F_(dst_store)(&vol, z, y, x, F_(c_add)(old, outv));
                if (vol_w.present)
                    F_(dst_add)(&vol_w, z, y, x, F_(c_make)(weights, 0));
            }
        }
    }
    return 0;
}

/* ---------------------------------------------------------------------------------------------------
 * extract_central_slices_3d: FourierExtract (FourierProject.hpp:599-694), 3-D and w-windowed forms.
 * The w-windowed form sums over w in increasing order per pixel, the order of the reference's serial
 * 4-D iwise (outputs zeroed first, FourierProject.hpp:1442-1452).
 * ------------------------------------------------------------------------------------------------- */
FPO_DECLARE_X(fpo_extract, SFX) {
    if (F_(window_size)(options->interp) == 0)
        return -1;
    (void) scale2; (void) rotation2;
    if (!input || !output || !output->data || !rotation)
        return -1;
    const int volume_centered = (remap & 4) != 0;
    const int slices_centered = (remap & 8) != 0;
    const F_(src) vol = F_(make_src)(input, 1);
    const F_(src) vol_w = F_(make_src)(input_weight, 1);
    const F_(dst) out = F_(make_dst)(output, 0);
    const F_(dst) out_w = F_(make_dst)(output_weight, 0);
    const F_(xform) sc = F_(make_xform)(scale);
    const F_(xform) rot = F_(make_xform)(rotation);
    const F_(ews) ews = F_(make_ews)(options->ews_radius);
    const F_(xform) sc_eff = (sc.kind == FPO_MAT22 || ews.on) ? sc : F_(make_xform)(NULL);
    const int64_t vshape[3] = {input_shape[1], input_shape[2], input_shape[3]};
    const int64_t B = output_shape[0], Hs = output_shape[2], Ws = output_shape[3];
    R target[3];
    F_(target3)(options, input_shape, target);
    const R fs0 = (R) Hs, fs1 = (R) Ws;
    const R cutoff_sqd = F_(cutoff_sqd)(options);
    const R fsinc = F_(rmax)((R) options->w_fftfreq_sinc, 1 / target[0]);
    const R fblack = F_(rmax)((R) options->w_fftfreq_blackman, 1 / target[0]);
    const int64_t wsize = F_(blackman_window_size)(fblack, target[0]);
    const int in_complex = vol.is_complex, out_complex = out.is_complex;

    #pragma omp parallel for collapse(2) schedule(static) num_threads(n_threads > 0 ? n_threads : 1)
    for (int64_t b = 0; b < B; ++b) {
        for (int64_t y = 0; y < Hs; ++y) {
            for (int64_t x = 0; x < Ws / 2 + 1; ++x) {
                const int64_t v = F_(i2f)(slices_centered, y, Hs);
                R f3[3];
                F_(slice2grid)((R) v / fs0, (R) x / fs1, &sc_eff, &rot, b, &ews, f3);
                cpx_t value = F_(c_make)(0, 0);
                R weight = 0;
                if (wsize <= 1) {
                    if (f3[0] * f3[0] + f3[1] * f3[1] + f3[2] * f3[2] <= cutoff_sqd) {
                        const R fr[3] = {f3[0] * target[0], f3[1] * target[1], f3[2] * target[2]};
                        value = F_(to_output)(F_(interp_spectrum)(&vol, 0, 3, vshape, volume_centered,
                                                                  options->interp, fr),
                                              in_complex, out_complex);
                        if (out_w.present)
                            weight = vol_w.present ?
                                     F_(interp_spectrum)(&vol_w, 0, 3, vshape, volume_centered,
                                                         options->interp, fr).re : (R) 1;
                    }
                } else {
                    for (int64_t w = 0; w < wsize; ++w) {
                        const R off = F_(w_offset)(w, wsize, target[0]);
                        const R g[3] = {f3[0] + off, f3[1], f3[2]};
                        if (g[0] * g[0] + g[1] * g[1] + g[2] * g[2] > cutoff_sqd)
                            continue;
                        const R fr[3] = {g[0] * target[0], g[1] * target[1], g[2] * target[2]};
                        const R cw = F_(windowed_sinc)(off, fsinc, fblack);
                        const cpx_t iv = F_(to_output)(F_(interp_spectrum)(&vol, 0, 3, vshape, volume_centered,
                                                                           options->interp, fr),
                                                       in_complex, out_complex);
                        value = F_(c_add)(value, F_(c_scale)(iv, cw));
                        if (out_w.present) {
                            const R iw = vol_w.present ?
                                         F_(interp_spectrum)(&vol_w, 0, 3, vshape, volume_centered,
                                                             options->interp, fr).re : (R) 1;
                            weight += iw * cw;
                        }
                    }
                }
                F_(dst_store)(&out, b, y, x, value);
                if (out_w.present)
                    F_(dst_store)(&out_w, b, y, x, F_(c_make)(weight, 0));
            }
        }
    }
    return 0;
}

/* ---------------------------------------------------------------------------------------------------
 * insert_and_extract_central_slices_3d: FourierInsertExtract (FourierProject.hpp:790-977).
 * ------------------------------------------------------------------------------------------------- */
static void F_(sample_virtual)(const F_(src)* in, const F_(src)* in_w, const int64_t in_shape2[3],
                               int in_centered, int interp, int64_t n_in,
                               const F_(xform)* sc, const F_(xform)* rot, const F_(ews)* ews,
                               R fsinc, R fblack, R fin0, R fin1, const R f3[3], int correct,
                               cpx_t* value_out, R* weight_out) {
    cpx_t value = F_(c_make)(0, 0);
    R weight = 0;
    for (int64_t i = 0; i < n_in; ++i) {
        R fz, f2[2];
        F_(grid2slice)(f3, sc, rot, i, ews, &fz, f2);
        if (R_FABS(fz) < fblack) {
            const R ws = F_(windowed_sinc)(fz, fsinc, fblack);
            const R fr[3] = {f2[0] * fin0, f2[1] * fin1, 0};
            value = F_(c_add)(value, F_(c_scale)(F_(interp_spectrum)(in, i, 2, in_shape2, in_centered, interp, fr), ws));
            if (in_w->present)
                weight += F_(interp_spectrum)(in_w, i, 2, in_shape2, in_centered, interp, fr).re * ws;
            else
                weight += ws;
        }
    }
    if (correct) {
        R aw = R_FABS(weight);
        const R fw = aw < 1 ? (R) 1 : aw;
        value.re = value.re / fw;
        value.im = value.im / fw;
    }
    *value_out = value;
    *weight_out = weight;
}

FPO_DECLARE_X(fpo_insert_extract, SFX) {
    if (F_(window_size)(options->interp) == 0)
        return -1;
    if (!input || !output || !output->data || !rotation || !rotation2)
        return -1;
    const int in_centered = (remap & 4) != 0;
    const int out_centered = (remap & 8) != 0;
    const F_(src) in = F_(make_src)(input, 0);
    const F_(src) in_w = F_(make_src)(input_weight, 0);
    const F_(dst) out = F_(make_dst)(output, 0);
    const F_(dst) out_w = F_(make_dst)(output_weight, 0);
    const F_(xform) sc_in = F_(make_xform)(scale);
    const F_(xform) rot_in = F_(make_xform)(rotation);
    const F_(xform) sc_out = F_(make_xform)(scale2);
    const F_(xform) rot_out = F_(make_xform)(rotation2);
    const F_(ews) ews = F_(make_ews)(options->ews_radius);
    const int any = sc_in.kind == FPO_MAT22 || sc_out.kind == FPO_MAT22 || ews.on;
    const F_(xform) none = F_(make_xform)(NULL);
    const F_(xform) sc_in_eff = any ? sc_in : none;
    const F_(xform) sc_out_eff = any ? sc_out : none;
    const int64_t in_shape2[3] = {input_shape[2], input_shape[3], 0};
    const int64_t n_in = input_shape[0];
    const int64_t B = output_shape[0], Ho = output_shape[2], Wo = output_shape[3];
    const R fin0 = (R) input_shape[2], fin1 = (R) input_shape[3];
    const R fo0 = (R) Ho, fo1 = (R) Wo;
    const R cutoff_sqd = F_(cutoff_sqd)(options);
    const R vz = (R) (Ho < Wo ? Ho : Wo);
    const R ifs = F_(rmax)((R) options->fftfreq_sinc, 1 / vz);
    const R ifb = F_(rmax)((R) options->fftfreq_blackman, 1 / vz);
    const R efs = F_(rmax)((R) options->w_fftfreq_sinc, 1 / vz);
    const R efb = F_(rmax)((R) options->w_fftfreq_blackman, 1 / vz);
    const int64_t ebs = F_(blackman_window_size)(efb, vz);
    const int add = options->add_to_output != 0;
    const int in_complex = in.is_complex, out_complex = out.is_complex;
    if (ebs > 1 && options->correct_weights)
        return -1;

    #pragma omp parallel for collapse(2) schedule(static) num_threads(n_threads > 0 ? n_threads : 1)
    for (int64_t b = 0; b < B; ++b) {
        for (int64_t y = 0; y < Ho; ++y) {
            for (int64_t x = 0; x < Wo / 2 + 1; ++x) {
                const int64_t v = F_(i2f)(out_centered, y, Ho);
                R f3[3];
                F_(slice2grid)((R) v / fo0, (R) x / fo1, &sc_out_eff, &rot_out, b, &ews, f3);
                if (ebs <= 1) {
                    if (f3[0] * f3[0] + f3[1] * f3[1] + f3[2] * f3[2] > cutoff_sqd) {
                        if (!add) {
                            F_(dst_store)(&out, b, y, x, F_(c_make)(0, 0));
                            if (out_w.present)
                                F_(dst_store)(&out_w, b, y, x, F_(c_make)(0, 0));
                        }
                        continue;
                    }
                    cpx_t value;
                    R weight;
                    F_(sample_virtual)(&in, &in_w, in_shape2, in_centered, options->interp, n_in,
                                       &sc_in_eff, &rot_in, &ews, ifs, ifb, fin0, fin1, f3,
                                       options->correct_weights, &value, &weight);
                    const cpx_t ov = F_(to_output)(value, in_complex, out_complex);
                    if (add)
                        F_(dst_store)(&out, b, y, x, F_(c_add)(F_(dst_load)(&out, b, y, x), ov));
                    else
                        F_(dst_store)(&out, b, y, x, ov);
                    if (out_w.present) {
                        if (add)
                            F_(dst_add)(&out_w, b, y, x, F_(c_make)(weight, 0));
                        else
                            F_(dst_store)(&out_w, b, y, x, F_(c_make)(weight, 0));
                    }
                } else {
                    cpx_t acc = add ? F_(dst_load)(&out, b, y, x) : F_(c_make)(0, 0);
                    R accw = (add && out_w.present) ? F_(dst_load)(&out_w, b, y, x).re : (R) 0;
                    for (int64_t w = 0; w < ebs; ++w) {
                        const R off = F_(w_offset)(w, ebs, vz);
                        const R g[3] = {f3[0] + off, f3[1], f3[2]};
                        if (g[0] * g[0] + g[1] * g[1] + g[2] * g[2] > cutoff_sqd)
                            continue;
                        cpx_t value;
                        R weight;
                        F_(sample_virtual)(&in, &in_w, in_shape2, in_centered, options->interp, n_in,
                                           &sc_in_eff, &rot_in, &ews, ifs, ifb, fin0, fin1, g, 0,
                                           &value, &weight);
                        const R cw = F_(windowed_sinc)(off, efs, efb);
                        acc = F_(c_add)(acc, F_(c_scale)(F_(to_output)(value, in_complex, out_complex), cw));
                        accw += weight * cw;
                    }
                    F_(dst_store)(&out, b, y, x, acc);
                    if (out_w.present)
                        F_(dst_store)(&out_w, b, y, x, F_(c_make)(accw, 0));
                }
            }
        }
    }
    return 0;
}

/* ------------------------------------------------------------------------------------------------
 * fourier_interpolation_correction (FourierProject.hpp:2062-2087) with GriddingCorrection
 * (:1009-1061): per voxel, dist = ((j, k, l) - half) / shape with half = shape / 2 (0 where a size is
 * 1), r = |dist|, sinc2 = sinc(pi r)^2 (noa::sinc: 1 at 0, base/Math.hpp:28-29); the output is
 * value / sinc2 (post-correction) or value * sinc2.
 * ------------------------------------------------------------------------------------------------ */
int F_(fpo_gridding_correction)(const fpo_array* input, const fpo_array* output, int32_t interp,
                                int32_t post_correction, int n_threads) {
    if (!input || !output || !output->data || (!input->data && !input->is_value))
        return -1;
    if (interp != 1 && interp != 101)
        return -2;
    const int64_t* sh = output->shape;
    const R fs[3] = {(R) sh[1], (R) sh[2], (R) sh[3]};
    R half[3];
    for (int i = 0; i < 3; ++i)
        half[i] = fs[i] / (R) 2 * (R) (sh[i + 1] != 1);
    const R PI = (R) 3.14159265358979323846;
    R* out = (R*) output->data;
    const R* in = (const R*) input->data;
    (void) n_threads;
    for (int64_t b = 0; b < sh[0]; ++b)
        for (int64_t j = 0; j < sh[1]; ++j)
            for (int64_t k = 0; k < sh[2]; ++k)
                for (int64_t l = 0; l < sh[3]; ++l) {
                    R d0 = (R) j, d1 = (R) k, d2 = (R) l;
                    d0 -= half[0]; d1 -= half[1]; d2 -= half[2];
                    d0 /= fs[0]; d1 /= fs[1]; d2 /= fs[2];
                    const R radius = R_SQRT(d0 * d0 + d1 * d1 + d2 * d2);
                    const R x = PI * radius;
                    const R sinc = x == 0 ? (R) 1 : R_SIN(x) / x;
                    const R sinc2 = sinc * sinc;
                    const R v = input->is_value ? (R) input->value[0]
                                                : in[b * input->strides[0] + j * input->strides[1] +
                                                     k * input->strides[2] + l * input->strides[3]];
                    out[b * output->strides[0] + j * output->strides[1] + k * output->strides[2] +
                        l * output->strides[3]] = post_correction ? v / sinc2 : v * sinc2;
                }
    return 0;
}

#undef cpx_t
#undef FPO_DECLARE_X
#undef F_
#undef CAT_
#undef CAT2_
