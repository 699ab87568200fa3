// FP32-bulk time evolution of one output interval (Magnus CF4, batched form).
//
// Precision split (errors are stated against the FP64 path, which matches the reference):
//   FP64  sample times, the rotating-frame phase (a phasor recurrence per interval), field samples
//         (tones by FP64 phasor recurrences), the frame transform, the CF4 generator combinations,
//         the linear part of every step's exponential (exp(A) - 1 = A + ..., A from the FP64
//         generators), and the product of steps within the output interval.
//   FP32  the rest of each exponential (its O(|A|^2) part), the product of the two CF4
//         exponentials of a step (its quadratic part) and the Magnus commutator (tensor-path
//         kernel).  So every FP32 rounding error of a step is O(2^-24 |g|^2) in the step generator
//         g: a step's first-order term, the one that adds up over 10^6 steps even when the field
//         varies slowly and its roundings repeat, is never rounded to FP32.  The kernels accumulate
//         sum |g|^2 per output step (the error statement, spinsim_b200.bulk_error_estimate).
//
// Exponentials.  Spin half: the exact SU(2) exponential exp(-i g.sigma/2) - 1 from even power
// series in r^2 = |g|^2 (no square root or division) for r <= 1/2, sincos otherwise.  Spin one with
// no quadratic shift in the step: the same SU(2) element mapped to its spin-one representation
// D1 (the homomorphism exp(-i g.J1) = D1(exp(-i g.sigma/2))); the step product and the interval
// product are then kept as SU(2) elements (2x2), mapped to 3x3 once per output interval.  Spin one
// with a quadratic shift: a Taylor series of exp(A) - 1 in A = -i(x Jx + y Jy + z Jz + q Q).  The
// reference's Lie-Trotter product approximates these exponentials to about
// |[A, B]| / (2 * 4^h) per exponential (h = number of squarings / 2).
#pragma once
#include "common.cuh"
#include "evolve64.cuh"

// 1: the next step's field samples are issued next to this step's exponentials (software pipeline).
#ifndef SPINSIM_BULK_PIPELINE
#define SPINSIM_BULK_PIPELINE 1
#endif

namespace spinsim {

struct c32 {
    float re, im;
};
SS_D c32 operator+(c32 a, c32 b) { return c32{a.re + b.re, a.im + b.im}; }
SS_D c32 operator-(c32 a, c32 b) { return c32{a.re - b.re, a.im - b.im}; }
SS_D c32 operator*(c32 a, c32 b) { return c32{fmaf(a.re, b.re, -a.im * b.im), fmaf(a.re, b.im, a.im * b.re)}; }
SS_D c32 operator*(float s, c32 a) { return c32{s * a.re, s * a.im}; }
SS_D c32 conjf(c32 a) { return c32{a.re, -a.im}; }
SS_D c32 cfmaf(c32 a, c32 b, c32 c) {
    return c32{fmaf(a.re, b.re, fmaf(-a.im, b.im, c.re)), fmaf(a.re, b.im, fmaf(a.im, b.re, c.im))};
}

template <int D>
struct Mat32 {
    c32 a[D][D];
};

// SU(2) element in residual form: alpha = 1 + am1, U = [[alpha, -conj(beta)], [beta, conj(alpha)]].
struct Su2f {
    c32 am1, beta;
};
struct Su2d {
    c64 am1, beta;
};

// The FP32 remainder of exp(-i g.sigma/2) - 1 beyond its linear part -i g.sigma/2 (which the caller
// takes in FP64): alpha - 1 = -i gz/2 + [c - i gz s'],  beta = (gy - i gx)/2 + [(gy - i gx) s'],
// c = cos(r/2) - 1, s' = sin(r/2)/r - 1/2, r = |g|: both O(r^2), from even series for r <= 1/2.
SS_D Su2f su2_exp_rest(float x, float y, float z) {
    const float r2 = fmaf(x, x, fmaf(y, y, z * z));
    float c, sp;
    if (r2 <= 0.25f) {
        c = r2 * (-0.125f + r2 * (1.0f / 384.0f + r2 * (-1.0f / 46080.0f + r2 * (1.0f / 10321920.0f -
                                                                            r2 * (1.0f / 3715891200.0f)))));
        sp = r2 * (-1.0f / 48.0f + r2 * (1.0f / 3840.0f + r2 * (-1.0f / 645120.0f + r2 * (1.0f / 185794560.0f))));
    } else {
        const float r = sqrtf(r2);
        float s4, c4;
        sincosf(0.25f * r, &s4, &c4);
        c = -2.0f * s4 * s4;
        sp = 2.0f * s4 * c4 / r - 0.5f;
    }
    Su2f e;
    e.am1 = c32{c, -z * sp};
    e.beta = c32{y * sp, -x * sp};
    return e;
}

// The whole element in FP32 (linear part rounded) from its remainder: for quadratic terms only.
SS_D Su2f su2_full(float x, float y, float z, const Su2f& rest) {
    return Su2f{c32{rest.am1.re, fmaf(-0.5f, z, rest.am1.im)}, c32{fmaf(0.5f, y, rest.beta.re), fmaf(-0.5f, x, rest.beta.im)}};
}

// The quadratic part b a of (1 + b)(1 + a) - 1 = a + b + b a (b later).
SS_D Su2f su2_prod(const Su2f& b, const Su2f& a) {
    Su2f o;
    o.am1 = b.am1 * a.am1 - conjf(b.beta) * a.beta;
    o.beta = b.beta * a.am1 + conjf(b.am1) * a.beta;
    return o;
}

SS_D Su2f su2_add(const Su2f& a, const Su2f& b) { return Su2f{a.am1 + b.am1, a.beta + b.beta}; }

// exp(A) - 1 for A = -i H, H = x Jx + y Jy + z Jz + q Q (spin one, Q = diag(1, -2, 1) / 3), by a
// Taylor series to A^6 / 6! on A scaled to norm <= 1/32 (truncation below 2e-13 relative),
// followed by residual squarings (E - 1 -> 2 (E - 1) + (E - 1)^2) when it was scaled.
SS_D Mat32<3> spin_one_exp_m1(float x, float y, float z, float q) {
    constexpr float ir2 = 0.70710678118654752f;
    const float pr = x * ir2, pi = y * ir2;
    const float h0 = z + q * (1.0f / 3.0f), h1 = -q * (2.0f / 3.0f), h2 = -z + q * (1.0f / 3.0f);
    int squarings = 0;
    float scale = 1.0f;
    const float norm = fabsf(x) + fabsf(y) + fabsf(z) + fabsf(q);
    while (norm * scale > 0.03125f && squarings < 40) {
        scale *= 0.5f;
        squarings++;
    }
    // A = -i H (scaled); H[1][0] = H[2][1] = (x + i y) / sqrt2, H[0][1] = H[1][2] = (x - i y) / sqrt2
    Mat32<3> A;
    A.a[0][0] = c32{0.0f, -h0 * scale};
    A.a[1][1] = c32{0.0f, -h1 * scale};
    A.a[2][2] = c32{0.0f, -h2 * scale};
    A.a[1][0] = c32{pi * scale, -pr * scale};
    A.a[2][1] = A.a[1][0];
    A.a[0][1] = c32{-pi * scale, -pr * scale};
    A.a[1][2] = A.a[0][1];
    A.a[2][0] = c32{0.0f, 0.0f};
    A.a[0][2] = c32{0.0f, 0.0f};
    // R_6 = A / 6;  R_k = (A + A R_{k+1}) / k for k = 5 .. 1;  E - 1 = R_1
    const float inv[6] = {1.0f, 0.5f, 1.0f / 3.0f, 0.25f, 0.2f, 1.0f / 6.0f};
    Mat32<3> R;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) R.a[i][j] = inv[5] * A.a[i][j];
#pragma unroll
    for (int k = 5; k >= 1; k--) {
        Mat32<3> N;
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) {
                c32 acc = A.a[i][j];
#pragma unroll
                for (int l = 0; l < 3; l++) acc = cfmaf(A.a[i][l], R.a[l][j], acc);
                N.a[i][j] = inv[k - 1] * acc;
            }
        R = N;
    }
    for (int s = 0; s < squarings; s++) {
        Mat32<3> N;
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) {
                c32 acc = c32{2.0f * R.a[i][j].re, 2.0f * R.a[i][j].im};
#pragma unroll
                for (int l = 0; l < 3; l++) acc = cfmaf(R.a[i][l], R.a[l][j], acc);
                N.a[i][j] = acc;
            }
        R = N;
    }
    return R;
}

// A = -i H for H = x Jx + y Jy + z Jz + q Q (spin one, Q = diag(1, -2, 1) / 3), the linear part of
// exp(A) - 1, in FP64 or FP32.
template <typename T, typename C>
SS_D void spin_one_generator_into(T x, T y, T z, T q, C (&a)[3][3]) {
    const T ir2 = (T)0.70710678118654752440;
    const T pr = x * ir2, pi = y * ir2;
    const T h0 = z + q / (T)3, h1 = -q * ((T)2 / (T)3), h2 = -z + q / (T)3;
    a[0][0] = C{(T)0, -h0};
    a[1][1] = C{(T)0, -h1};
    a[2][2] = C{(T)0, -h2};
    a[1][0] = C{pi, -pr};
    a[2][1] = C{pi, -pr};
    a[0][1] = C{-pi, -pr};
    a[1][2] = C{-pi, -pr};
    a[2][0] = C{(T)0, (T)0};
    a[0][2] = C{(T)0, (T)0};
}

// u <- u + (a64 + rest) u: the step's linear part in FP64, its remainder converted from FP32.
SS_D void apply_split3(Mat<3>& u, const c64 (&a64)[3][3], const Mat32<3>& rest) {
    c64 d[3][3];
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int k = 0; k < 3; k++) d[i][k] = c64{a64[i][k].re + (double)rest.a[i][k].re, a64[i][k].im + (double)rest.a[i][k].im};
    Mat<3> o;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            c64 acc = u.a[i][j];
#pragma unroll
            for (int k = 0; k < 3; k++) acc = cfma(d[i][k], u.a[k][j], acc);
            o.a[i][j] = acc;
        }
    u = o;
}

// One CF4 step of spin one with a quadratic shift: E = Ea + Eb + Eb Ea with Ea = exp(A(ga)) - 1, its
// linear part A(ga + gb) in FP64, the rest (series remainders and the product) in FP32.
SS_D void spin_one_cf4_step(Mat<3>& u, const double* ga, const double* gb, float* nsq) {
    float a[4], b[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        a[k] = __double2float_rn(ga[k]);
        b[k] = __double2float_rn(gb[k]);
        *nsq = fmaf(a[k], a[k], fmaf(b[k], b[k], *nsq));
    }
    const Mat32<3> ra = spin_one_exp_m1(a[0], a[1], a[2], a[3]);
    const Mat32<3> rb = spin_one_exp_m1(b[0], b[1], b[2], b[3]);
    c32 la[3][3], lb[3][3];
    spin_one_generator_into<float, c32>(a[0], a[1], a[2], a[3], la);
    spin_one_generator_into<float, c32>(b[0], b[1], b[2], b[3], lb);
    Mat32<3> rest;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            c32 acc = (ra.a[i][j] - la[i][j]) + (rb.a[i][j] - lb[i][j]);
#pragma unroll
            for (int k = 0; k < 3; k++) acc = cfmaf(rb.a[i][k], ra.a[k][j], acc);
            rest.a[i][j] = acc;
        }
    c64 lin[3][3];
    spin_one_generator_into<double, c64>(ga[0] + gb[0], ga[1] + gb[1], ga[2] + gb[2], ga[3] + gb[3], lin);
    apply_split3(u, lin, rest);
}

// The spin-one Euler step: the 3x3 exponential's linear part in FP64, its remainder in FP32.
SS_D void spin_one_euler_step(Mat<3>& u, const double* g, float* nsq) {
    float a[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        a[k] = __double2float_rn(g[k]);
        *nsq = fmaf(a[k], a[k], *nsq);
    }
    const Mat32<3> ra = spin_one_exp_m1(a[0], a[1], a[2], a[3]);
    c32 la[3][3];
    spin_one_generator_into<float, c32>(a[0], a[1], a[2], a[3], la);
    Mat32<3> rest;
#pragma unroll
    for (int i2 = 0; i2 < 3; i2++)
#pragma unroll
        for (int j2 = 0; j2 < 3; j2++) rest.a[i2][j2] = ra.a[i2][j2] - la[i2][j2];
    c64 lin[3][3];
    spin_one_generator_into<double, c64>(g[0], g[1], g[2], g[3], lin);
    apply_split3(u, lin, rest);
}

// P <- (1 + E) P in FP64 with E = -i g.sigma/2 (g the step's FP64 generator: the linear part, never
// rounded to FP32) + rest (its FP32 remainder).
SS_D void su2_apply_split(Su2d& p, double gx, double gy, double gz, const Su2f& rest) {
    const c64 am1 = c64{(double)rest.am1.re, fma(-0.5, gz, (double)rest.am1.im)};
    const c64 b = c64{fma(0.5, gy, (double)rest.beta.re), fma(-0.5, gx, (double)rest.beta.im)};
    // alpha' = alpha_e alpha - conj(beta_e) beta ; beta' = beta_e alpha + conj(alpha_e) beta
    const c64 alpha = c64{1.0 + p.am1.re, p.am1.im};
    const c64 beta = p.beta;
    // (alpha - 1) + am1 alpha - conj(b) beta and b alpha + conj(am1) beta + beta, each part one chain
    // of four FMAs
    c64 na, nb;
    na.re = fma(-am1.im, alpha.im, fma(am1.re, alpha.re, fma(-b.im, beta.im, fma(-b.re, beta.re, p.am1.re))));
    na.im = fma(am1.im, alpha.re, fma(am1.re, alpha.im, fma(b.im, beta.re, fma(-b.re, beta.im, p.am1.im))));
    nb.re = fma(-b.im, alpha.im, fma(b.re, alpha.re, fma(am1.im, beta.im, fma(am1.re, beta.re, beta.re))));
    nb.im = fma(b.im, alpha.re, fma(b.re, alpha.im, fma(-am1.im, beta.re, fma(am1.re, beta.im, beta.im))));
    p.am1 = na;
    p.beta = nb;
}

// One CF4 step as an SU(2) element: E = Ea + Eb + Eb Ea with Ea = exp(-i ga.sigma/2) - 1; its linear
// part -i (ga + gb).sigma/2 in FP64, the series remainders and the product Eb Ea in FP32.
SS_D void su2_cf4_step(Su2d& p, const double* ga, const double* gb, float* nsq) {
    float a[3], b[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        a[c] = __double2float_rn(ga[c]);
        b[c] = __double2float_rn(gb[c]);
        *nsq = fmaf(a[c], a[c], fmaf(b[c], b[c], *nsq));
    }
    const Su2f ra = su2_exp_rest(a[0], a[1], a[2]);
    const Su2f rb = su2_exp_rest(b[0], b[1], b[2]);
    const Su2f prod = su2_prod(su2_full(b[0], b[1], b[2], rb), su2_full(a[0], a[1], a[2], ra));
    su2_apply_split(p, ga[0] + gb[0], ga[1] + gb[1], ga[2] + gb[2], su2_add(su2_add(ra, rb), prod));
}

// One Euler step (a single exponential of the generator g, I:759-791) in the same split: the linear
// part in FP64, the remainder in FP32.
SS_D void su2_euler_step(Su2d& p, const double* g, float* nsq) {
    float a[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        a[c] = __double2float_rn(g[c]);
        *nsq = fmaf(a[c], a[c], *nsq);
    }
    su2_apply_split(p, g[0], g[1], g[2], su2_exp_rest(a[0], a[1], a[2]));
}

// ---------------------------------------------------------------------------------- generic bulk path
// One output interval per lane (USER and TABLE fields, tone fields the synthesis below does not take:
// spin one with a quadratic shift, and the Euler and Heun integrators).  The integrators differ only
// in where a step samples the field and how it weights the samples: Magnus CF4 at the two Gauss
// points with two exponentials (I:624-686), Heun at the step's ends with two half-step exponentials
// (I:693-752), Euler at the midpoint with one exponential (I:759-791).
// The state of interval32's step loop that the field samples need: the frame phasor W(t) =
// exp(-i P rw (t - t_c)) advanced by an FP64 recurrence, its step and sample-offset factors, the
// step start, the sample offsets and weights, and the table cursors.
template <int L>
struct Steps32 {
    c64 W, Wrot, Woff;
    double rw, t_fine, dt, off_a, off_b, c0, c1;
    bool rotating;
    TableCursor cur[L];
};

// One step's field samples (FP64) -> frame transform -> the integrator's generators (FP64); the
// frame phasor moves on by one step.
template <int FIELD, int L, int P, int INTEG>
SS_D void step_generators32(const FieldDesc& f, Steps32<L>& st, double* ga, double* gb) {
    double s0[8], s1[8];  // a user field writes all eight channels
#pragma unroll
    for (int k = 0; k < 8; k++) {
        s0[k] = 0.0;
        s1[k] = 0.0;
    }
    sample_field<FIELD, L>(f, st.t_fine + st.off_a, s0, st.cur);
    if (INTEG != INTEG_EULER) sample_field<FIELD, L>(f, st.t_fine + st.off_b, s1, st.cur);
    if (st.rotating) {  // xy times exp(-i P rw tau), z minus P rw
        const c64 Wn = st.W * st.Wrot;
        const c64 xa = c64{s0[0], s0[1]} * (st.W * st.Woff);
        s0[0] = xa.re;
        s0[1] = xa.im;
        s0[2] -= (double)P * st.rw;
        if (INTEG != INTEG_EULER) {
            const c64 xb = c64{s1[0], s1[1]} * (Wn * conj(st.Woff));
            s1[0] = xb.re;
            s1[1] = xb.im;
            s1[2] -= (double)P * st.rw;
        }
        st.W = Wn;
    }
#pragma unroll
    for (int k = 0; k < L; k++) {  // Euler: the one generator in ga (gb zero)
        ga[k] = fma(st.c0, s0[k], st.c1 * s1[k]);
        gb[k] = INTEG == INTEG_HEUN ? st.c0 * s1[k] : fma(st.c1, s0[k], st.c0 * s1[k]);
    }
}

struct Generators4 {
    double a[4], b[4];
};

struct SpinOneProduct {
    Mat<3> u;
    float nsq;
};

// Steps j .. j1-1 of a spin-one interval whose quadratic shift is non-zero: full 3x3 exponentials
// and an FP64 3x3 product, from the product u of the steps before.  On entry st.t_fine is step j's
// start and its generators are in g.  Out of line (and with its state passed by value), so that the
// registers of the common SU(2) loop are allocated without this path's.
template <int INTEG, int FIELD>
__device__ __noinline__ SpinOneProduct spin_one_quadratic_steps32(const FieldDesc& f, Steps32<4> st, Mat<3> u,
                                                                  Generators4 g, int j, int j1, float nsq) {
    bool first = true;
    for (; j < j1; j++) {
        if (!first) step_generators32<FIELD, 4, 1, INTEG>(f, st, g.a, g.b);
        first = false;
        if constexpr (INTEG == INTEG_EULER) spin_one_euler_step(u, g.a, &nsq);
        else spin_one_cf4_step(u, g.a, g.b, &nsq);
        st.t_fine += st.dt;
    }
    return SpinOneProduct{u, nsq};
}

template <int D, int INTEG, int EXPO, int FIELD>
SS_D void interval32(const MethodConfig& m, const Instance& inst, const FieldDesc& f, int64_t index, bool active,
                     int lane_in_group, double* time_out, double* u_out, float* norms_out) {
    static_assert(EXPO != EXPO_LIE_TROTTER_8, "the FP32-bulk form has no eight-generator exponential");
    constexpr int L = (D == 2) ? 3 : 4;
    constexpr int P = (D == 2) ? 2 : 1;  // power of the frame winding in the xy transform (I:599-613)
    const int lanes = m.lanes;
    const double dt = inst.dt_int, dt_out = inst.dt_out;
    const double t_c = __dadd_rn(inst.t0, __dmul_rn(dt_out, (double)(inst.interval0 + index)));  // I:818, unfused
    double rw = 0.0;
    if (active && m.rotating) {
        double s0[8];
#pragma unroll
        for (int k = 0; k < 8; k++) s0[k] = 0.0;
        sample_field<FIELD, L>(f, t_c + dt_out / 2, s0);
        rw = s0[2];
        if (D == 2) rw /= 2;
    }
    const int K = active ? inst.n_fine : 0;
    const int j0 = (int)(((int64_t)K * lane_in_group) / lanes);
    const int j1 = (int)(((int64_t)K * (lane_in_group + 1)) / lanes);
    double t_fine = t_c;
    for (int j = 0; j < j0; j++) t_fine += dt;

    const double a_lo = 0.5 * dt * (1.0 - 1.0 / kSqrt3);
    const double a_hi = 0.5 * dt * (1.0 + 1.0 / kSqrt3);
    const double w0 = (1.5 + kSqrt3) / 6.0, w1 = (1.5 - kSqrt3) / 6.0;
    // sample offsets in the step (off_b = dt - off_a) and the weights of the samples in the two
    // exponentials' generators
    const double off_a = INTEG == INTEG_CF4 ? a_lo : INTEG == INTEG_HEUN ? 0.0 : 0.5 * dt;
    const double off_b = INTEG == INTEG_CF4 ? a_hi : dt;
    const double c0 = INTEG == INTEG_CF4 ? dt * w0 : INTEG == INTEG_HEUN ? 0.5 * dt : dt;
    const double c1 = INTEG == INTEG_CF4 ? dt * w1 : 0.0;

    // Frame phasor W(t) = exp(-i P rw (t - t_c)) by an FP64 recurrence, anchored at this lane's start.
    Steps32<L> st;
    st.W = st.Wrot = st.Woff = c64{1.0, 0.0};
    if (m.rotating && K > 0) {
        sincos(-(double)P * rw * (t_fine - t_c), &st.W.im, &st.W.re);
        sincos(-(double)P * rw * dt, &st.Wrot.im, &st.Wrot.re);
        sincos(-(double)P * rw * off_a, &st.Woff.im, &st.Woff.re);
    }
    st.rw = rw;
    st.t_fine = t_fine;
    st.dt = dt;
    st.off_a = off_a;
    st.off_b = off_b;
    st.c0 = c0;
    st.c1 = c1;
    st.rotating = m.rotating;
#pragma unroll
    for (int c = 0; c < L; c++) st.cur[c] = TableCursor{};  // for the increasing sample times of the steps
    auto step_generators = [&](double* ga, double* gb) { step_generators32<FIELD, L, P, INTEG>(f, st, ga, gb); };

    // Phase 1: every step an SU(2) element (spin half always; spin one while the quadratic shift
    // is zero); the interval product is an FP64 SU(2) element.  Software-pipelined: the next step's
    // field samples (independent FP64 work) are issued next to this step's exponentials and product.
    Su2d su2 = Su2d{c64{0.0, 0.0}, c64{0.0, 0.0}};
    double ga[4] = {0.0, 0.0, 0.0, 0.0}, gb[4] = {0.0, 0.0, 0.0, 0.0};
    float nsq = 0.0f;  // sum of |g|^2 over this lane's steps (the error statement's scale)
    int j = j0;
    bool pending = false;
    if (j < j1) step_generators(ga, gb);
    for (; j < j1; j++) {
        if constexpr (D == 3) {
            if (ga[3] != 0.0 || gb[3] != 0.0) {
                pending = true;
                break;
            }
        }
        double na[4] = {0.0, 0.0, 0.0, 0.0}, nb[4] = {0.0, 0.0, 0.0, 0.0};
        st.t_fine += dt;
        if (j + 1 < j1) step_generators(na, nb);
        if constexpr (INTEG == INTEG_EULER) su2_euler_step(su2, ga, &nsq);
        else su2_cf4_step(su2, ga, gb, &nsq);
#pragma unroll
        for (int k = 0; k < 4; k++) {
            ga[k] = na[k];
            gb[k] = nb[k];
        }
    }
    Mat<D> u;
    {
        const c64 alpha = c64{1.0 + su2.am1.re, su2.am1.im};
        if constexpr (D == 3) {
            u = su2_to_spin_one(alpha, su2.beta);
        } else {
            u.a[0][0] = alpha;
            u.a[1][0] = su2.beta;
            u.a[0][1] = c64{-su2.beta.re, su2.beta.im};
            u.a[1][1] = conj(alpha);
        }
    }
    // Phase 2 (spin one with a quadratic shift): full 3x3 exponentials and an FP64 3x3 product.
    // On entry st.t_fine is the pending step's start and its generators are in ga, gb.
    if constexpr (D == 3) {
        if (pending) {
            Generators4 g;
#pragma unroll
            for (int k = 0; k < 4; k++) {
                g.a[k] = ga[k];
                g.b[k] = gb[k];
            }
            const SpinOneProduct r = spin_one_quadratic_steps32<INTEG, FIELD>(f, st, u, g, j, j1, nsq);
            u = r.u;
            nsq = r.nsq;
        }
    }

    for (int s = 1; s < lanes; s <<= 1) {
        const Mat<D> later = shfl_down_mat(u, s);
        nsq += __shfl_down_sync(0xffffffffu, nsq, s);
        if ((lane_in_group & (2 * s - 1)) == 0) u = matmul(later, u);
    }
    if (!active || lane_in_group != 0) return;
    if (m.rotating) {  // leave the rotating frame, I:839-852
        c64 wo;
        sincos(rw * dt_out, &wo.im, &wo.re);
        const c64 woc = conj(wo);
#pragma unroll
        for (int k = 0; k < D; k++) {
            u.a[0][k] = u.a[0][k] * woc;
            u.a[D - 1][k] = u.a[D - 1][k] * wo;
        }
    }
    time_out[index] = t_c;
    if (norms_out != nullptr) norms_out[index] = nsq;
    double2* dst = reinterpret_cast<double2*>(u_out) + index * (D * D);
#pragma unroll
    for (int i = 0; i < D; i++)
#pragma unroll
        for (int k = 0; k < D; k++) dst[i * D + k] = make_double2(u.a[i][k].re, u.a[i][k].im);
}

// ---------------------------------------------------------------------------------- tone synthesis
// Warp-cooperative evaluation of tone fields (FIELD_TONES, no quadratic shift).  A warp takes a
// tile of 32 * kSynthIntervals consecutive output intervals of one instance; lane l works on
// intervals l, l + 32, ...; every lane steps through the instance's K fine steps in lockstep, so
// the sample times differ between intervals only by the interval start t_c.  Writing
//     A sin(w (t_c + tau) + phi) = Im( L(t_c) U(tau) ),  L = A exp(i (w t_c + phi)),  U = exp(i w tau),
// each lane keeps L of its first interval in shared memory (read-only for the tile); its interval
// 32 i later has L G^i with G = exp(i w 32 dt_out), the same for the whole warp.  U(tau) for the
// current step is also the same for the whole warp: lane k advances tone k's U by an FP64 recurrence
// (U <- U exp(i w dt)) and publishes G^i U and G^i V, V = U exp(i w (a_hi - a_lo)) for the second
// Gauss point, through a double-buffered shared slot.  A sample then costs two FMAs per tone and
// interval; the intervals' dependent chains interleave.
extern __shared__ __align__(16) unsigned char spinsim_dyn_smem[];
static_assert(sizeof(ToneShared) == kToneSharedBytes, "tone shared layout");

SS_D bool tones_have_quadratic_shift(const FieldDesc& f) { return f.bias[3] != 0.0 || f.tone_count[3] > 0; }

template <int D, int EXPO>
SS_D void intervals32_synth(const MethodConfig& m, const Instance& inst, const FieldDesc& f, const Tile& tile,
                            double* time_out, double* u_out, float* norms_out) {
    constexpr int NI = kSynthIntervals;
    constexpr int P = (D == 2) ? 2 : 1;  // power of the frame winding in the xy transform (I:599-613)
    const int lane = threadIdx.x & 31;
    ToneShared* ts = reinterpret_cast<ToneShared*>(spinsim_dyn_smem) + (threadIdx.x >> 5);
    const double dt = inst.dt_int, dt_out = inst.dt_out;
    const int K = inst.n_fine;
    const double a_lo = 0.5 * dt * (1.0 - 1.0 / kSqrt3);
    const double a_hi = 0.5 * dt * (1.0 + 1.0 / kSqrt3);
    const double w0 = (1.5 + kSqrt3) / 6.0, w1 = (1.5 - kSqrt3) / 6.0;
    const double c0 = dt * w0, c1 = dt * w1;

    bool active[NI];
    int64_t index[NI];
    double t_c[NI], rw[NI];
    c64 W[NI], Wrot[NI], Woff[NI];
#pragma unroll
    for (int i = 0; i < NI; i++) {
        active[i] = lane + 32 * i < tile.count;
        index[i] = tile.first + (active[i] ? lane + 32 * i : 0);
        t_c[i] = __dadd_rn(inst.t0, __dmul_rn(dt_out, (double)(inst.interval0 + index[i])));  // I:818, unfused
        rw[i] = 0.0;
        W[i] = Wrot[i] = Woff[i] = c64{1.0, 0.0};
        if (active[i] && m.rotating) {
            double smp[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
            sample_field<FIELD_TONES, 3>(f, t_c[i] + dt_out / 2, smp);
            rw[i] = (D == 2) ? smp[2] / 2 : smp[2];
            sincos(-(double)P * rw[i] * dt, &Wrot[i].im, &Wrot[i].re);
            sincos(-(double)P * rw[i] * a_lo, &Woff[i].im, &Woff[i].re);
        }
    }
    bool direct = false;  // tones past the synthesis slots (sampled directly)
    double bias[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        direct |= f.tone_count[c] > kBulkTones;
        bias[c] = f.bias[c];
    }
    // L of every slot for the lane's first interval; the producer constants of slot `lane`
#pragma unroll 1
    for (int slot = 0; slot < kToneSlots; slot++) {
        const int c = slot / kBulkTones, k = slot % kBulkTones;
        double re = 0.0, im = 0.0;
        if (k < f.tone_count[c]) {
            const double* tone = f.tones + 3 * (f.tone_start[c] + k);
            const double amp = f.gain[c] * __ldg(tone + 1);
            double sn, cs;
            sincos(fma(__ldg(tone), t_c[0], __ldg(tone + 2)), &sn, &cs);
            re = amp * cs;
            im = amp * sn;
        }
        ts->l[slot][lane][0] = re;
        ts->l[slot][lane][1] = im;
    }
    // producer constants of slot `lane` (registers for the whole tile): exp(i w dt), exp(i w (a_hi - a_lo)), G
    c64 u_prod = c64{0.0, 0.0}, rot = c64{1.0, 0.0}, gap = c64{1.0, 0.0}, g = c64{1.0, 0.0};
    if (lane < kToneSlots) {
        const int c = lane / kBulkTones, k = lane % kBulkTones;
        if (k < f.tone_count[c]) {
            const double w = __ldg(f.tones + 3 * (f.tone_start[c] + k));
            sincos(w * a_lo, &u_prod.im, &u_prod.re);
            sincos(w * dt, &rot.im, &rot.re);
            sincos(w * (a_hi - a_lo), &gap.im, &gap.re);
            // G = exp(i w (t_c(l + 32) - t_c(l))), t_c rounded as the intervals' own starts are
            const int64_t i0 = inst.interval0 + index[0];
            sincos(w * (__dmul_rn(dt_out, (double)(i0 + 32)) - __dmul_rn(dt_out, (double)i0)), &g.im, &g.re);
        }
    }

    Su2d su2[NI];
    float nsq[NI];
#pragma unroll
    for (int i = 0; i < NI; i++) {
        su2[i] = Su2d{c64{0.0, 0.0}, c64{0.0, 0.0}};
        nsq[i] = 0.0f;
    }
    for (int j = 0; j < K; j++) {
        // publish G^i U, G^i V of step j
        if (lane < kToneSlots) {
            c64 uu = u_prod, vv = u_prod * gap;
#pragma unroll
            for (int i = 0; i < NI; i++) {
                ts->uv[j & 1][i][0][lane] = make_double2(uu.re, uu.im);
                ts->uv[j & 1][i][1][lane] = make_double2(vv.re, vv.im);
                if (i + 1 < NI) {
                    uu = uu * g;
                    vv = vv * g;
                }
            }
            u_prod = u_prod * rot;
        }
        __syncwarp();
        // field samples at the two Gauss points of every interval (FP64)
        double sa[NI][3], sb[NI][3];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            double pa[NI], pb[NI];
#pragma unroll
            for (int i = 0; i < NI; i++) {
                sa[i][c] = bias[c];
                sb[i][c] = bias[c];
                pa[i] = 0.0;
                pb[i] = 0.0;
            }
#pragma unroll
            for (int k = 0; k < kBulkTones; k++) {
                const int slot = c * kBulkTones + k;
                const double2 lv = *reinterpret_cast<const double2*>(ts->l[slot][lane]);
#pragma unroll
                for (int i = 0; i < NI; i++) {
                    const double2 uu = ts->uv[j & 1][i][0][slot];
                    const double2 vv = ts->uv[j & 1][i][1][slot];
                    if (k & 1) {
                        pa[i] = fma(lv.x, uu.y, fma(lv.y, uu.x, pa[i]));
                        pb[i] = fma(lv.x, vv.y, fma(lv.y, vv.x, pb[i]));
                    } else {
                        sa[i][c] = fma(lv.x, uu.y, fma(lv.y, uu.x, sa[i][c]));
                        sb[i][c] = fma(lv.x, vv.y, fma(lv.y, vv.x, sb[i][c]));
                    }
                }
            }
#pragma unroll
            for (int i = 0; i < NI; i++) {
                sa[i][c] += pa[i];
                sb[i][c] += pb[i];
            }
            if (direct) {
#pragma unroll
                for (int i = 0; i < NI; i++) {
                    const double t_step = t_c[i] + (double)j * dt;
                    for (int k = kBulkTones; k < f.tone_count[c]; k++) {
                        const double* tone = f.tones + 3 * (f.tone_start[c] + k);
                        const double w = __ldg(tone), a = f.gain[c] * __ldg(tone + 1), ph = __ldg(tone + 2);
                        sa[i][c] = fma(a, sin(fma(w, t_step + a_lo, ph)), sa[i][c]);
                        sb[i][c] = fma(a, sin(fma(w, t_step + a_hi, ph)), sb[i][c]);
                    }
                }
            }
        }
        // frame transform, CF4 generators (rounded once to FP32), SU(2) exponentials and product
#pragma unroll
        for (int i = 0; i < NI; i++) {
            if (m.rotating) {
                const c64 Wn = W[i] * Wrot[i];
                const c64 xa = c64{sa[i][0], sa[i][1]} * (W[i] * Woff[i]);
                const c64 xb = c64{sb[i][0], sb[i][1]} * (Wn * conj(Woff[i]));
                sa[i][0] = xa.re;
                sa[i][1] = xa.im;
                sb[i][0] = xb.re;
                sb[i][1] = xb.im;
                sa[i][2] -= (double)P * rw[i];
                sb[i][2] -= (double)P * rw[i];
                W[i] = Wn;
            }
            double ga[3], gb[3];
#pragma unroll
            for (int c = 0; c < 3; c++) {
                ga[c] = fma(c0, sa[i][c], c1 * sb[i][c]);
                gb[c] = fma(c1, sa[i][c], c0 * sb[i][c]);
            }
            su2_cf4_step(su2[i], ga, gb, &nsq[i]);
        }
    }
    __syncwarp();  // the shared slots are reused by the warp's next tile

#pragma unroll
    for (int i = 0; i < NI; i++) {
        if (!active[i]) continue;
        const c64 alpha = c64{1.0 + su2[i].am1.re, su2[i].am1.im};
        Mat<D> u;
        if constexpr (D == 3) {
            u = su2_to_spin_one(alpha, su2[i].beta);
        } else {
            u.a[0][0] = alpha;
            u.a[1][0] = su2[i].beta;
            u.a[0][1] = c64{-su2[i].beta.re, su2[i].beta.im};
            u.a[1][1] = conj(alpha);
        }
        if (m.rotating) {  // leave the rotating frame, I:839-852
            c64 wo;
            sincos(rw[i] * dt_out, &wo.im, &wo.re);
            const c64 woc = conj(wo);
#pragma unroll
            for (int k = 0; k < D; k++) {
                u.a[0][k] = u.a[0][k] * woc;
                u.a[D - 1][k] = u.a[D - 1][k] * wo;
            }
        }
        time_out[index[i]] = t_c[i];
        if (norms_out != nullptr) norms_out[index[i]] = nsq[i];
        double2* dst = reinterpret_cast<double2*>(u_out) + index[i] * (D * D);
#pragma unroll
        for (int r = 0; r < D; r++)
#pragma unroll
            for (int k = 0; k < D; k++) dst[r * D + k] = make_double2(u.a[r][k].re, u.a[r][k].im);
    }
}

}  // namespace spinsim
