// FP64 matrix exponentials of the reference (Utilities, spinsim/__init__.py:1528-1939), held in
// registers.  The same mathematical formulas as the reference, written so that each needs fewer
// transcendental calls: sin(x) = 2 sin(x/2) cos(x/2) from one sincos, a complex phase exp(i p)
// from (x + i y) / |x + i y| instead of atan2, and phase products by angle addition.  These
// rewrites change results only at the level of double rounding.
#pragma once
#include "common.cuh"

namespace spinsim {

constexpr double kSqrt2 = 1.4142135623730951;
constexpr double kSqrt3 = 1.7320508075688772;

// expm1i(x) = exp(i x) - 1 = -2 sin^2(x/2) + i sin(x)   (I:1557-1559)
SS_D c64 expm1i(double x) {
    double s, c;
    sincos(0.5 * x, &s, &c);
    return c64{-2.0 * (s * s), 2.0 * s * c};
}

// cos_exp_m1(c, e) = (expm1i(c + e) + expm1i(-c + e)) / 2 = cos(c) exp(i e) - 1   (I:1561-1563)
SS_D c64 cos_exp_m1(double c, double e) {
    const c64 a = expm1i(c + e), b = expm1i(-c + e);
    return c64{0.5 * (a.re + b.re), 0.5 * (a.im + b.im)};
}

// cos_m1(t) = cos(t) - 1 = -2 sin^2(t/2)   (I:1565-1567)
SS_D double cos_m1(double t) {
    const double s = sin(0.5 * t);
    return -2.0 * (s * s);
}

// ------------------------------------------------------------------ spin half
// matrix_exponential_analytic (I:1618-1642): exp of -i(x Jx + y Jy + z Jz) for spin half.
SS_D Mat<2> expo_analytic_half(const double* g) {
    Mat<2> r;
    double x = g[0], y = g[1], z = g[2];
    const double rr = sqrt(x * x + y * y + z * z);
    if (rr > 0) {
        const double inv = 1.0 / rr;
        x *= inv;
        y *= inv;
        z *= inv;
        double s4, c4;
        sincos(0.25 * rr, &s4, &c4);
        const double c = -2.0 * (s4 * s4);  // cos_exp_m1(r/2, 0) (its imaginary part is zero)
        const double s = 2.0 * s4 * c4;     // sin(r/2)
        r.a[0][0] = c64{c + 1.0, -z * s};
        r.a[1][0] = c64{y * s, -x * s};
        r.a[0][1] = c64{-y * s, -x * s};
        r.a[1][1] = c64{c + 1.0, z * s};
    } else {
        set_identity(r);
    }
    return r;
}

// matrix_exponential_lie_trotter for spin half (I:1644-1673)
SS_D Mat<2> expo_lt_half(const double* g, int hypercubes, double precision) {
    double a = sqrt(g[0] * g[0] + g[1] * g[1]);
    c64 ep = c64{1.0, 0.0};
    if (a > 0) {
        const double inv = 1.0 / a;
        ep = c64{g[0] * inv, g[1] * inv};
    }
    a = a / precision;
    const double z = g[2] / (2.0 * precision);
    // Sa = -i sin(a/2); R00 = cos_exp_m1(a/2, -z); R11 = cos_exp_m1(a/2, z) = conj(R00) up to rounding
    const double sa = sin(0.5 * a);
    const c64 Sa = c64{0.0, -sa};
    Mat<2> r;
    r.a[0][0] = cos_exp_m1(0.5 * a, -z);
    r.a[1][0] = Sa * ep;
    r.a[0][1] = Sa * conj(ep);  // Sa / ep with |ep| = 1
    r.a[1][1] = cos_exp_m1(0.5 * a, z);
    for (int h = 0; h < hypercubes; h++) {
        r = square_m1(r);
        r = square_m1(r);
    }
    r.a[0][0].re += 1.0;
    r.a[1][1].re += 1.0;
    return r;
}

// ------------------------------------------------------------------ spin one
// matrix_exponential_lie_trotter for spin one (I:1768-1808); exp(i p) = (x + i y) / a replaces
// p = atan2(y, x).
SS_D Mat<3> expo_lt_one(const double* g, int hypercubes, double precision) {
    double a = sqrt(g[0] * g[0] + g[1] * g[1]);
    c64 ep = c64{1.0, 0.0};  // exp(i p)
    if (a > 0) {
        const double inv = 1.0 / a;
        ep = c64{g[0] * inv, g[1] * inv};
    }
    a = a / precision;
    double sh, ch;
    sincos(0.5 * a, &sh, &ch);
    const double Sa = sh;                                   // sin(a/2)
    const c64 sa = c64{0.0, -(2.0 * sh * ch) / kSqrt2};    // -i sin(a) / sqrt2
    const double z = g[2] / (2.0 * precision);
    const double q = g[3] / (6.0 * precision);
    double sz, cz, sq, cq;
    sincos(z, &sz, &cz);
    sincos(q, &sq, &cq);
    const c64 ez = c64{cz, sz}, eq = c64{cq, sq};
    const c64 epc = conj(ep), ezc = conj(ez), eqc = conj(eq);
    const double Sa2 = Sa * Sa;
    Mat<3> r;
    c64 cem = cos_exp_m1(0.5 * a, -z - q);
    r.a[0][0] = cem * (cem + c64{2.0, 0.0});
    r.a[1][0] = sa * ((eq * ep) * ezc);           // exp(i(q + p - z))
    r.a[2][0] = (-Sa2) * ((ep * ep) * (eqc * eqc));   // exp(2i(p - q))
    r.a[0][1] = sa * ((eq * epc) * ezc);          // exp(i(q - p - z))
    r.a[1][1] = cos_exp_m1(a, 4.0 * q);
    r.a[2][1] = sa * ((eq * ep) * ez);            // exp(i(q + p + z))
    r.a[0][2] = (-Sa2) * ((eq * eq) * (epc * epc));   // exp(2i(q - p))
    r.a[1][2] = sa * ((eq * epc) * ez);           // exp(i(q - p + z))
    cem = cos_exp_m1(0.5 * a, z - q);
    r.a[2][2] = cem * (cem + c64{2.0, 0.0});
    for (int h = 0; h < hypercubes; h++) {
        r = square_m1(r);
        r = square_m1(r);
    }
    r.a[0][0].re += 1.0;
    r.a[1][1].re += 1.0;
    r.a[2][2].re += 1.0;
    return r;
}

// matrix_exponential_lie_trotter_8 (I:1810-1925).  As in the reference, the third block
// (generators 4, 5) reuses `sa` from the second block (generators 6, 7) when its amplitude is
// non-zero, and sets it to zero otherwise.
SS_D Mat<3> expo_lt8_one(const double* g, int hypercubes, double precision) {
    Mat<3> r, t1, t2;
    double a = sqrt(g[0] * g[0] + g[1] * g[1]);
    c64 ep, sa;
    double Sa, Cam1;
    if (a > 0) {
        ep = c64{g[0] / a, g[1] / a};
        a = a / precision;
        double sh, ch;
        sincos(0.5 * a, &sh, &ch);
        Sa = sh;
        sa = c64{0.0, -(2.0 * sh * ch) / kSqrt2};
        Cam1 = cos_m1(0.5 * a);
    } else {
        ep = c64{1.0, 0.0};
        Sa = 0;
        sa = c64{0.0, 0.0};
        Cam1 = 0;
    }
    {
        const c64 sep = Sa * ep, sepc = Sa * conj(ep);
        r.a[0][0] = c64{Cam1 * (Cam1 + 2), 0.0};
        r.a[1][0] = sa * ep;
        r.a[2][0] = (-1.0) * (sep * sep);
        r.a[0][1] = sa * conj(ep);
        r.a[1][1] = c64{cos_m1(a), 0.0};
        r.a[2][1] = sa * ep;
        r.a[0][2] = (-1.0) * (sepc * sepc);
        r.a[1][2] = sa * conj(ep);
        r.a[2][2] = c64{Cam1 * (Cam1 + 2), 0.0};
    }
    a = sqrt(g[6] * g[6] + g[7] * g[7]);
    if (a > 0) {
        ep = c64{g[6] / a, g[7] / a};
        a = a / precision;
        double sh, ch;
        sincos(0.5 * a, &sh, &ch);
        Sa = sh;
        sa = c64{0.0, -(2.0 * sh * ch) / kSqrt2};
        Cam1 = cos_m1(0.5 * a);
    } else {
        ep = c64{1.0, 0.0};
        Sa = 0;
        sa = c64{0.0, 0.0};
        Cam1 = 0;
    }
    {
        const c64 sep = Sa * ep, sepc = Sa * conj(ep);
        t1.a[0][0] = c64{Cam1 * (Cam1 + 2), 0.0};
        t1.a[1][0] = sa * ep;
        t1.a[2][0] = (-1.0) * (sep * sep);
        t1.a[0][1] = sa * conj(ep);
        t1.a[1][1] = c64{cos_m1(a), 0.0};
        t1.a[2][1] = (-1.0) * (sa * ep);
        t1.a[0][2] = (-1.0) * (sepc * sepc);
        t1.a[1][2] = (-1.0) * (sa * conj(ep));
        t1.a[2][2] = c64{Cam1 * (Cam1 + 2), 0.0};
    }
    t2 = multiply_m1(r, t1);
    a = sqrt(g[4] * g[4] + g[5] * g[5]);
    if (a > 0) {
        ep = c64{g[4] / a, g[5] / a};
        a = a / precision;
        Sa = sin(a);
        Cam1 = cos_m1(a);
    } else {
        ep = c64{1.0, 0.0};
        Sa = 0;
        sa = c64{0.0, 0.0};
        Cam1 = 0;
    }
    {
        const c64 sep = Sa * ep, sepc = Sa * conj(ep);
        const c64 zero = c64{0.0, 0.0};
        r.a[0][0] = c64{Cam1, 0.0};
        r.a[1][0] = zero;
        r.a[2][0] = (-1.0) * (sep * sep);
        r.a[0][1] = sa * conj(ep);
        r.a[1][1] = zero;
        r.a[2][1] = (-1.0) * (sa * ep);
        r.a[0][2] = (-1.0) * (sepc * sepc);
        r.a[1][2] = zero;
        r.a[2][2] = c64{Cam1, 0.0};
    }
    t1 = multiply_m1(r, t2);
    a = g[2] / precision;
    const double e = g[3] / (3.0 * precision);
    {
        const c64 zero = c64{0.0, 0.0};
        t2.a[0][0] = expm1i(-a - e);
        t2.a[1][0] = zero;
        t2.a[2][0] = zero;
        t2.a[0][1] = zero;
        t2.a[1][1] = expm1i(2.0 * e);
        t2.a[2][1] = zero;
        t2.a[0][2] = zero;
        t2.a[1][2] = zero;
        t2.a[2][2] = expm1i(a - e);
    }
    r = multiply_m1(t1, t2);
    for (int h = 0; h < hypercubes; h++) {
        r = square_m1(r);
        r = square_m1(r);
    }
    r.a[0][0].re += 1.0;
    r.a[1][1].re += 1.0;
    r.a[2][2].re += 1.0;
    return r;
}

}  // namespace spinsim
