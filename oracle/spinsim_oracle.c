/*
 * spinsim oracle: a CPU restatement of the reference's evaluation path, in C.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker the parity tests compare the sm_100a kernels
 * against, and the CPU baseline that bench.py times beside them.  The product path
 * (spinsim_b200 and its CUDA library) never links, loads or calls it.
 *
 * Reference: alexander-tritt-monash/spinsim, spinsim/__init__.py (one file; cited as I:line).
 * Each function cites the reference lines it restates and keeps the reference's operation order,
 * including its residual ("minus one") forms and the quirks of the eight-generator exponential.
 * The restatement is pinned against fixtures produced by running the reference itself
 * (tests/golden/make_golden.py -> tests/golden/golden.npz).
 *
 * Layouts (all row-major, complex as interleaved re/im doubles like numpy complex128):
 *   time[N], U[N][d][d] complex, state[N][d] complex, spin[N][3].
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double complex cplx;

#define SQRT2 1.4142135623730951
#define SQRT3 1.7320508075688772
#define TAU 6.283185307179586

/* ---------------------------------------------------------------- configuration */
enum { INTEG_CF4 = 0, INTEG_EULER = 1, INTEG_HEUN = 2 };
enum { EXPO_ANALYTIC = 0, EXPO_LIE_TROTTER = 1, EXPO_LIE_TROTTER_8 = 2 };

typedef struct {
    int dim;          /* 2 (spin half) or 3 (spin one) */
    int integration;  /* INTEG_* */
    int expo;         /* EXPO_* (already resolved: analytic only for dim 2) */
    int rotating;     /* use_rotating_frame */
    int n_squares;    /* number_of_squares */
} oracle_config;

/* Interpolation table for one field channel (generate_interpolation_sampler, I:1941-2147). */
typedef struct {
    const double* time;
    const double* amplitude;
    int64_t size;
    int order;          /* 0, 1 or 3 */
    int zero_boundary;
} oracle_table;

typedef struct {
    int code;                    /* field code, see field_eval */
    const oracle_table* tables;  /* code 9: one table per channel (NULL time = no table) */
    int n_tables;
} oracle_field;

/* ---------------------------------------------------------------- interpolation sampler */
/* find_time_index, I:2026-2061: guessed index from equal spacing, then bisection. */
static int64_t find_time_index(const oracle_table* tb, double ts, double* interp) {
    const double* time = tb->time;
    int64_t size = tb->size;
    *interp = 0.0;
    if (time[0] <= ts && ts <= time[size - 1]) {
        int64_t idx = (int64_t)((ts - time[0]) / (time[1] - time[0]));
        int low_enough = 0, high_enough = 1;
        if (idx + 1 < size) {
            low_enough = time[idx] <= ts;
            high_enough = ts <= time[idx + 1];
        } else {
            idx = size;
        }
        if (!(low_enough && high_enough)) {
            int64_t idx_max = size - 1, idx_min = 0, get_out = size;
            while (!(low_enough && high_enough)) {
                if (!low_enough) idx_max = idx; else idx_min = idx;
                idx = (int64_t)((double)(idx_max + idx_min) / 2.0);
                low_enough = 0;
                high_enough = 1;
                if (idx + 1 < size) {
                    low_enough = time[idx] <= ts;
                    high_enough = ts <= time[idx + 1];
                }
                get_out -= 1;
                if (get_out == 0) return -1;
            }
        }
        *interp = (ts - time[idx]) / (time[idx + 1] - time[idx]);
        return idx;
    }
    return -1;
}

/* sampler bodies, I:2065-2140 (order 0: ZOH, 1: linear, 3: cubic Hermite with finite differences). */
double oracle_interpolate(const oracle_table* tb, double ts) {
    const double* time = tb->time;
    const double* amp = tb->amplitude;
    int64_t size = tb->size;
    if (!tb->zero_boundary) {
        if (ts <= time[0]) return amp[0];
        if (ts >= time[size - 1]) return amp[size - 1];
    }
    double u;
    int64_t i = find_time_index(tb, ts, &u);
    if (tb->order == 0) {
        return i >= 0 ? amp[i] : 0.0;
    }
    if (!(i >= 0 && i + 1 < size)) return 0.0;
    if (tb->order == 1) {
        return amp[i] * (1 - u) + amp[i + 1] * u;
    }
    double g_mid = (time[i] != time[i + 1]) ? (amp[i + 1] - amp[i]) / (time[i + 1] - time[i]) : 0.0;
    double g_left;
    if (i == 0) g_left = g_mid;
    else if (time[i - 1] != time[i]) g_left = 0.5 * ((amp[i] - amp[i - 1]) / (time[i] - time[i - 1]) + g_mid);
    else g_left = 0.0;
    g_left *= (time[i + 1] - time[i]);
    double g_right;
    if (i + 2 == size) g_right = g_mid;
    else if (time[i + 1] != time[i + 2]) g_right = 0.5 * ((amp[i + 2] - amp[i + 1]) / (time[i + 2] - time[i + 1]) + g_mid);
    else g_right = 0.0;
    g_right *= (time[i + 1] - time[i]);
    double u2 = u * u, u3 = u2 * u;
    return amp[i] * (2 * u3 - 3 * u2 + 1) + amp[i + 1] * (-2 * u3 + 3 * u2) + g_left * (u3 - 2 * u2 + u) +
           g_right * (u3 - u2);
}

/* ---------------------------------------------------------------- fields */
/* The test fields of tests/golden/fields.py, restated.  Code 9 is the tabulated field of
 * tests/golden/make_golden.py (make_table_field): x = p0 sx(t), y = p1 sy(t), z = p2 + p3 sz(t),
 * q = 0, with three interpolation tables. */
static void field_eval(const oracle_field* f, double t, const double* p, int64_t np, double* out) {
    (void)np;
    switch (f->code) {
    case 1: /* larmor */
        out[0] = 0; out[1] = 0; out[2] = TAU * 1000;
        break;
    case 2: /* rabi */
        out[0] = 2 * p[1] * cos(p[0] * t); out[1] = 0; out[2] = p[0];
        break;
    case 3: /* rabi_one */
        out[0] = 2 * p[1] * cos(p[0] * t); out[1] = 0; out[2] = p[0]; out[3] = 0;
        break;
    case 4: /* detuned_rabi */
        out[0] = TAU * 2e3 * cos(TAU * 840e3 * t); out[1] = 0; out[2] = TAU * (840e3 + p[0]); out[3] = 0;
        break;
    case 5: { /* gaussian_ensemble */
        double a = (t - 10e-6) / 2e-6;
        out[0] = TAU * 50e3 * exp(-0.5 * (a * a)); out[1] = 0; out[2] = TAU * p[0];
        break;
    }
    case 6: /* full_su3 */
        out[0] = TAU * 2000 * cos(p[0] * t); out[1] = 0; out[2] = p[0];
        out[3] = TAU * 1000; out[4] = TAU * 1000; out[5] = TAU * 1000; out[6] = TAU * 1000; out[7] = TAU * 1000;
        break;
    case 7: /* gaussian_pulse */
        out[0] = M_PI / sqrt(TAU) * exp(-0.5 * (t * t)); out[1] = 0.0; out[2] = 0.0;
        break;
    case 8: /* tones */
        for (int axis = 0; axis < 3; axis++) {
            double value = p[axis];
            for (int k = 0; k < 8; k++) {
                int b = 4 + 24 * axis + 3 * k;
                value += p[b + 1] * sin(p[b] * t + p[b + 2]);
            }
            out[axis] = value;
        }
        out[3] = p[3];
        break;
    case 9: /* tabulated */
        out[0] = p[0] * oracle_interpolate(&f->tables[0], t);
        out[1] = p[1] * oracle_interpolate(&f->tables[1], t);
        out[2] = p[2] + p[3] * oracle_interpolate(&f->tables[2], t);
        out[3] = 0;
        break;
    default:
        break;
    }
}

/* ---------------------------------------------------------------- small helpers, I:1552-1566 */
static inline cplx expm1i(double x) { double s = sin(x / 2); return -2 * (s * s) + I * sin(x); }
static inline cplx cos_exp_m1(double c, double e) { return (expm1i(c + e) + expm1i(-c + e)) / 2; }
static inline double cos_m1(double x) { double s = sin(x / 2); return -2 * (s * s); }
static inline cplx conjc(cplx z) { return creal(z) - I * cimag(z); }

#define M(a, r, c) a[(r) * 3 + (c)] /* all matrices stored with row stride 3 */

/* matrix_multiply, I:1594-1600 (d = 2) and I:1722-1734 (d = 3) */
static void matmul(int d, const cplx* l, const cplx* r, cplx* out) {
    for (int i = 0; i < d; i++)
        for (int j = 0; j < d; j++) {
            cplx acc = M(l, i, 0) * M(r, 0, j);
            for (int k = 1; k < d; k++) acc = acc + M(l, i, k) * M(r, k, j);
            M(out, i, j) = acc;
        }
}

/* matrix_square_m1, I:1602-1608 (d = 2) and I:1736-1748 (d = 3): (2 + A)A, entry (i, j) summed
 * over k in order, the k == i term written (2 + A[i][i]) A[i][j] as the reference groups it. */
static void square_m1(int d, const cplx* a, cplx* out) {
    for (int i = 0; i < d; i++)
        for (int j = 0; j < d; j++) {
            cplx acc = 0;
            for (int k = 0; k < d; k++) {
                cplx term = (k == i) ? (2 + M(a, i, i)) * M(a, i, j) : M(a, i, k) * M(a, k, j);
                acc = (k == 0) ? term : acc + term;
            }
            M(out, i, j) = acc;
        }
}

/* matrix_multiply_m1, I:1610-1616 (d = 2) and I:1750-1762 (d = 3): (l + r) + l r */
static void multiply_m1(int d, const cplx* l, const cplx* r, cplx* out) {
    for (int i = 0; i < d; i++)
        for (int j = 0; j < d; j++) {
            cplx acc = M(l, i, 0) * M(r, 0, j);
            for (int k = 1; k < d; k++) acc = acc + M(l, i, k) * M(r, k, j);
            M(out, i, j) = (M(l, i, j) + M(r, i, j)) + acc;
        }
}

/* ---------------------------------------------------------------- exponentials */
/* matrix_exponential_analytic (spin half), I:1618-1642 */
static void expo_analytic_half(const double* g, cplx* r) {
    double x = g[0], y = g[1], z = g[2];
    double rr = sqrt(x * x + y * y + z * z);
    if (rr > 0) {
        x /= rr; y /= rr; z /= rr;
        cplx c = cos_exp_m1(rr / 2, 0);
        double s = sin(rr / 2);
        M(r, 0, 0) = c - I * z * s + 1;
        M(r, 1, 0) = (y - I * x) * s;
        M(r, 0, 1) = -(y + I * x) * s;
        M(r, 1, 1) = c + I * z * s + 1;
    } else {
        M(r, 0, 0) = 1; M(r, 1, 0) = 0; M(r, 0, 1) = 0; M(r, 1, 1) = 1;
    }
}

/* matrix_exponential_lie_trotter (spin half), I:1644-1673 */
static void expo_lt_half(const double* g, int hypercubes, double precision, cplx* r) {
    double a = sqrt(g[0] * g[0] + g[1] * g[1]);
    cplx ep = (a > 0) ? (g[0] + I * g[1]) / a : 1;
    a = a / precision;
    cplx Sa = -I * sin(a / 2);
    double z = g[2] / (2 * precision);
    M(r, 0, 0) = cos_exp_m1(a / 2, -z);
    M(r, 1, 0) = Sa * ep;
    M(r, 0, 1) = Sa / ep;
    M(r, 1, 1) = cos_exp_m1(a / 2, z);
    cplx tmp[9];
    for (int h = 0; h < hypercubes; h++) {
        square_m1(2, r, tmp);
        square_m1(2, tmp, r);
    }
    M(r, 0, 0) += 1;
    M(r, 1, 1) += 1;
}

/* matrix_exponential_lie_trotter (spin one), I:1768-1808 */
static void expo_lt_one(const double* g, int hypercubes, double precision, cplx* r) {
    double a = sqrt(g[0] * g[0] + g[1] * g[1]);
    double p = (a > 0) ? atan2(g[1], g[0]) : 0;
    a = a / precision;
    double Sa = sin(a / 2);
    cplx sa = -I * sin(a) / SQRT2;
    double z = g[2] / (2 * precision);
    double q = g[3] / (6 * precision);
    cplx cem = cos_exp_m1(a / 2, -z - q);
    M(r, 0, 0) = cem * (cem + 2);
    M(r, 1, 0) = sa * cexp(I * (q + p - z));
    M(r, 2, 0) = -(Sa * Sa) * cexp(2 * I * (p - q));
    M(r, 0, 1) = sa * cexp(I * (q - p - z));
    M(r, 1, 1) = cos_exp_m1(a, 4 * q);
    M(r, 2, 1) = sa * cexp(I * (q + p + z));
    M(r, 0, 2) = -(Sa * Sa) * cexp(2 * I * (q - p));
    M(r, 1, 2) = sa * cexp(I * (q - p + z));
    cem = cos_exp_m1(a / 2, z - q);
    M(r, 2, 2) = cem * (cem + 2);
    cplx tmp[9];
    for (int h = 0; h < hypercubes; h++) {
        square_m1(3, r, tmp);
        square_m1(3, tmp, r);
    }
    M(r, 0, 0) += 1; M(r, 1, 1) += 1; M(r, 2, 2) += 1;
}

/* matrix_exponential_lie_trotter_8 (spin one), I:1810-1925.  Kept as written, including that the
 * third block (generators 4, 5) reuses `sa` from the second block when its amplitude is non-zero. */
static void expo_lt8_one(const double* g, int hypercubes, double precision, cplx* r) {
    cplx t1[9], t2[9];
    double a = sqrt(g[0] * g[0] + g[1] * g[1]);
    cplx ep, sa;
    double Sa, Cam1;
    if (a > 0) {
        ep = (g[0] + I * g[1]) / a;
        a = a / precision;
        Sa = sin(a / 2);
        sa = -I * sin(a) / SQRT2;
        Cam1 = cos_m1(a / 2);
    } else {
        ep = 1; Sa = 0; sa = 0; Cam1 = 0;
    }
    M(r, 0, 0) = Cam1 * (Cam1 + 2);
    M(r, 1, 0) = sa * ep;
    M(r, 2, 0) = -((Sa * ep) * (Sa * ep));
    M(r, 0, 1) = sa * conjc(ep);
    M(r, 1, 1) = cos_m1(a);
    M(r, 2, 1) = sa * ep;
    M(r, 0, 2) = -((Sa * conjc(ep)) * (Sa * conjc(ep)));
    M(r, 1, 2) = sa * conjc(ep);
    M(r, 2, 2) = Cam1 * (Cam1 + 2);

    a = sqrt(g[6] * g[6] + g[7] * g[7]);
    if (a > 0) {
        ep = (g[6] + I * g[7]) / a;
        a = a / precision;
        Sa = sin(a / 2);
        sa = -I * sin(a) / SQRT2;
        Cam1 = cos_m1(a / 2);
    } else {
        ep = 1; Sa = 0; sa = 0; Cam1 = 0;
    }
    M(t1, 0, 0) = Cam1 * (Cam1 + 2);
    M(t1, 1, 0) = sa * ep;
    M(t1, 2, 0) = -((Sa * ep) * (Sa * ep));
    M(t1, 0, 1) = sa * conjc(ep);
    M(t1, 1, 1) = cos_m1(a);
    M(t1, 2, 1) = -sa * ep;
    M(t1, 0, 2) = -((Sa * conjc(ep)) * (Sa * conjc(ep)));
    M(t1, 1, 2) = -sa * conjc(ep);
    M(t1, 2, 2) = Cam1 * (Cam1 + 2);
    multiply_m1(3, r, t1, t2);

    a = sqrt(g[4] * g[4] + g[5] * g[5]);
    if (a > 0) {
        ep = (g[4] + I * g[5]) / a;
        a = a / precision;
        Sa = sin(a);
        Cam1 = cos_m1(a);
    } else {
        ep = 1; Sa = 0; sa = 0; Cam1 = 0;
    }
    M(r, 0, 0) = Cam1;
    M(r, 1, 0) = 0.0;
    M(r, 2, 0) = -((Sa * ep) * (Sa * ep));
    M(r, 0, 1) = sa * conjc(ep);
    M(r, 1, 1) = 0.0;
    M(r, 2, 1) = -sa * ep;
    M(r, 0, 2) = -((Sa * conjc(ep)) * (Sa * conjc(ep)));
    M(r, 1, 2) = 0.0;
    M(r, 2, 2) = Cam1;
    multiply_m1(3, r, t2, t1);

    a = g[2] / precision;
    double e = g[3] / (3 * precision);
    M(t2, 0, 0) = expm1i(-a - e);
    M(t2, 1, 0) = 0.0; M(t2, 2, 0) = 0.0; M(t2, 0, 1) = 0.0;
    M(t2, 1, 1) = expm1i(2 * e);
    M(t2, 2, 1) = 0.0; M(t2, 0, 2) = 0.0; M(t2, 1, 2) = 0.0;
    M(t2, 2, 2) = expm1i(a - e);
    multiply_m1(3, t1, t2, r);
    for (int h = 0; h < hypercubes; h++) {
        square_m1(3, r, t1);
        square_m1(3, t1, r);
    }
    M(r, 0, 0) += 1; M(r, 1, 1) += 1; M(r, 2, 2) += 1;
}

/* ---------------------------------------------------------------- one output interval */
typedef struct {
    oracle_config cfg;
    int lie_dim;
    int hypercubes;
    double precision;
} prepared;

static void prepare(const oracle_config* cfg, prepared* pp) {
    pp->cfg = *cfg;
    /* Utilities.__init__, I:1547-1550 */
    int h = (int)ceil(cfg->n_squares / 2.0);
    if (h < 0) h = 0;
    pp->hypercubes = h;
    pp->precision = pow(4.0, h);
    /* compile_time_evolver, I:547-554 */
    pp->lie_dim = (cfg->dim == 2) ? 3 : (cfg->expo == EXPO_LIE_TROTTER_8 ? 8 : 4);
}

/* append_exponentiation, I:561-580: U_out <- exp(field) U_out */
static void append_exponentiation(const prepared* pp, const double* g, cplx* u) {
    cplx e[9], old[9];
    int d = pp->cfg.dim;
    if (pp->cfg.expo == EXPO_ANALYTIC) expo_analytic_half(g, e);
    else if (pp->cfg.expo == EXPO_LIE_TROTTER) {
        if (d == 2) expo_lt_half(g, pp->hypercubes, pp->precision, e);
        else expo_lt_one(g, pp->hypercubes, pp->precision, e);
    } else expo_lt8_one(g, pp->hypercubes, pp->precision, e);
    memcpy(old, u, sizeof(old));
    matmul(d, e, old, u);
}

/* transform_frame_*, I:582-618 */
static void transform_frame(const prepared* pp, double* s, double rw, cplx w) {
    if (!pp->cfg.rotating) return;
    if (pp->cfg.dim == 3) {
        if (pp->cfg.expo == EXPO_LIE_TROTTER_8) {
            cplx X = (s[0] + I * s[1]) * conjc(w);
            s[0] = creal(X); s[1] = cimag(X);
            s[2] = s[2] - rw;
            X = (s[4] + I * s[5]) * conjc(w) * conjc(w);
            s[4] = creal(X); s[5] = cimag(X);
            X = (s[6] + I * s[7]) * conjc(w);
            s[6] = creal(X); s[7] = cimag(X);
        } else {
            cplx X = (s[0] + I * s[1]) / w;
            s[0] = creal(X); s[1] = cimag(X);
            s[2] = s[2] - rw;
        }
    } else {
        cplx X = (s[0] + I * s[1]) / (w * w);
        s[0] = creal(X); s[1] = cimag(X);
        s[2] = s[2] - 2 * rw;
    }
}

/* get_time_evolution_loop, I:797-852, with the integrators of I:622-794 */
static void time_evolution_interval(const prepared* pp, const oracle_field* f, const double* sweep, int64_t nsweep,
                                    int64_t index, double t0, double dt_int, double dt_out, double* time_out,
                                    double* u_out) {
    const int d = pp->cfg.dim, L = pp->lie_dim;
    double s[3][8];
    cplx w[4];
    cplx u[9];
    time_out[index] = t0 + dt_out * index;
    double t_c = time_out[index];
    double t_fine = t_c;
    for (int i = 0; i < 9; i++) u[i] = 0;
    for (int i = 0; i < d; i++) M(u, i, i) = 1;
    memset(s, 0, sizeof(s));
    s[0][2] = 0;
    if (pp->cfg.rotating) field_eval(f, t_c + dt_out / 2, sweep, nsweep, s[0]);
    double rw = s[0][2];
    if (d == 2) rw /= 2;
    int K = (int)floor(dt_out / dt_int + 0.5);
    const double w0 = (1.5 + SQRT3) / 6, w1 = (1.5 - SQRT3) / 6;
    for (int j = 0; j < K; j++) {
        if (pp->cfg.integration == INTEG_CF4) {
            /* get_field_integration_magnus_cf4, I:624-652 */
            for (int k = 0; k < L; k++) { s[0][k] = 0; s[1][k] = 0; }
            double ts = ((t_fine + 0.5 * dt_int * (1 - 1 / SQRT3)) - t_c);
            w[0] = cexp(I * rw * ts);
            ts += t_c;
            field_eval(f, ts, sweep, nsweep, s[0]);
            ts = ((t_fine + 0.5 * dt_int * (1 + 1 / SQRT3)) - t_c);
            w[1] = cexp(I * rw * ts);
            ts += t_c;
            field_eval(f, ts, sweep, nsweep, s[1]);
            /* append_exponentiation_integration_magnus_cf4, I:655-686 */
            transform_frame(pp, s[0], rw, w[0]);
            transform_frame(pp, s[1], rw, w[1]);
            for (int k = 0; k < L; k++) s[2][k] = dt_int * (w0 * s[0][k] + w1 * s[1][k]);
            append_exponentiation(pp, s[2], u);
            for (int k = 0; k < L; k++) s[2][k] = dt_int * (w1 * s[0][k] + w0 * s[1][k]);
            append_exponentiation(pp, s[2], u);
        } else if (pp->cfg.integration == INTEG_HEUN) {
            /* get_field_integration_heun, I:693-721 and append, I:724-752 */
            for (int k = 0; k < L; k++) { s[0][k] = 0; s[1][k] = 0; }
            double ts = t_fine - t_c;
            w[0] = cexp(I * rw * ts);
            ts += t_c;
            field_eval(f, ts, sweep, nsweep, s[0]);
            ts = t_fine + dt_int - t_c;
            w[1] = cexp(I * rw * ts);
            ts += t_c;
            field_eval(f, ts, sweep, nsweep, s[1]);
            transform_frame(pp, s[0], rw, w[0]);
            transform_frame(pp, s[1], rw, w[1]);
            for (int k = 0; k < L; k++) s[2][k] = dt_int * s[0][k] / 2;
            append_exponentiation(pp, s[2], u);
            for (int k = 0; k < L; k++) s[2][k] = dt_int * s[1][k] / 2;
            append_exponentiation(pp, s[2], u);
        } else {
            /* get_field_integration_euler, I:759-774 and append, I:777-791 */
            for (int k = 0; k < L; k++) s[0][k] = 0;
            double ts = t_fine + 0.5 * dt_int - t_c;
            w[0] = cexp(I * rw * ts);
            ts += t_c;
            field_eval(f, ts, sweep, nsweep, s[0]);
            transform_frame(pp, s[0], rw, w[0]);
            for (int k = 0; k < L; k++) s[0][k] = dt_int * s[0][k];
            append_exponentiation(pp, s[0], u);
        }
        t_fine += dt_int;
    }
    if (pp->cfg.rotating) {
        /* I:839-852 */
        cplx wo = cexp(I * rw * dt_out);
        M(u, 0, 0) /= wo;
        M(u, 0, 1) /= wo;
        if (d > 2) {
            M(u, 0, 2) /= wo;
            M(u, 2, 0) *= wo; M(u, 2, 1) *= wo; M(u, 2, 2) *= wo;
        } else {
            M(u, 1, 0) *= wo; M(u, 1, 1) *= wo;
        }
    }
    double* dst = u_out + (size_t)index * d * d * 2;
    for (int i = 0; i < d; i++)
        for (int k = 0; k < d; k++) {
            dst[(i * d + k) * 2] = creal(M(u, i, k));
            dst[(i * d + k) * 2 + 1] = cimag(M(u, i, k));
        }
}

/* ---------------------------------------------------------------- public entry points */
/* get_time_evolution, I:855-896 (CPU branch: prange over output intervals).
 * first/count select a sub-range of output intervals (for bounded timing samples). */
int oracle_time_evolution(const oracle_config* cfg, const oracle_field* f, const double* sweep, int64_t nsweep,
                          double t0, double dt_int, double dt_out, int64_t n_out, int64_t first, int64_t count,
                          double* time_out, double* u_out, int n_threads) {
    prepared pp;
    prepare(cfg, &pp);
    if (cfg->dim != 2 && cfg->dim != 3) return -1;
    if (first < 0 || count < 0 || first + count > n_out) return -1;
#ifdef _OPENMP
    if (n_threads <= 0) n_threads = omp_get_max_threads();
#pragma omp parallel for schedule(static) num_threads(n_threads)
#endif
    for (int64_t i = first; i < first + count; i++)
        time_evolution_interval(&pp, f, sweep, nsweep, i, t0, dt_int, dt_out, time_out, u_out);
    (void)n_threads;
    return 0;
}

/* get_state, I:1089-1111: state[0] = psi0, state[i] = U[i-1] state[i-1] (serial). */
void oracle_state(int d, const double* u, const double* psi0, int64_t n, double* state) {
    const cplx* U = (const cplx*)u;
    cplx* S = (cplx*)state;
    const cplx* P = (const cplx*)psi0;
    for (int64_t i = 0; i < n; i++) {
        for (int x = 0; x < d; x++) {
            cplx acc = 0;
            if (i > 0) {
                for (int z = 0; z < d; z++) acc += U[((i - 1) * d + x) * d + z] * S[(i - 1) * d + z];
            } else {
                acc += P[x];
            }
            S[i * d + x] = acc;
        }
    }
}

/* get_spin, I:899-959 (CPU branch). */
void oracle_spin(int d, const double* state, int64_t n, double* spin) {
    const cplx* S = (const cplx*)state;
    for (int64_t i = 0; i < n; i++) {
        const cplx* s = S + i * d;
        if (d == 2) {
            spin[i * 3 + 0] = creal(s[0] * conjc(s[1]));
            spin[i * 3 + 1] = creal(I * s[0] * conjc(s[1]));
            spin[i * 3 + 2] = 0.5 * (creal(s[0]) * creal(s[0]) + cimag(s[0]) * cimag(s[0]) -
                                     creal(s[1]) * creal(s[1]) - cimag(s[1]) * cimag(s[1]));
        } else {
            spin[i * 3 + 0] = creal(2 * conjc(s[1]) * (s[0] + s[2]) / SQRT2);
            spin[i * 3 + 1] = creal(2 * I * conjc(s[1]) * (s[0] - s[2]) / SQRT2);
            spin[i * 3 + 2] = creal(s[0]) * creal(s[0]) + cimag(s[0]) * cimag(s[0]) -
                              creal(s[2]) * creal(s[2]) - cimag(s[2]) * cimag(s[2]);
        }
    }
}

int oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
