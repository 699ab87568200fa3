// Plain FP64 time evolution of one output interval: the reference's get_time_evolution_loop
// (spinsim/__init__.py:797-852) with its integrators (I:622-794), frame transforms (I:582-618) and
// step composition (I:561-580).  All operators live in registers.
//
// An interval's K fine steps may be shared by `lanes` consecutive lanes of a warp: lane l runs
// steps [l K / lanes, (l + 1) K / lanes) and the partial products are combined in step order with
// warp shuffles (the later product multiplies from the left, as append_exponentiation does).
#pragma once
#include "common.cuh"
#include "expo64.cuh"
#include "fields.cuh"

namespace spinsim {

// Lie-algebra dimension of the field vector (I:547-554).
template <int D, int EXPO>
struct LieDim {
    static constexpr int value = (D == 2) ? 3 : (EXPO == EXPO_LIE_TROTTER_8 ? 8 : 4);
};

template <int D, int EXPO>
SS_D Mat<D> exponential64(const double* g, const MethodConfig& m) {
    if constexpr (D == 2) {
        if constexpr (EXPO == EXPO_ANALYTIC) return expo_analytic_half(g);
        else return expo_lt_half(g, m.hypercubes, m.precision);
    } else {
        if constexpr (EXPO == EXPO_LIE_TROTTER_8) return expo_lt8_one(g, m.hypercubes, m.precision);
        else return expo_lt_one(g, m.hypercubes, m.precision);
    }
}

// transform_frame_* (I:582-618).  Division by the unit winding w is written as multiplication by
// its conjugate.
template <int D, int EXPO>
SS_D void transform_frame64(double* s, double rw, c64 w) {
    if constexpr (D == 2) {
        const c64 wc = conj(w);
        const c64 X = c64{s[0], s[1]} * (wc * wc);
        s[0] = X.re;
        s[1] = X.im;
        s[2] = s[2] - 2.0 * rw;
    } else if constexpr (EXPO == EXPO_LIE_TROTTER_8) {
        const c64 wc = conj(w);
        c64 X = c64{s[0], s[1]} * wc;
        s[0] = X.re;
        s[1] = X.im;
        s[2] = s[2] - rw;
        X = (c64{s[4], s[5]} * wc) * wc;
        s[4] = X.re;
        s[5] = X.im;
        X = c64{s[6], s[7]} * wc;
        s[6] = X.re;
        s[7] = X.im;
    } else {
        const c64 X = c64{s[0], s[1]} * conj(w);
        s[0] = X.re;
        s[1] = X.im;
        s[2] = s[2] - rw;
    }
}

// Evolve one output interval.  Every lane of the warp must call this (shuffles use the full mask);
// lanes with `active == false` do no steps and write nothing.
template <int D, int INTEG, int EXPO, int FIELD>
SS_D void interval64(const MethodConfig& m, const Instance& inst, const FieldDesc& f, int64_t index, bool active,
                     int lane_in_group, double* time_out, double* u_out) {
    constexpr int L = LieDim<D, EXPO>::value;
    const int lanes = m.lanes;
    const double dt = inst.dt_int, dt_out = inst.dt_out;
    // I:818, rounded as the reference rounds it (no fused multiply-add), so time[] is bit-exact
    const double t_c = __dadd_rn(inst.t0, __dmul_rn(dt_out, (double)(inst.interval0 + index)));
    double s0[8], s1[8];
#pragma unroll
    for (int k = 0; k < 8; k++) s0[k] = 0.0;
    double rw = 0.0;
    if (active && m.rotating) {  // I:823-829
        sample_field<FIELD, L>(f, t_c + dt_out / 2, s0);
        rw = s0[2];
        if (D == 2) rw /= 2;
    }
    const int K = active ? inst.n_fine : 0;
    const int j0 = (int)(((int64_t)K * lane_in_group) / lanes);
    const int j1 = (int)(((int64_t)K * (lane_in_group + 1)) / lanes);
    double t_fine = t_c;
    for (int j = 0; j < j0; j++) t_fine += dt;  // the reference's running sum (I:836)

    Mat<D> u;
    set_identity(u);
    TableCursor cur[L];  // per-channel table cursors for the increasing sample times of the steps
#pragma unroll
    for (int c = 0; c < L; c++) cur[c] = TableCursor{};
    const double a_lo = 0.5 * dt * (1.0 - 1.0 / kSqrt3);
    const double a_hi = 0.5 * dt * (1.0 + 1.0 / kSqrt3);
    const double w0 = (1.5 + kSqrt3) / 6.0, w1 = (1.5 - kSqrt3) / 6.0;
    for (int j = j0; j < j1; j++) {
        if constexpr (INTEG == INTEG_EULER) {
            // I:759-791
#pragma unroll
            for (int k = 0; k < L; k++) s0[k] = 0.0;
            double ts = t_fine + 0.5 * dt - t_c;
            c64 wa = c64{1.0, 0.0};
            if (m.rotating) sincos(rw * ts, &wa.im, &wa.re);
            ts += t_c;
            sample_field<FIELD, L>(f, ts, s0, cur);
            if (m.rotating) transform_frame64<D, EXPO>(s0, rw, wa);
            double g[L];
#pragma unroll
            for (int k = 0; k < L; k++) g[k] = dt * s0[k];
            u = matmul(exponential64<D, EXPO>(g, m), u);
        } else {
            // CF4: I:624-686; Heun: I:693-752
#pragma unroll
            for (int k = 0; k < L; k++) {
                s0[k] = 0.0;
                s1[k] = 0.0;
            }
            double ts = (INTEG == INTEG_CF4) ? ((t_fine + a_lo) - t_c) : (t_fine - t_c);
            c64 wa = c64{1.0, 0.0}, wb = c64{1.0, 0.0};
            if (m.rotating) sincos(rw * ts, &wa.im, &wa.re);
            ts += t_c;
            sample_field<FIELD, L>(f, ts, s0, cur);
            ts = (INTEG == INTEG_CF4) ? ((t_fine + a_hi) - t_c) : (t_fine + dt - t_c);
            if (m.rotating) sincos(rw * ts, &wb.im, &wb.re);
            ts += t_c;
            sample_field<FIELD, L>(f, ts, s1, cur);
            if (m.rotating) {
                transform_frame64<D, EXPO>(s0, rw, wa);
                transform_frame64<D, EXPO>(s1, rw, wb);
            }
            double g[L];
            if constexpr (INTEG == INTEG_CF4) {
#pragma unroll
                for (int k = 0; k < L; k++) g[k] = dt * (w0 * s0[k] + w1 * s1[k]);
            } else {
#pragma unroll
                for (int k = 0; k < L; k++) g[k] = dt * s0[k] / 2;
            }
            u = matmul(exponential64<D, EXPO>(g, m), u);
            if constexpr (INTEG == INTEG_CF4) {
#pragma unroll
                for (int k = 0; k < L; k++) g[k] = dt * (w1 * s0[k] + w0 * s1[k]);
            } else {
#pragma unroll
                for (int k = 0; k < L; k++) g[k] = dt * s1[k] / 2;
            }
            u = matmul(exponential64<D, EXPO>(g, m), u);
        }
        t_fine += dt;
    }

    // Combine the lanes' partial products in step order: later steps multiply from the left.
    for (int s = 1; s < lanes; s <<= 1) {
        const Mat<D> later = shfl_down_mat(u, s);
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
    double2* dst = reinterpret_cast<double2*>(u_out) + index * (D * D);
#pragma unroll
    for (int i = 0; i < D; i++)
#pragma unroll
        for (int k = 0; k < D; k++) dst[i * D + k] = make_double2(u.a[i][k].re, u.a[i][k].im);
}

}  // namespace spinsim
