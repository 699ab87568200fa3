// FP32-bulk time evolution of tone fields with the field samples formed on the FP64 tensor path.
//
// The reference samples its field once per Gauss point of every fine step of every output interval
// (get_field_integration_magnus_cf4, spinsim/__init__.py:624-652).  For a tone field
//     B_c(t_c + tau) = bias_c + sum_k A_k sin(w_k (t_c + tau) + phi_k)
//                    = bias_c + sum_k [Re L_ck sin(w_k tau) + Im L_ck cos(w_k tau)],  L_ck = A_k exp(i (w_k t_c + phi_k)),
// so the samples of a block of output intervals (rows, through L) at a block of sample offsets tau
// (columns, through sin / cos) are a matrix product with inner dimension 2 x (tones per channel).
// That product runs as mma.sync.m8n8k4.f64 (FP64 in, FP64 accumulate: the samples are exact to FP64
// rounding), which takes eight multiply-adds per lane per instruction instead of one.
//
// Mapping.  A CTA takes a tile of kDmmaTile consecutive output intervals of one instance; warp w
// takes intervals 8 w .. 8 w + 7 (the eight rows of the m8n8k4 product).  Each interval's K fine
// steps are split into kDmmaSegments consecutive segments, one per lane of a quad: in the
// accumulator layout lane 4 g + q holds row g, columns 2 q and 2 q + 1, which are made to be the
// two Gauss points of one step of segment q.  So every lane receives exactly the two field
// samples of its own step, runs the step's exponentials and keeps the FP64 product of its
// segment; the four segment products are combined once per interval with quad shuffles (later
// segments multiply from the left, as append_exponentiation does, I:561-580).
//
// Operands.  A (8 x 4 per k-step): lane 4 g + q holds L of interval g for tone 2 s + q / 2, real
// part for even q and imaginary part for odd q, computed once per tile with FP64 sincos.  B (4 x 8):
// lane 4 g + q needs sin / cos (w tau) for that tone at the step of segment g / 2, Gauss point
// g % 2.  These depend on the instance only, not on the interval, so the CTA builds them in shared
// memory: 192 phasor recurrences exp(i w tau) (channel, tone, segment, Gauss point) advanced by
// exp(i w dt) per step in FP64, written in lane order so that every B load is one conflict-free
// 8-byte load per lane.  The table is double-buffered in phases of kDmmaPhase steps (one CTA barrier
// per phase).  The accumulator starts at the channel bias.
//
// Step.  The reference's Magnus CF4 (I:655-686) composes two exponentials per step; its order-four
// Magnus expansion at the same Gauss points, exp(g), g = (h/2)(b1 + b2) + (sqrt3 h^2 / 12) b2 x b1
// (the commutator [A2, A1] of A = -i b.J is -i (b2 x b1).J; Blanes, Casas and Ros, BIT 40 (2000)),
// is the same map to O(h^5): one SU(2) exponential per step.  A tile takes it when the step is small
// against the field, theta = h (|B|max + w_max) <= kMagnusTheta, and CF4 otherwise.  The frame
// transform, the sum and difference of the samples and the exponential's linear part stay in FP64;
// the commutator and the exponential's O(|g|^2) remainder are FP32, the interval product FP64
// (su2_apply_split).  On the benchmark's longest instances (theta = 0.07) the two compositions agree
// to 1e-11 in the final state.  Instances with more than kBulkTones
// tones on a channel, or spin one with a quadratic shift, take the per-interval path (interval32,
// CF4) inside the same kernel.
//
// Scan partials.  A CTA tile is one state scan tile (scan.cuh).  Each interval's lab-frame operator is
// an SU(2) pair (spin one: its representation), so each warp also multiplies its eight rows' pairs
// with three shuffle rounds and writes the product (4 doubles); the scan's prefix kernel combines a
// tile's four warp products and the scan launches no tile products pass over U.
#pragma once
#include "common.cuh"
#include "evolve32.cuh"

namespace spinsim {

constexpr int kDmmaSegments = 4;                             // lanes (time segments) per interval
#ifndef SPINSIM_DMMA_PHASE
#define SPINSIM_DMMA_PHASE 5
#endif
// Steps per segment in one table buffer: 5 divides the 25-step segments of K = 100 (1 us output
// steps of 10 ns), so no phase is a short remainder; 4 was 1% slower there.
constexpr int kDmmaPhase = SPINSIM_DMMA_PHASE;
// Largest step size bound theta = h (|B|max + w_max) for which a tile takes the Magnus step.  The
// Magnus and CF4 steps differ by O(theta^5) per step: measured 4.6e-6 at theta = 6.7 (one 1 us step)
// and 1e-11 over 10^6 steps at theta = 0.07, i.e. about 3e-10 theta^5 per step, so at theta <= 0.1
// below 4e-15 per step, 4e-9 over 10^6 steps.
constexpr double kMagnusTheta = 0.1;
constexpr int kDmmaChunkDoubles = 3 * 4 * 32;                // B operands of one step: [channel][k-step][lane]
static_assert(kDmmaRecurrences == 3 * kBulkTones * kDmmaSegments * 2, "(channel, tone, segment, Gauss point)");

struct __align__(16) DmmaShared {
    double table[2][kDmmaPhase][kDmmaChunkDoubles];
    double2 z[kDmmaRecurrences];  // exp(i w tau) of each recurrence at its next step
    double2 rot[3 * kBulkTones];  // exp(i w dt)
    double2 half_step[3 * kBulkTones];  // exp(i w dt_out / 2)
    int32_t tile;
    int32_t magnus;                     // 1: the tile takes the one-exponential Magnus step
};

// d[0..1] += a b over the 8 x 8 x 4 product of the warp (FP64 tensor path).
SS_D void dmma_m8n8k4(double& d0, double& d1, double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
        : "+d"(d0), "+d"(d1)
        : "d"(a), "d"(b));
}

// b a in FP64 residual form (b later): alpha - 1 = a.am1 + b.am1 + b.am1 a.am1 - conj(b.beta) a.beta,
// beta = b.beta + a.beta + b.beta a.am1 + conj(b.am1) a.beta.
SS_D Su2d su2d_mul(const Su2d& b, const Su2d& a) {
    Su2d o;
    o.am1 = cfma(b.am1, a.am1, a.am1 + b.am1) - conj(b.beta) * a.beta;
    o.beta = cfma(b.beta, a.am1, b.beta + a.beta) + conj(b.am1) * a.beta;
    return o;
}

SS_D Su2d shfl_down_su2(const Su2d& v, int delta) {
    Su2d o;
    o.am1.re = __shfl_down_sync(0xffffffffu, v.am1.re, delta);
    o.am1.im = __shfl_down_sync(0xffffffffu, v.am1.im, delta);
    o.beta.re = __shfl_down_sync(0xffffffffu, v.beta.re, delta);
    o.beta.im = __shfl_down_sync(0xffffffffu, v.beta.im, delta);
    return o;
}

static_assert(kDmmaTile == kScanTile, "a CTA tile is one state scan tile (its warps' row products are its partials)");

// Recurrence r = ((channel * kBulkTones + tone) * kDmmaSegments + segment) * 2 + Gauss point of an
// instance with K fine steps of dt: its start phasor exp(i w tau), tau = (segment start) dt + a_lo or
// a_hi (the reference's sample offsets, I:644-647), and its tone's step rotation exp(i w dt).
SS_D void dmma_recurrence(const FieldDesc& f, int K, double dt, int r, double2* z, double2* rot) {
    const int gauss = r & 1, seg = (r >> 1) & (kDmmaSegments - 1), slot = r >> 3;
    const int c = slot / kBulkTones, tone = slot % kBulkTones;
    *z = make_double2(0.0, 0.0);
    *rot = make_double2(1.0, 0.0);
    if (tone < f.tone_count[c]) {
        const double a = 0.5 * dt * (gauss ? 1.0 + 1.0 / kSqrt3 : 1.0 - 1.0 / kSqrt3);
        const double w = __ldg(f.tones + 3 * (f.tone_start[c] + tone));
        const int start = (int)(((int64_t)K * seg) / kDmmaSegments);
        double sn, cs;
        sincos(w * fma((double)start, dt, a), &sn, &cs);
        *z = make_double2(cs, sn);
        sincos(w * dt, &sn, &cs);
        *rot = make_double2(cs, sn);
    }
}

// exp(i w dt_out / 2) of tone slot (1 for an absent tone).
SS_D double2 dmma_half_step(const FieldDesc& f, int slot, double dt_out) {
    const int c = slot / kBulkTones, tone = slot % kBulkTones;
    if (tone >= f.tone_count[c]) return make_double2(1.0, 0.0);
    double sn, cs;
    sincos(0.5 * __ldg(f.tones + 3 * (f.tone_start[c] + tone)) * dt_out, &sn, &cs);
    return make_double2(cs, sn);
}

// 1 when the instance takes the Magnus step: theta = dt (|B|max + w_max) <= kMagnusTheta, |B|max from
// the channels' biases and amplitudes summed in a fixed order (every launch takes the same branch).
SS_D int32_t dmma_magnus(const FieldDesc& f, double dt) {
    double bsq = 0.0, wmax = 0.0;
    for (int c = 0; c < 3; c++) {
        double bc = fabs(f.bias[c]);
        for (int k = 0; k < f.tone_count[c] && k < kBulkTones; k++) {
            const double* tn = f.tones + 3 * (f.tone_start[c] + k);
            bc += fabs(f.gain[c] * __ldg(tn + 1));
            wmax = fmax(wmax, fabs(__ldg(tn)));
        }
        bsq = fma(bc, bc, bsq);
    }
    return dt * (sqrt(bsq) + wmax) <= kMagnusTheta ? 1 : 0;
}

#ifdef SPINSIM_DMMA_CONSTS_KERNEL
// The per-instance constants of the tensor path (DmmaConsts), one CTA of kDmmaRecurrences threads
// per instance, launched before the time evolution so its tiles load them instead of recomputing
// them (384 FP64 sincos and the step test per tile).
__global__ void __launch_bounds__(kDmmaRecurrences) dmma_consts_kernel(EvolveArgs a, DmmaConsts* out, int32_t n) {
    grid_dependency_release();  // the time evolution may start its tiles' set-up meanwhile
    const int32_t i = blockIdx.x;
    if (i >= n) return;
    const Instance& inst = a.instances[i];
    const FieldDesc& f = a.fields[inst.field];
    if (!tones_on_tensor_path(f, inst.dim)) return;
    DmmaConsts& c = out[i];
    const int r = threadIdx.x;
    double2 z, rot;
    dmma_recurrence(f, inst.n_fine, inst.dt_int, r, &z, &rot);
    c.z[r] = z;
    if ((r & 7) == 0) c.rot[r >> 3] = rot;
    if (r < kToneSlots) c.half_step[r] = dmma_half_step(f, r, inst.dt_out);
    if (r == 0) c.magnus = dmma_magnus(f, inst.dt_int);
}
#endif


// The interval's lab-frame operator from its SU(2) pair: itself (spin half) or its representation.
template <int D>
SS_D void store_interval_operator(const Su2p& v, double* u_out, int64_t idx) {
    const Mat<D> u = su2p_to_mat<D>(v);
    double2* dst = reinterpret_cast<double2*>(u_out) + idx * (D * D);
#pragma unroll
    for (int r = 0; r < D; r++)
#pragma unroll
        for (int k = 0; k < D; k++) dst[r * D + k] = make_double2(u.a[r][k].re, u.a[r][k].im);
}

// partial_out (may be null): the tile's scan partials, where this warp writes the lab-frame SU(2) pair of
// its rows' product (later rows from the left; rows past the tile's end are the identity).  cst (may be
// null): the instance's constants from dmma_consts_kernel; without them the tile computes them.  The
// spin dimension enters only the frame winding and the stored operator, so a mixed-spin launch
// (DIMS 0) runs one copy of the step loop for both spins.
template <int DIMS>
SS_D void tile_dmma(const MethodConfig& m, const Instance& inst, const FieldDesc& f, const Tile& tile, DmmaShared& sh,
                    double* time_out, double* u_out, float* norms_out, double* partial_out, const DmmaConsts* cst,
                    double* rows_out) {
    const int D = DIMS != 0 ? DIMS : inst.dim;
    const int P = (D == 2) ? 2 : 1;  // power of the frame winding in the xy transform (I:599-613)
    const int lane = threadIdx.x & 31;
    const int g = lane >> 2, q = lane & 3;
    const int row = (threadIdx.x >> 5) * kDmmaRows + g;
    const bool active = row < tile.count;
    const int64_t idx = tile.first + (active ? row : 0);
    const double dt = inst.dt_int, dt_out = inst.dt_out;
    const int K = inst.n_fine;
    const int seg_start = (int)(((int64_t)K * q) / kDmmaSegments);
    const int seg_len = (int)(((int64_t)K * (q + 1)) / kDmmaSegments) - seg_start;
    const int n_steps = (K + kDmmaSegments - 1) / kDmmaSegments;  // steps of the longest segment
    const double a_lo = 0.5 * dt * (1.0 - 1.0 / kSqrt3);
    const double a_hi = 0.5 * dt * (1.0 + 1.0 / kSqrt3);
    const double half_dt = 0.5 * dt;
    const double t_c = __dadd_rn(inst.t0, __dmul_rn(dt_out, (double)(inst.interval0 + idx)));  // I:818, unfused

    // Producer recurrences (dmma_recurrence), their rotations and the step choice: the instance's
    // constants, or computed here.
    if (cst != nullptr) {
        grid_dependency_wait();  // the constants' kernel may still be running (it lets this launch start early)
        for (int r = threadIdx.x; r < kDmmaRecurrences; r += kDmmaThreads) sh.z[r] = cst->z[r];
        if (threadIdx.x < kToneSlots) sh.rot[threadIdx.x] = cst->rot[threadIdx.x];
        if (threadIdx.x == 0) sh.magnus = cst->magnus;
    } else {
        for (int r = threadIdx.x; r < kDmmaRecurrences; r += kDmmaThreads) {
            double2 z, rot;
            dmma_recurrence(f, K, dt, r, &z, &rot);
            sh.z[r] = z;
            if ((r & 7) == 0) sh.rot[r >> 3] = rot;
        }
        if (threadIdx.x == 0) sh.magnus = dmma_magnus(f, dt);
    }

    // L of every tone and interval of the tile (buffer 1 of the table holds it until the first refill):
    // thread 4 slot + quarter evaluates interval 8 quarter once and steps to the next seven intervals
    // with exp(i w dt_out); h = exp(i w dt_out / 2) per tone is kept for the frame's mid-interval sample.
    double2* lval = reinterpret_cast<double2*>(&sh.table[1][0][0]);  // [slot][interval of the tile]
    static_assert(sizeof(sh.table[1]) >= sizeof(double2) * kToneSlots * kDmmaTile, "L table fits one buffer");
    if (threadIdx.x < 4 * kToneSlots) {
        const int slot = threadIdx.x >> 2, quarter = threadIdx.x & 3;
        const int c = slot / kBulkTones, tone = slot % kBulkTones;
        c64 l = c64{0.0, 0.0}, gstep = c64{1.0, 0.0}, h = c64{1.0, 0.0};
        if (tone < f.tone_count[c]) {
            const double* tn = f.tones + 3 * (f.tone_start[c] + tone);
            const double w = __ldg(tn), amp = f.gain[c] * __ldg(tn + 1);
            const int64_t i0 = inst.interval0 + tile.first + kDmmaRows * quarter;
            const double tq = __dadd_rn(inst.t0, __dmul_rn(dt_out, (double)i0));  // as the intervals' own t_c
            double sn, cs;
            sincos(fma(w, tq, __ldg(tn + 2)), &sn, &cs);
            l = c64{half_dt * amp * cs, half_dt * amp * sn};
            const double2 hs = cst != nullptr ? cst->half_step[slot] : dmma_half_step(f, slot, dt_out);
            h = c64{hs.x, hs.y};
            gstep = h * h;
        }
        if (quarter == 0) sh.half_step[slot] = make_double2(h.re, h.im);
#pragma unroll
        for (int r = 0; r < kDmmaRows; r++) {
            lval[slot * kDmmaTile + kDmmaRows * quarter + r] = make_double2(l.re, l.im);
            l = l * gstep;
        }
    }
    __syncthreads();  // producer phasors, rotations, step choice and L in place

    // A operands: L of this lane's interval for tone 2 s + q / 2 (Re L for even q, Im L for odd q)
    double afr[3][4];
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
        for (int s = 0; s < 4; s++) {
            const double* lv = reinterpret_cast<const double*>(&lval[(c * kBulkTones + 2 * s + (q >> 1)) * kDmmaTile + row]);
            afr[c][s] = active ? lv[q & 1] : 0.0;
        }
    // Rotating frame (I:823-829): Bz at the middle of the interval, sum_k Im(L_zk h_k) + bias;
    // lane q sums tones 2 q, 2 q + 1 and the quad adds the four parts.
    double rw = 0.0;
    if (m.rotating) {
        double part = 0.0;
#pragma unroll
        for (int k = 2 * q; k < 2 * q + 2; k++) {
            const double2 lz = lval[(2 * kBulkTones + k) * kDmmaTile + row];
            const double2 hk = sh.half_step[2 * kBulkTones + k];
            part += fma(lz.x, hk.y, lz.y * hk.x);
        }
        part += __shfl_xor_sync(0xffffffffu, part, 1);
        part += __shfl_xor_sync(0xffffffffu, part, 2);
        rw = f.bias[2] + part / half_dt;
        if (D == 2) rw /= 2;
    }
    const double prw = (double)P * rw;
    const double hprw = half_dt * prw;
    // (h / 2) bias, the starting value of the samples' accumulation; in the rotating frame z also
    // carries the frame's -P rw (I:582-618), added once here instead of to every sample
    double bias[3];
#pragma unroll
    for (int c = 0; c < 3; c++) bias[c] = half_dt * f.bias[c];
    bias[2] -= hprw;
    // Frame phasors at the Gauss points of this segment's steps: exp(-i P rw (tau - 0)), tau as above
    c64 wa = c64{1.0, 0.0}, wb = c64{1.0, 0.0}, wrot = c64{1.0, 0.0};
    if (m.rotating) {
        sincos_small(-prw * dt, &wrot.im, &wrot.re);
        sincos_small(-prw * fma((double)seg_start, dt, a_lo), &wa.im, &wa.re);
        sincos_small(-prw * fma((double)seg_start, dt, a_hi), &wb.im, &wb.re);
    }

    // Fill table buffer (ph & 1) with the B operands of steps [ph kDmmaPhase, ...) of every segment.
    auto fill = [&](int ph) {
        const int m0 = ph * kDmmaPhase;
        const int mc = min(kDmmaPhase, n_steps - m0);
        for (int r = threadIdx.x; r < kDmmaRecurrences; r += kDmmaThreads) {
            const int gauss = r & 1, seg = (r >> 1) & (kDmmaSegments - 1), slot = r >> 3;
            const int c = slot / kBulkTones, tone = slot % kBulkTones;
            // consumer lane 4 g' + q' with g' = 2 segment + Gauss point, q' = 2 (tone & 1) + (0 sin, 1 cos)
            double* dst = &sh.table[ph & 1][0][(c * 4 + (tone >> 1)) * 32 + 4 * (2 * seg + gauss) + 2 * (tone & 1)];
            double2 z = sh.z[r];
            const double2 rt = sh.rot[slot];
            for (int mm = 0; mm < mc; mm++) {
                *reinterpret_cast<double2*>(dst + mm * kDmmaChunkDoubles) = make_double2(z.y, z.x);
                z = make_double2(fma(z.x, rt.x, -z.y * rt.y), fma(z.x, rt.y, z.y * rt.x));
            }
            sh.z[r] = z;
        }
    };

    fill(0);  // buffer 0; buffer 1 (the L table) is first refilled after the barrier below
    __syncthreads();
    const bool magnus = sh.magnus != 0;
    // CF4 generators from samples in units of h / 2: h (w0 b1 + w1 b2) = 2 w0 sa + 2 w1 sb
    constexpr double kW0 = (1.5 + kSqrt3) / 3.0, kW1 = (1.5 - kSqrt3) / 3.0;
    Su2d acc = Su2d{c64{0.0, 0.0}, c64{0.0, 0.0}};
    float nsq = 0.0f;  // sum of |g|^2 over this lane's steps (the error statement's scale)
    const int n_phases = (n_steps + kDmmaPhase - 1) / kDmmaPhase;
    for (int ph = 0; ph < n_phases; ph++) {
        if (ph + 1 < n_phases) fill(ph + 1);
        const int m0 = ph * kDmmaPhase;
        const int mc = min(kDmmaPhase, n_steps - m0);
        const double* tb = &sh.table[ph & 1][0][lane];
        // The samples of step mm + 1 (tensor path) are issued at the end of step mm, so they are in flight
        // while the next step begins.
        double na[3], nb[3];
        auto samples = [&](int mm, double* xa, double* xb) {
#pragma unroll
            for (int c = 0; c < 3; c++) {
                double d0 = bias[c], d1 = bias[c];
#pragma unroll
                for (int s = 0; s < 4; s++) dmma_m8n8k4(d0, d1, afr[c][s], tb[mm * kDmmaChunkDoubles + (c * 4 + s) * 32]);
                xa[c] = d0;
                xb[c] = d1;
            }
        };
        samples(0, na, nb);
        for (int mm = 0; mm < mc; mm++) {
            double sa[3], sb[3];
#pragma unroll
            for (int c = 0; c < 3; c++) {
                sa[c] = na[c];
                sb[c] = nb[c];
            }
            if (active && m0 + mm < seg_len) {
                if (m.rotating) {  // xy times exp(-i P rw tau) (I:582-618), in units of h / 2 (z: in the bias)
                    const c64 xa = c64{sa[0], sa[1]} * wa;
                    const c64 xb = c64{sb[0], sb[1]} * wb;
                    sa[0] = xa.re;
                    sa[1] = xa.im;
                    sb[0] = xb.re;
                    sb[1] = xb.im;
                    wa = wa * wrot;
                    wb = wb * wrot;
                }
                if (magnus) {
                    // g = (h / 2)(b1 + b2) + (sqrt3 h^2 / 12) b2 x b1, with (h / 2) b in sa, sb: the
                    // linear part g_lin = sa + sb stays FP64; the commutator (sqrt3 / 6) d x g_lin,
                    // d = (h / 2)(b2 - b1), and the exponential's remainder are FP32.
                    double gl64[3];
                    float gl[3], dd[3];
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        gl64[c] = sa[c] + sb[c];
                        gl[c] = __double2float_rn(gl64[c]);
                        dd[c] = __double2float_rn(sb[c] - sa[c]);
                    }
                    constexpr float kComm = 0.28867513459481287f;  // sqrt3 / 6
                    const float cx = kComm * fmaf(dd[1], gl[2], -dd[2] * gl[1]);
                    const float cy = kComm * fmaf(dd[2], gl[0], -dd[0] * gl[2]);
                    const float cz = kComm * fmaf(dd[0], gl[1], -dd[1] * gl[0]);
                    Su2f rest = su2_exp_rest(gl[0] + cx, gl[1] + cy, gl[2] + cz);
                    rest.am1.im = fmaf(-0.5f, cz, rest.am1.im);  // the commutator's linear part
                    rest.beta.re = fmaf(0.5f, cy, rest.beta.re);
                    rest.beta.im = fmaf(-0.5f, cx, rest.beta.im);
                    nsq = fmaf(gl[0], gl[0], fmaf(gl[1], gl[1], fmaf(gl[2], gl[2], nsq)));
                    su2_apply_split(acc, gl64[0], gl64[1], gl64[2], rest);
                } else {  // the reference's CF4 (I:655-686): two exponentials
                    double ga[3], gb[3];
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        ga[c] = fma(kW0, sa[c], kW1 * sb[c]);
                        gb[c] = fma(kW1, sa[c], kW0 * sb[c]);
                    }
                    su2_cf4_step(acc, ga, gb, &nsq);
                }
            }
            // the next step's samples, issued after this step's arithmetic (all lanes: mma.sync is
            // warp-collective); measured 0.7% faster than issuing them before it
            if (mm + 1 < mc) samples(mm + 1, na, nb);
        }
        __syncthreads();  // buffer (ph & 1) is refilled in phase ph + 1
    }

    // The interval's product: segment 3 ... segment 0 (later segments from the left)
#pragma unroll
    for (int sft = 1; sft < kDmmaSegments; sft <<= 1) {
        const Su2d later = shfl_down_su2(acc, sft);
        nsq += __shfl_down_sync(0xffffffffu, nsq, sft);
        if ((q & (2 * sft - 1)) == 0) acc = su2d_mul(later, acc);
    }
    // The interval's lab-frame operator as an SU(2) pair: leaving the frame (I:839-852) multiplies by
    // the SU(2) element diag(exp(-i phi), exp(i phi)), phi = rw dt_out (spin half, rw halved above) or
    // rw dt_out / 2 (spin one, whose representation doubles the phase).  Rows past the tile's end and
    // the other lanes of a quad hold the identity.
    Su2p v = su2p_identity();
    if (active && q == 0) {
        v.a = c64{1.0 + acc.am1.re, acc.am1.im};
        v.b = acc.beta;
        if (m.rotating) {
            c64 wh;
            sincos_small(rw * dt_out * (D == 2 ? 1.0 : 0.5), &wh.im, &wh.re);
            v.a = v.a * conj(wh);
            v.b = v.b * wh;
        }
        time_out[idx] = t_c;
        if (norms_out != nullptr) norms_out[idx] = nsq;
        if (D == 2) store_interval_operator<2>(v, u_out, idx);
        else store_interval_operator<3>(v, u_out, idx);
        if (rows_out != nullptr) {  // the same operator as its SU(2) pair, for the state scan
            double2* r = reinterpret_cast<double2*>(rows_out) + 2 * idx;
            r[0] = make_double2(v.a.re, v.a.im);
            r[1] = make_double2(v.b.re, v.b.im);
        }
    }
    if (partial_out != nullptr) {  // the warp's product of its rows (lanes 4 g), later rows from the left
#pragma unroll
        for (int sft = kDmmaSegments; sft < 32; sft <<= 1) {
            const Su2p later = shfl_down_su2p(v, sft);
            if ((lane & (2 * sft - 1)) == 0) v = su2p_mul(later, v);
        }
        if (lane == 0) {
            double2* dst = reinterpret_cast<double2*>(partial_out) + 2 * (threadIdx.x >> 5);
            dst[0] = make_double2(v.a.re, v.a.im);
            dst[1] = make_double2(v.b.re, v.b.im);
        }
    }
}

// More tones than the products take, or a quadratic shift: one interval per thread (not inlined, so its
// registers do not weigh on the tensor path's step loop).
template <int DIMS>
__device__ __noinline__ void dmma_tile_fallback(const MethodConfig& m, const Instance& inst, const FieldDesc& f,
                                                int64_t interval, int dim, double* time_out, double* u_out,
                                                float* norms_out) {
    if (DIMS != 3 && dim == 2)
        interval32<2, INTEG_CF4, EXPO_ANALYTIC, FIELD_TONES>(m, inst, f, interval, true, 0, time_out, u_out, norms_out);
    else if (DIMS != 2)
        interval32<3, INTEG_CF4, EXPO_LIE_TROTTER, FIELD_TONES>(m, inst, f, interval, true, 0, time_out, u_out, norms_out);
}

// Persistent launch: CTAs pull tiles of kDmmaTile intervals from the queue (or, without a queue, CTA
// b takes tile b of a single instance).
template <int DIMS>
SS_D void evolve_dmma_body(const EvolveArgs& a, DmmaShared& sh) {
    int64_t tile_id = blockIdx.x;
    int32_t reserved = -1;  // thread 0: the next tile, taken from the queue while this one runs
    for (;;) {
        if (a.tile_counter != nullptr) {
            if (threadIdx.x == 0) sh.tile = reserved >= 0 ? reserved : atomicAdd(a.tile_counter, 1);
            __syncthreads();
            tile_id = sh.tile;
            // Away from the end of the queue, take the next tile now (its atomic's latency then passes
            // during this tile); near the end tiles are taken only when a CTA is free, so no CTA holds
            // a tile that another could have run.
            if (threadIdx.x == 0)
                reserved = tile_id + 2 * (int64_t)gridDim.x < a.n_tiles ? atomicAdd(a.tile_counter, 1) : -1;
        }
        if (tile_id >= a.n_tiles) {
            grid_dependency_release();  // no tiles left for this CTA: the scan may start launching
            return;
        }
        Tile tile;
        if (a.tiles != nullptr) {
            tile = a.tiles[tile_id];
        } else {
            const int64_t n = a.instances[0].n_out;
            tile.instance = 0;
            tile.first = tile_id * kDmmaTile;
            tile.count = (int)((n - tile.first) < kDmmaTile ? (n - tile.first) : kDmmaTile);
        }
        const Instance& inst = a.instances[tile.instance];
        const FieldDesc& f = a.fields[inst.field];
        double* time_out = a.time + inst.out_offset;
        double* u_out = a.u + inst.u_offset;
        float* norms_out = a.step_norms != nullptr ? a.step_norms + inst.out_offset : nullptr;
        const int dim = (DIMS == 0) ? inst.dim : DIMS;
        if (tones_on_tensor_path(f, dim)) {
            double* partial_out = nullptr;
            if (a.tile_partials != nullptr) {
                const int64_t k = (a.scan_begin != nullptr ? a.scan_begin[tile.instance] : 0) + tile.first / kScanTile;
                partial_out = a.tile_partials + k * kScanMat;
            }
            const DmmaConsts* cst = a.dmma_consts != nullptr ? a.dmma_consts + tile.instance : nullptr;
            double* rows_out = a.rows != nullptr ? a.rows + 4 * inst.out_offset : nullptr;
            tile_dmma<DIMS>(a.m, inst, f, tile, sh, time_out, u_out, norms_out, partial_out, cst, rows_out);
        } else if (threadIdx.x < tile.count) {
            dmma_tile_fallback<DIMS>(a.m, inst, f, tile.first + threadIdx.x, dim, time_out, u_out, norms_out);
        }
        __syncthreads();  // shared memory and the tile slot are reused by the next tile
        if (a.tile_counter == nullptr) return;
    }
}

// MINB: minimum resident CTAs per SM for the register allocation (6: 80 registers, 5: 96, 4: 128, 3: 168).
template <int DIMS, int MINB>
__global__ void __launch_bounds__(kDmmaThreads, MINB) evolve_dmma_kernel(EvolveArgs a) {
    __shared__ DmmaShared sh;
    evolve_dmma_body<DIMS>(a, sh);
}

}  // namespace spinsim
