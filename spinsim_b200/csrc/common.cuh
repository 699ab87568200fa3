// Shared device/host definitions for the spinsim sm_100a kernels.
//
// Layouts in HBM (the same as the reference's numpy outputs, spinsim/__init__.py:1040-1041, :1081):
//   time[N]             float64
//   U[N][d][d]          complex128, row-major per output interval (interleaved re, im)
//   state[N][d]         complex128
//   spin[N][3]          float64
// A batch stores its instances back to back in the same flat arrays; every instance carries the
// offsets of its first output interval.
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define SS_HD __host__ __device__ __forceinline__
#define SS_D __device__ __forceinline__
#else
#define SS_HD inline
#define SS_D inline
#endif

namespace spinsim {

// ------------------------------------------------------------------ method enumerations
// Values follow the reference's enums (IntegrationMethod I:68-93, ExponentiationMethod.index I:95-129).
enum Integration : int { INTEG_CF4 = 0, INTEG_EULER = 1, INTEG_HEUN = 2 };
enum Exponentiation : int { EXPO_ANALYTIC = 0, EXPO_LIE_TROTTER = 1, EXPO_LIE_TROTTER_8 = 2 };
enum FieldKind : int { FIELD_USER = 0, FIELD_TABLE = 1, FIELD_TONES = 2 };
enum Precision : int { PREC_FP64 = 0, PREC_FP32_BULK = 1 };

constexpr int kMaxChannels = 8;  // x, y, z, q, u1, u2, v1, v2 (reference docs I:381-389)
constexpr int kEvolveThreadsDefault = 128;  // time-evolution CTA size unless the plan asks otherwise
constexpr int kEvolveThreadsMax = 128;      // __launch_bounds__ of the time-evolution kernels

// ------------------------------------------------------------------ field descriptors
// One interpolation table (the reference's generate_interpolation_sampler, I:1941-2147).
struct TableChannel {
    const double* time;       // [size], non-decreasing
    const double* amplitude;  // [size]
    int64_t size;             // 0 = no table on this channel
    int32_t order;            // 0 zero-order hold, 1 linear, 3 cubic Hermite
    int32_t zero_boundary;    // 1: zero outside [time[0], time[size-1]]; 0: hold the end values
};

// Per-instance field.  channel c = bias[c] + gain[c] * source_c(t), where source_c is the
// channel's table (FIELD_TABLE) or its tone sum sum_k A_k sin(w_k t + phi_k) (FIELD_TONES).
// FIELD_USER ignores everything but params/n_params, which go to the linked get_field().
struct FieldDesc {
    const double* params;          // sweep parameters for a user get_field (device)
    int64_t n_params;
    const TableChannel* tables;    // [kMaxChannels] (FIELD_TABLE)
    const double* tones;           // FIELD_TONES: (w, A, phi) triples, channel after channel
    int32_t tone_start[kMaxChannels];
    int32_t tone_count[kMaxChannels];
    double bias[kMaxChannels];
    double gain[kMaxChannels];
};

// ------------------------------------------------------------------ work description
// One simulated instance (one evaluate() call of the reference).
struct Instance {
    double t0;            // time_start
    double dt_int;        // normalised integration step (I:1025-1026)
    double dt_out;        // time_step_output
    int64_t n_out;        // N = int((t1 - t0) / dt_out)  (I:1034)
    int64_t out_offset;   // first output interval of this instance in time[] and spin[]
    int64_t u_offset;     // first double of this instance in U[] (out_offset * 2 d^2 when all d agree)
    int64_t state_offset; // first double of this instance in state[]
    int32_t n_fine;       // K = floor(dt_out / dt_int + 0.5)  (I:832)
    int32_t dim;          // 2 or 3
    int32_t field;        // index into the FieldDesc array
    int32_t interval0;    // time index of output interval 0: time[i] = t0 + dt_out * (interval0 + i)
    double psi0[6];       // initial state, complex[dim] interleaved
};

// A tile is a warp's unit of work: up to 32 / lanes consecutive output intervals of one instance.
struct Tile {
    int32_t instance;
    int32_t count;      // intervals in this tile
    int64_t first;      // first output interval (relative to the instance)
};

// Static configuration of one time-evolution launch (identical for every instance in it).
struct MethodConfig {
    int32_t integration;    // Integration
    int32_t expo_half;      // Exponentiation used for dim 2 instances
    int32_t expo_one;       // Exponentiation used for dim 3 instances
    int32_t rotating;       // use_rotating_frame
    int32_t hypercubes;     // ceil(number_of_squares / 2), >= 0  (I:1547-1549)
    int32_t lanes;          // lanes sharing one output interval (1, 2, 4, 8, 16, 32)
    double precision;       // 4 ** hypercubes  (I:1550)
};

// Launch arguments of the time-evolution kernels.
struct EvolveArgs {
    MethodConfig m;
    const Instance* instances;
    const FieldDesc* fields;
    const Tile* tiles;       // null: single instance, implicit tiles of 32 / lanes intervals (a CTA's 32 on the tensor path)
    int64_t n_tiles;
    int32_t* tile_counter;   // null: one tile per warp (per CTA on the tensor path) of the grid, no queue
    double* time;            // [sum N]
    double* u;               // complex [sum N * d * d]; instance i starts at u_offset doubles
    float* step_norms;       // FP32-bulk: per output step, the sum over its fine steps of |g|^2 (the squared
                             // norms of the generators rounded to FP32); null: not written
    double* tile_partials;   // tensor path: per scan tile (kScanTile output steps, kScanMat doubles), each
                             // warp's product of its rows as an SU(2) pair in the lab frame (4 doubles per
                             // warp, warp after warp); null: not written
    const int32_t* scan_begin;  // per instance: its first scan tile (null: one instance, tile 0)
    const struct DmmaConsts* dmma_consts;  // tensor path: per instance, written by dmma_consts_kernel
                                           // earlier in the launch (null: each tile computes them)
    double* rows;  // tensor path: per output step (indexed like time), the interval's lab-frame operator
                   // as its SU(2) pair (a, b), 4 doubles, for the state scan (null: not written)
};

// State scan tiles (scan.cuh): consecutive output steps of one instance per tile, and the doubles
// kept per stored tile operator (3 x 3 complex; spin half uses 8).
constexpr int kScanTile = 32;
constexpr int kScanMat = 18;

// ------------------------------------------------------------------ FP32-bulk tone synthesis
// Shared memory of the FP32-bulk tone kernels (see evolve32.cuh), per warp.
constexpr int kBulkTones = 8;               // tones per channel (x, y, z) synthesised per warp
constexpr int kToneSlots = 3 * kBulkTones;  // slot = channel * kBulkTones + tone

// Per-instance constants of the tensor-path kernel (evolve_dmma.cuh), the same for all of an
// instance's tiles: the phasor table's start values exp(i w tau) of every (channel, tone, time
// segment, Gauss point), each tone's step rotation exp(i w dt) and half-interval phasor
// exp(i w dt_out / 2), and the choice of step (1: Magnus).
constexpr int kDmmaRecurrences = 3 * kBulkTones * 4 * 2;
struct __align__(16) DmmaConsts {
    double2 z[kDmmaRecurrences];
    double2 rot[kToneSlots];
    double2 half_step[kToneSlots];
    int32_t magnus;
    int32_t pad[3];
};

// A tone field whose samples the tensor-path kernel forms as products: at most kBulkTones tones per
// channel and, for spin one, no quadratic shift (other fields take that kernel's per-interval path).
SS_HD bool tones_on_tensor_path(const FieldDesc& f, int dim) {
    for (int c = 0; c < 3; c++)
        if (f.tone_count[c] > kBulkTones) return false;
    return !(dim == 3 && (f.bias[3] != 0.0 || f.tone_count[3] > 0));
}
constexpr int kSynthIntervals = 2;          // output intervals per lane, 32 intervals apart
// Slot-fastest layouts: a warp's 16-byte stores and loads of one quantity for all slots are
// contiguous (no bank conflicts); the consumers' reads of one slot are broadcasts.
struct ToneShared {
    double l[kToneSlots][32][2];                 // [slot][lane] (re, im) of L for the lane's first interval
    double2 uv[2][kSynthIntervals][2][kToneSlots];  // [buffer][interval][U or V][slot] G^i U, G^i V of the step
};
constexpr int kToneSharedBytes = kToneSlots * 32 * 2 * 8 + 2 * kToneSlots * kSynthIntervals * 4 * 8;
// FP32-bulk tone kernel with the field samples on the FP64 tensor path (see evolve_dmma.cuh): a CTA
// of kDmmaWarps warps takes a tile of kDmmaTile consecutive output intervals of one instance.
constexpr int kDmmaWarps = 4;
constexpr int kDmmaThreads = 32 * kDmmaWarps;
constexpr int kDmmaRows = 8;                       // output intervals per warp (rows of m8n8k4)
constexpr int kDmmaTile = kDmmaWarps * kDmmaRows;  // output intervals per CTA tile

// ------------------------------------------------------------------ complex helpers (FP64)
struct c64 {
    double re, im;
};
SS_HD c64 mk(double r, double i) { return c64{r, i}; }
SS_HD c64 operator+(c64 a, c64 b) { return c64{a.re + b.re, a.im + b.im}; }
SS_HD c64 operator-(c64 a, c64 b) { return c64{a.re - b.re, a.im - b.im}; }
SS_HD c64 operator*(c64 a, c64 b) { return c64{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
SS_HD c64 operator*(double s, c64 a) { return c64{s * a.re, s * a.im}; }
SS_HD c64 conj(c64 a) { return c64{a.re, -a.im}; }
// a * b + c
SS_HD c64 cfma(c64 a, c64 b, c64 c) {
#ifdef __CUDA_ARCH__
    return c64{fma(a.re, b.re, fma(-a.im, b.im, c.re)), fma(a.re, b.im, fma(a.im, b.re, c.im))};
#else
    return c64{a.re * b.re - a.im * b.im + c.re, a.re * b.im + a.im * b.re + c.im};
#endif
}

template <int D>
struct Mat {
    c64 a[D][D];
};

template <int D>
SS_HD void set_identity(Mat<D>& m) {
#pragma unroll
    for (int i = 0; i < D; i++)
#pragma unroll
        for (int j = 0; j < D; j++) m.a[i][j] = c64{i == j ? 1.0 : 0.0, 0.0};
}

// matrix_multiply (I:1594-1600, I:1722-1734): out = l r
template <int D>
SS_HD Mat<D> matmul(const Mat<D>& l, const Mat<D>& r) {
    Mat<D> o;
#pragma unroll
    for (int i = 0; i < D; i++)
#pragma unroll
        for (int j = 0; j < D; j++) {
            c64 acc = l.a[i][0] * r.a[0][j];
#pragma unroll
            for (int k = 1; k < D; k++) acc = cfma(l.a[i][k], r.a[k][j], acc);
            o.a[i][j] = acc;
        }
    return o;
}

// matrix_square_m1 (I:1602-1608, I:1736-1748): (2 + A) A, the k == i term grouped as (2 + A_ii) A_ij
template <int D>
SS_HD Mat<D> square_m1(const Mat<D>& m) {
    Mat<D> o;
#pragma unroll
    for (int i = 0; i < D; i++)
#pragma unroll
        for (int j = 0; j < D; j++) {
            c64 acc = c64{0.0, 0.0};
#pragma unroll
            for (int k = 0; k < D; k++) {
                if (k == i) {
                    c64 two_plus = c64{2.0 + m.a[i][i].re, m.a[i][i].im};
                    acc = (k == 0) ? two_plus * m.a[i][j] : cfma(two_plus, m.a[i][j], acc);
                } else {
                    acc = (k == 0) ? m.a[i][k] * m.a[k][j] : cfma(m.a[i][k], m.a[k][j], acc);
                }
            }
            o.a[i][j] = acc;
        }
    return o;
}

// matrix_multiply_m1 (I:1610-1616, I:1750-1762): (l + r) + l r
template <int D>
SS_HD Mat<D> multiply_m1(const Mat<D>& l, const Mat<D>& r) {
    Mat<D> o;
#pragma unroll
    for (int i = 0; i < D; i++)
#pragma unroll
        for (int j = 0; j < D; j++) {
            c64 acc = l.a[i][0] * r.a[0][j];
#pragma unroll
            for (int k = 1; k < D; k++) acc = cfma(l.a[i][k], r.a[k][j], acc);
            o.a[i][j] = (l.a[i][j] + r.a[i][j]) + acc;
        }
    return o;
}

// An SU(2) element as its pair (a, b): U = [[a, -conj b], [b, conj a]].
struct Su2p {
    c64 a, b;
};

SS_D Su2p su2p_identity() { return Su2p{c64{1.0, 0.0}, c64{0.0, 0.0}}; }

// x y (x later)
SS_D Su2p su2p_mul(const Su2p& x, const Su2p& y) {
    return Su2p{x.a * y.a - conj(x.b) * y.b, cfma(x.b, y.a, conj(x.a) * y.b)};
}

// Spin-one representation of an SU(2) element (the image of U under the spin-one map).
SS_D Mat<3> su2_to_spin_one(const c64& alpha, const c64& beta) {
    constexpr double r2 = 1.4142135623730951;
    Mat<3> m;
    const c64 ac = conj(alpha), bc = conj(beta);
    m.a[0][0] = alpha * alpha;
    m.a[1][0] = r2 * (alpha * beta);
    m.a[2][0] = beta * beta;
    m.a[0][1] = (-r2) * (alpha * bc);
    m.a[1][1] = c64{alpha.re * alpha.re + alpha.im * alpha.im - beta.re * beta.re - beta.im * beta.im, 0.0};
    m.a[2][1] = r2 * (ac * beta);
    m.a[0][2] = bc * bc;
    m.a[1][2] = (-r2) * (ac * bc);
    m.a[2][2] = ac * ac;
    return m;
}

// The d x d operator of an SU(2) element: itself (spin half) or its spin-one representation.
template <int D>
SS_D Mat<D> su2p_to_mat(const Su2p& v) {
    if constexpr (D == 2) {
        Mat<2> m;
        m.a[0][0] = v.a;
        m.a[1][0] = v.b;
        m.a[0][1] = c64{-v.b.re, v.b.im};
        m.a[1][1] = conj(v.a);
        return m;
    } else {
        return su2_to_spin_one(v.a, v.b);
    }
}

// sin x and cos x: for |x| <= 1/2 by their Taylor series (terms to x^15 and x^16, coefficients 1/n!;
// the first omitted terms are below 2e-17 there, and the results agree with sin and cos to one
// rounding), else by sincos.  For the small per-interval frame phases of the tensor path.
SS_D void sincos_small(double x, double* s, double* c) {
    if (fabs(x) <= 0.5) {
        const double y = x * x;
        double q = -1.0 / 1307674368000.0;        // -1/15!
        q = fma(q, y, 1.0 / 6227020800.0);        //  1/13!
        q = fma(q, y, -1.0 / 39916800.0);         // -1/11!
        q = fma(q, y, 1.0 / 362880.0);            //  1/9!
        q = fma(q, y, -1.0 / 5040.0);             // -1/7!
        q = fma(q, y, 1.0 / 120.0);               //  1/5!
        q = fma(q, y, -1.0 / 6.0);                // -1/3!
        *s = fma(x * y, q, x);
        double r = 1.0 / 20922789888000.0;        //  1/16!
        r = fma(r, y, -1.0 / 87178291200.0);      // -1/14!
        r = fma(r, y, 1.0 / 479001600.0);         //  1/12!
        r = fma(r, y, -1.0 / 3628800.0);          // -1/10!
        r = fma(r, y, 1.0 / 40320.0);             //  1/8!
        r = fma(r, y, -1.0 / 720.0);              // -1/6!
        r = fma(r, y, 1.0 / 24.0);                //  1/4!
        r = fma(r, y, -0.5);
        *c = fma(y, r, 1.0);
    } else {
        sincos(x, s, c);
    }
}

#ifdef __CUDACC__
// Programmatic dependent launch (kernels launched with programmatic stream serialization):
// grid_dependency_wait blocks until the preceding kernel in the stream has completed and its writes
// are visible; grid_dependency_release lets the following kernel start launching.  Both are no-ops
// for kernels launched without the attribute.
SS_D void grid_dependency_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
SS_D void grid_dependency_release() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }

SS_D Su2p shfl_down_su2p(const Su2p& v, int delta) {
    Su2p o;
    o.a.re = __shfl_down_sync(0xffffffffu, v.a.re, delta);
    o.a.im = __shfl_down_sync(0xffffffffu, v.a.im, delta);
    o.b.re = __shfl_down_sync(0xffffffffu, v.b.re, delta);
    o.b.im = __shfl_down_sync(0xffffffffu, v.b.im, delta);
    return o;
}

SS_D Su2p shfl_up_su2p(const Su2p& v, int delta) {
    Su2p o;
    o.a.re = __shfl_up_sync(0xffffffffu, v.a.re, delta);
    o.a.im = __shfl_up_sync(0xffffffffu, v.a.im, delta);
    o.b.re = __shfl_up_sync(0xffffffffu, v.b.re, delta);
    o.b.im = __shfl_up_sync(0xffffffffu, v.b.im, delta);
    return o;
}

SS_D Su2p shfl_su2p(const Su2p& v, int src) {
    Su2p o;
    o.a.re = __shfl_sync(0xffffffffu, v.a.re, src);
    o.a.im = __shfl_sync(0xffffffffu, v.a.im, src);
    o.b.re = __shfl_sync(0xffffffffu, v.b.re, src);
    o.b.im = __shfl_sync(0xffffffffu, v.b.im, src);
    return o;
}

// Warp shuffles of a whole operator (every lane of the warp must take part).
template <int D>
__device__ __forceinline__ Mat<D> shfl_down_mat(const Mat<D>& m, int delta) {
    Mat<D> o;
#pragma unroll
    for (int i = 0; i < D; i++)
#pragma unroll
        for (int j = 0; j < D; j++) {
            o.a[i][j].re = __shfl_down_sync(0xffffffffu, m.a[i][j].re, delta);
            o.a[i][j].im = __shfl_down_sync(0xffffffffu, m.a[i][j].im, delta);
        }
    return o;
}

template <int D>
__device__ __forceinline__ Mat<D> shfl_up_mat(const Mat<D>& m, int delta) {
    Mat<D> o;
#pragma unroll
    for (int i = 0; i < D; i++)
#pragma unroll
        for (int j = 0; j < D; j++) {
            o.a[i][j].re = __shfl_up_sync(0xffffffffu, m.a[i][j].re, delta);
            o.a[i][j].im = __shfl_up_sync(0xffffffffu, m.a[i][j].im, delta);
        }
    return o;
}
#endif

}  // namespace spinsim
