// State propagation and spin expectation.
//
// The reference propagates the state serially on the host (get_state, spinsim/__init__.py:1089-1111):
//     state[0] = psi0,   state[i] = U[i-1] state[i-1]
// i.e. state[i] = (U[i-1] ... U[0]) psi0 and the last operator is never applied.  Here that is a
// parallel prefix scan of the d x d operators in FP64, in three launches with no inter-block waits:
//   A  scan_reduce_kernel: each CTA takes a scan tile of kScanThreads * kScanChunk consecutive
//      intervals of one instance; thread t multiplies its kScanChunk operators, the CTA scans the
//      thread products in shared memory and stores each thread's exclusive in-tile prefix and the
//      tile product.
//   B  scan_tiles_kernel: one thread per instance walks its tiles in order and stores the
//      exclusive prefix of every tile (and, when asked, the instance's whole product).
//   C  scan_apply_kernel: thread t forms prefix = (in-tile prefix) (tile prefix), applies it to psi0
//      and walks its chunk writing state and spin (get_spin, I:899-959), fused.
#pragma once
#include "common.cuh"

namespace spinsim {

constexpr int kScanThreads = 256;
constexpr int kScanChunk = 8;
constexpr int kScanTile = kScanThreads * kScanChunk;

template <int D>
SS_D Mat<D> load_mat(const double* p) {
    Mat<D> m;
    const double2* q = reinterpret_cast<const double2*>(p);
#pragma unroll
    for (int i = 0; i < D; i++)
#pragma unroll
        for (int j = 0; j < D; j++) {
            const double2 v = __ldg(q + i * D + j);
            m.a[i][j] = c64{v.x, v.y};
        }
    return m;
}

template <int D>
SS_D void store_mat(double* p, const Mat<D>& m) {
    double2* q = reinterpret_cast<double2*>(p);
#pragma unroll
    for (int i = 0; i < D; i++)
#pragma unroll
        for (int j = 0; j < D; j++) q[i * D + j] = make_double2(m.a[i][j].re, m.a[i][j].im);
}

// get_spin, I:938-944 (spin half) and I:942-944 (spin one)
template <int D>
SS_D void spin_of(const c64* s, double* out) {
    if constexpr (D == 2) {
        const c64 p = s[0] * conj(s[1]);
        out[0] = p.re;
        out[1] = -p.im;  // Re(i s0 conj(s1))
        out[2] = 0.5 * (s[0].re * s[0].re + s[0].im * s[0].im - s[1].re * s[1].re - s[1].im * s[1].im);
    } else {
        const c64 a = conj(s[1]) * (s[0] + s[2]);
        const c64 b = conj(s[1]) * (s[0] - s[2]);
        constexpr double r2 = 1.4142135623730951;
        out[0] = 2.0 * a.re / r2;
        out[1] = -2.0 * b.im / r2;  // Re(2i conj(s1)(s0 - s2)) / sqrt2
        out[2] = s[0].re * s[0].re + s[0].im * s[0].im - s[2].re * s[2].re - s[2].im * s[2].im;
    }
}

// Scan tiles: tile -> (instance, first interval, count); instance-local.
struct ScanArgs {
    const Instance* instances;
    const Tile* tiles;       // scan tiles (kScanTile intervals max), grouped by instance, in order
    int64_t n_tiles;
    const int32_t* tile_begin;  // per instance: first scan tile index (instances with this dim only)
    const int32_t* tile_end;
    int32_t n_instances;
    const double* u;          // operators, FP64 complex
    double* thread_prefix;    // [n_tiles][kScanThreads][D][D] complex: exclusive in-tile prefixes
    double* tile_product;     // [n_tiles][D][D] complex
    double* tile_prefix;      // [n_tiles][D][D] complex
    double* state;            // complex [sum N * d]
    double* spin;             // [sum N * 3], may be null
    double* total;            // per instance (of this dim): U[N-1] ... U[0], complex [D][D]; may be null
};

template <int D>
__global__ void __launch_bounds__(kScanThreads) scan_reduce_kernel(ScanArgs a) {
    constexpr int MD = 2 * D * D;  // doubles per matrix
    __shared__ double sh[kScanThreads * MD];
    const int64_t tile_id = blockIdx.x;
    if (tile_id >= a.n_tiles) return;
    const Tile tile = a.tiles[tile_id];
    const Instance& inst = a.instances[tile.instance];
    const double* u = a.u + inst.u_offset + (tile.first) * MD;
    const int t = threadIdx.x;
    const int lo = t * kScanChunk;
    int hi = lo + kScanChunk;
    if (hi > tile.count) hi = tile.count;
    Mat<D> p;
    set_identity(p);
    for (int i = lo; i < hi; i++) p = matmul(load_mat<D>(u + (int64_t)i * MD), p);
    // Hillis-Steele inclusive scan over threads: incl[t] = p[t] p[t-1] ... p[0]
    store_mat<D>(sh + t * MD, p);
    __syncthreads();
    for (int off = 1; off < kScanThreads; off <<= 1) {
        Mat<D> earlier;
        const bool take = t >= off;
        if (take) {
#pragma unroll
            for (int i = 0; i < D; i++)
#pragma unroll
                for (int j = 0; j < D; j++)
                    earlier.a[i][j] = c64{sh[(t - off) * MD + 2 * (i * D + j)], sh[(t - off) * MD + 2 * (i * D + j) + 1]};
        }
        __syncthreads();
        if (take) {
            p = matmul(p, earlier);
            store_mat<D>(sh + t * MD, p);
        }
        __syncthreads();
    }
    // exclusive prefix for thread t = inclusive of t - 1
    Mat<D> ex;
    if (t == 0) {
        set_identity(ex);
    } else {
#pragma unroll
        for (int i = 0; i < D; i++)
#pragma unroll
            for (int j = 0; j < D; j++)
                ex.a[i][j] = c64{sh[(t - 1) * MD + 2 * (i * D + j)], sh[(t - 1) * MD + 2 * (i * D + j) + 1]};
    }
    store_mat<D>(a.thread_prefix + (tile_id * kScanThreads + t) * MD, ex);
    if (t == kScanThreads - 1) store_mat<D>(a.tile_product + tile_id * MD, p);
}

template <int D>
__global__ void scan_tiles_kernel(ScanArgs a) {
    constexpr int MD = 2 * D * D;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n_instances) return;
    Mat<D> run;
    set_identity(run);
    for (int k = a.tile_begin[i]; k < a.tile_end[i]; k++) {
        store_mat<D>(a.tile_prefix + (int64_t)k * MD, run);
        run = matmul(load_mat<D>(a.tile_product + (int64_t)k * MD), run);
    }
    if (a.total) store_mat<D>(a.total + (int64_t)i * MD, run);
}

template <int D>
__global__ void __launch_bounds__(kScanThreads) scan_apply_kernel(ScanArgs a) {
    constexpr int MD = 2 * D * D;
    const int64_t tile_id = blockIdx.x;
    if (tile_id >= a.n_tiles) return;
    const Tile tile = a.tiles[tile_id];
    const Instance& inst = a.instances[tile.instance];
    const int t = threadIdx.x;
    const int lo = t * kScanChunk;
    if (lo >= tile.count) return;
    int hi = lo + kScanChunk;
    if (hi > tile.count) hi = tile.count;
    const Mat<D> pre = matmul(load_mat<D>(a.thread_prefix + (tile_id * kScanThreads + t) * MD),
                              load_mat<D>(a.tile_prefix + tile_id * MD));
    c64 psi[D], v[D];
#pragma unroll
    for (int k = 0; k < D; k++) v[k] = c64{inst.psi0[2 * k], inst.psi0[2 * k + 1]};
#pragma unroll
    for (int r = 0; r < D; r++) {
        c64 acc = pre.a[r][0] * v[0];
#pragma unroll
        for (int k = 1; k < D; k++) acc = cfma(pre.a[r][k], v[k], acc);
        psi[r] = acc;
    }
    const double* u = a.u + inst.u_offset + tile.first * MD;
    double2* st = reinterpret_cast<double2*>(a.state + inst.state_offset) + tile.first * D;
    double* sp = a.spin ? a.spin + (inst.out_offset + tile.first) * 3 : nullptr;
    for (int i = lo; i < hi; i++) {
#pragma unroll
        for (int k = 0; k < D; k++) st[(int64_t)i * D + k] = make_double2(psi[k].re, psi[k].im);
        if (sp) {
            double s3[3];
            spin_of<D>(psi, s3);
            sp[(int64_t)i * 3 + 0] = s3[0];
            sp[(int64_t)i * 3 + 1] = s3[1];
            sp[(int64_t)i * 3 + 2] = s3[2];
        }
        if (i + 1 < hi) {
            const Mat<D> m = load_mat<D>(u + (int64_t)i * MD);
            c64 nx[D];
#pragma unroll
            for (int r = 0; r < D; r++) {
                c64 acc = m.a[r][0] * psi[0];
#pragma unroll
                for (int k = 1; k < D; k++) acc = cfma(m.a[r][k], psi[k], acc);
                nx[r] = acc;
            }
#pragma unroll
            for (int r = 0; r < D; r++) psi[r] = nx[r];
        }
    }
}

// Standalone get_spin (I:899-959) for a state series: spin[i] from state[i].
template <int D>
__global__ void spin_kernel(const double* state, int64_t n, double* spin) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double2* s = reinterpret_cast<const double2*>(state) + i * D;
    c64 psi[D];
#pragma unroll
    for (int k = 0; k < D; k++) {
        const double2 v = __ldg(s + k);
        psi[k] = c64{v.x, v.y};
    }
    double o[3];
    spin_of<D>(psi, o);
    spin[i * 3 + 0] = o[0];
    spin[i * 3 + 1] = o[1];
    spin[i * 3 + 2] = o[2];
}

// Ensemble mean of the spin over members that share their output times (one evaluate() each,
// equal N, laid out one after another): mean[i][c] = (1/M) sum_m spin[first + m * stride + i][c].
// Launch A sums a chunk of members for 128 output steps per CTA (coalesced over i), launch B adds
// the chunk sums in chunk order, so the result does not depend on the launch shape's timing.
constexpr int kMeanThreads = 128;

__global__ void __launch_bounds__(kMeanThreads) spin_mean_partial_kernel(const double* spin, int64_t first,
                                                                         int64_t stride, int32_t members,
                                                                         int32_t per_chunk, int64_t n_out,
                                                                         double* partial) {
    const int64_t i = (int64_t)blockIdx.x * kMeanThreads + threadIdx.x;
    const int chunk = blockIdx.y;
    if (i >= n_out) return;
    const int m0 = chunk * per_chunk;
    const int m1 = min(members, m0 + per_chunk);
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (int m = m0; m < m1; m++) {
        const double* p = spin + (first + (int64_t)m * stride + i) * 3;
        sx += __ldg(p);
        sy += __ldg(p + 1);
        sz += __ldg(p + 2);
    }
    double* q = partial + ((int64_t)chunk * n_out + i) * 3;
    q[0] = sx;
    q[1] = sy;
    q[2] = sz;
}

__global__ void __launch_bounds__(kMeanThreads) spin_mean_final_kernel(const double* partial, int32_t chunks,
                                                                       int32_t members, int64_t n_out, double* mean) {
    const int64_t k = (int64_t)blockIdx.x * kMeanThreads + threadIdx.x;  // (i, c) flattened
    if (k >= n_out * 3) return;
    double s = 0.0;
    for (int c = 0; c < chunks; c++) s += partial[(int64_t)c * n_out * 3 + k];
    mean[k] = s / (double)members;
}

}  // namespace spinsim
