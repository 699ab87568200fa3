// State propagation and spin expectation.
//
// The reference propagates the state serially on the host (get_state, spinsim/__init__.py:1089-1111):
//     state[0] = psi0,   state[i] = U[i-1] state[i-1]
// i.e. state[i] = (U[i-1] ... U[0]) psi0 and the last operator is never applied.  Here that is a
// parallel prefix scan of the d x d operators in FP64 over scan tiles of kScanTile consecutive
// output steps of one instance (one warp each), with no waits between blocks:
// A tile is taken by an 8-lane group (four tiles per warp); lane j of the group holds the product of
// the tile's operators 4 j .. 4 j + 3, so a tile costs three shuffle rounds instead of five.  A warp
// first copies its four tiles' operators into shared memory with coalesced loads (consecutive lanes,
// consecutive 16-byte words), and the apply kernel stages the states there for a coalesced write-out.
//   A  scan_products_kernel: each group multiplies its tile's operators into the tile product.  On the
//      tensor path (evolve_dmma.cuh) the time evolution writes each tile's four warp products as
//      SU(2) pairs instead, and A is not launched; B then scans SU(2) pairs (partials mode).
//   B  scan_prefix_kernel: a warp per instance scans the instance's tile products 32 at a time and
//      stores every tile's exclusive prefix (and, when asked, the instance's whole product).
//   C  scan_apply_kernel: each group scans its lanes' products (lane j: U[4j+3] ... U[0] of the
//      tile), applies the exclusive part times the tile's prefix to psi0 and steps through its
//      four output steps writing state and spin (get_spin, I:899-959), fused.
// The tile list holds the spin-half tiles, then the spin-one tiles, each run padded to whole warps
// (count 0); the tile kernels are launched once per spin dimension over its run of tiles.
#pragma once
#include "common.cuh"

namespace spinsim {

constexpr int kScanPerLane = 4;      // consecutive operators multiplied by one lane (kScanTile steps per tile)
constexpr int kScanGroup = kScanTile / kScanPerLane;  // lanes per tile (8)
constexpr int kScanTilesPerWarp = 32 / kScanGroup;    // 4
constexpr int kScanBlock = 128;      // threads per CTA of the scan kernels

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

#ifdef __CUDACC__
// Inclusive scan: lane i receives M[i] ... M[0].
template <int D>
SS_D Mat<D> warp_scan(Mat<D> m, int lane) {
#pragma unroll
    for (int s = 1; s < 32; s <<= 1) {
        const Mat<D> earlier = shfl_up_mat(m, s);
        if (lane >= s) m = matmul(m, earlier);
    }
    return m;
}
#endif

// Scan tiles: tile -> (instance, first output step, count).  Without a tile list (tiles == null) the
// launch covers one instance, instances[0], with implicit tiles of kScanTile steps.
struct ScanArgs {
    const Instance* instances;
    const Tile* tiles;          // scan tiles, grouped by instance in order; null: implicit tiles
    int64_t n_tiles;
    const int32_t* tile_begin;  // per instance: first scan tile (implicit for a single instance)
    const int32_t* tile_end;
    int32_t n_instances;
    const double* u;            // operators, FP64 complex
    double* tile_product;       // [n_tiles][kScanMat]
    double* tile_prefix;        // [n_tiles][kScanMat]
    double* state;              // complex [sum N * d]
    double* spin;               // [sum N * 3], may be null
    double* total;              // per instance: U[N-1] ... U[0], complex [d][d]; may be null
    int64_t single_n_out;       // output steps of the single instance (implicit tiles)
    int32_t partials;           // 1: tile_product holds each tile's four warp partials (SU(2) pairs) written by
                                // the tensor-path time evolution, in place of the tile products
    const double* rows;         // partials mode: each output step's operator as its SU(2) pair (4 doubles,
                                // indexed like time), which the apply reads in place of u; may be null
};

SS_D const Instance& scan_instance(const ScanArgs& a, int32_t i) { return a.instances[i]; }

// Tile k, or an empty tile (count 0) past the end of the list.
SS_D Tile scan_tile(const ScanArgs& a, int64_t k) {
    Tile t;
    t.instance = 0;
    t.first = 0;
    t.count = 0;
    if (k >= a.n_tiles) return t;
    if (a.tiles != nullptr) return a.tiles[k];
    t.first = k * kScanTile;
    const int64_t rest = a.single_n_out - t.first;
    t.count = (int32_t)(rest < kScanTile ? rest : kScanTile);
    return t;
}

// Writes a single call's instance (and field) descriptors into its workspace from the launch's own
// arguments: no host-to-device copy, so the call stays stream-ordered and capturable.
struct DescriptorArgs {
    Instance inst;
    FieldDesc field;
    Instance* inst_dst;
    FieldDesc* field_dst;  // may be null
};

#ifdef __CUDACC__
// Shared memory of a scan CTA for spin dimension D: per warp, its four tiles' operators; the apply
// kernel reuses the area for the tiles' states once every lane has read its operators.  Each lane's
// four operators (its segment) are padded by one 16-byte word, so that the eight lanes of a group,
// which read their segments in one phase of a 16-byte load, fall on distinct banks (segment strides
// of 272 and 592 bytes); staged states are padded the same way (144 and 208 bytes).  Spin-one CTAs
// take two warps, so both sizes stay within the default 48 KB of dynamic shared memory.
template <int D>
struct ScanShared {
    static constexpr int kWarps = D == 2 ? 4 : 2;
    static constexpr int kThreads = 32 * kWarps;
    static constexpr int kOpWords = kScanPerLane * D * D;     // 16-byte words of a lane's operators
    static constexpr int kSeg = 2 * (kOpWords + 1);          // doubles per lane segment, padded
    static constexpr int kStateWords = kScanPerLane * D;      // 16-byte words of a lane's states
    static constexpr int kStateSeg = 2 * (kStateWords + 1);  // doubles, padded
    static constexpr int kTile = kScanGroup * kSeg;          // doubles per tile
    static constexpr int kPerWarp = kScanTilesPerWarp * kTile;
    static constexpr size_t kBytes = sizeof(double) * (size_t)kPerWarp * kWarps;
    static_assert(kScanGroup * kStateSeg <= kTile, "staged states fit in the operators' area");
    static_assert(kBytes <= 48 * 1024, "scan tile kernels use the default dynamic shared memory limit");
};

// A warp's four tiles of operators, copied into shared memory with coalesced loads (one warp-wide
// pass per tile); lanes then read their four consecutive operators from there.
template <int D>
SS_D void stage_operators(const ScanArgs& a, int64_t first_tile, int64_t tile_hi, int lane, double* su) {
    using S = ScanShared<D>;
    constexpr int MD = 2 * D * D;
#pragma unroll
    for (int t = 0; t < kScanTilesPerWarp; t++) {
        const Tile tile = scan_tile(a, first_tile + t < tile_hi ? first_tile + t : a.n_tiles);
        if (tile.count <= 0) continue;
        const Instance& inst = scan_instance(a, tile.instance);
        const double2* src = reinterpret_cast<const double2*>(a.u + inst.u_offset + tile.first * MD);
        double2* dst = reinterpret_cast<double2*>(su + t * S::kTile);
        const int words = tile.count * D * D;
#pragma unroll
        for (int r = 0; r < D * D; r++) {  // a full tile is D * D words per lane
            const int e = lane + 32 * r;
            if (e < words) dst[e + e / S::kOpWords] = __ldg(src + e);
        }
    }
    __syncwarp();
}

template <int D>
SS_D Mat<D> shared_mat(const double* p) {
    Mat<D> m;
    const double2* q = reinterpret_cast<const double2*>(p);
#pragma unroll
    for (int i = 0; i < D; i++)
#pragma unroll
        for (int j = 0; j < D; j++) {
            const double2 v = q[i * D + j];
            m.a[i][j] = c64{v.x, v.y};
        }
    return m;
}

// Lane j of the tile's group: U[4j + 3] ... U[4j] of the tile (identity past its end), from the
// tile's operators in shared memory (su: the tile's area).
template <int D>
SS_D Mat<D> lane_operators(const double* su, const Tile& tile, int j) {
    constexpr int MD = 2 * D * D;
    const double* u = su + j * ScanShared<D>::kSeg;
    const int n = min(kScanPerLane, tile.count - kScanPerLane * j);
    Mat<D> p;
    if (n > 0) p = shared_mat<D>(u);
    else set_identity(p);
#pragma unroll
    for (int i = 1; i < kScanPerLane; i++)
        if (i < n) p = matmul(shared_mat<D>(u + i * MD), p);
    return p;
}

template <int D>
SS_D void products_group(const ScanArgs& a, const Tile& tile, int64_t k, int j, const double* su) {
    Mat<D> m;
    if (tile.count > 0) m = lane_operators<D>(su, tile, j);
    else set_identity(m);
#pragma unroll
    for (int s = 1; s < kScanGroup; s <<= 1) {  // tree over the group's lanes, later ones from the left
        const Mat<D> later = shfl_down_mat(m, s);
        if ((j & (2 * s - 1)) == 0) m = matmul(later, m);
    }
    if (j == 0 && tile.count > 0) store_mat<D>(a.tile_product + k * kScanMat, m);
}

#ifdef SPINSIM_SCAN_KERNELS  // the launches themselves are defined once, in the C ABI's unit
__global__ void put_descriptors_kernel(DescriptorArgs a) {
    if (threadIdx.x == 0) {
        *a.inst_dst = a.inst;
        if (a.field_dst != nullptr) *a.field_dst = a.field;
    }
}

extern __shared__ __align__(16) double scan_smem[];

// Tiles [tile_lo, tile_hi) of spin dimension D (the tile list keeps each dimension's tiles together).
template <int D>
__global__ void __launch_bounds__(ScanShared<D>::kThreads) scan_products_kernel(ScanArgs a, int64_t tile_lo,
                                                                               int64_t tile_hi) {
    const int64_t w0 =
        tile_lo + (((int64_t)blockIdx.x * ScanShared<D>::kThreads + threadIdx.x) >> 5) * kScanTilesPerWarp;
    const int lane = threadIdx.x & 31;
    if (w0 >= tile_hi) return;
    double* su = scan_smem + (threadIdx.x >> 5) * ScanShared<D>::kPerWarp;
    stage_operators<D>(a, w0, tile_hi, lane, su);
    const int t = lane / kScanGroup;
    const int64_t k = w0 + t;
    products_group<D>(a, scan_tile(a, k < tile_hi ? k : a.n_tiles), k, lane % kScanGroup, su + t * ScanShared<D>::kTile);
}

#endif

template <int D>
SS_D void prefix_warp(const ScanArgs& a, int32_t i, int lane) {
    const int32_t b = a.tile_begin != nullptr ? a.tile_begin[i] : 0;
    const int32_t e = a.tile_end != nullptr ? a.tile_end[i] : (int32_t)a.n_tiles;
    Mat<D> run, next;
    set_identity(run);
    if (b + lane < e) next = load_mat<D>(a.tile_product + (int64_t)(b + lane) * kScanMat);
    else set_identity(next);
    for (int32_t c0 = b; c0 < e; c0 += 32) {
        const int32_t k = c0 + lane;
        const Mat<D> p = next;
        if (c0 + 32 + lane < e) next = load_mat<D>(a.tile_product + (int64_t)(c0 + 32 + lane) * kScanMat);  // prefetch
        else set_identity(next);
        const Mat<D> incl = warp_scan<D>(p, lane);
        Mat<D> excl = shfl_up_mat(incl, 1);
        if (lane == 0) set_identity(excl);
        if (k < e) store_mat<D>(a.tile_prefix + (int64_t)k * kScanMat, matmul(excl, run));
        run = matmul(shfl_down_mat(incl, 31 - lane), run);  // lane 31's inclusive product (a full chunk)
    }
    if (a.total != nullptr && lane == 0) store_mat<D>(a.total + (int64_t)i * 2 * D * D, run);
}

// A tile's four warp partials (SU(2) pairs), loaded as they are stored; identity past the instance.
struct TilePartials {
    double2 v[8];
};

SS_D TilePartials load_partials(const ScanArgs& a, int64_t k, bool valid) {
    TilePartials t;
    const double2* p = reinterpret_cast<const double2*>(a.tile_product + k * kScanMat);
#pragma unroll
    for (int e = 0; e < 8; e++) t.v[e] = valid ? __ldg(p + e) : make_double2((e & 1) ? 0.0 : 1.0, 0.0);
    return t;
}

// The tile's product from its partials (warp 3's rows are the latest).
SS_D Su2p tile_product_of(const TilePartials& t) {
    Su2p r;
#pragma unroll
    for (int w = 0; w < 4; w++) {
        const Su2p v = Su2p{c64{t.v[2 * w].x, t.v[2 * w].y}, c64{t.v[2 * w + 1].x, t.v[2 * w + 1].y}};
        r = w == 0 ? v : su2p_mul(v, r);
    }
    return r;
}

// prefix_warp on SU(2) pairs (tile products from the time evolution's partials); the stored prefixes
// and total are the d x d operators.
template <int D>
SS_D void prefix_warp_su2(const ScanArgs& a, int32_t i, int lane) {
    const int32_t b = a.tile_begin != nullptr ? a.tile_begin[i] : 0;
    const int32_t e = a.tile_end != nullptr ? a.tile_end[i] : (int32_t)a.n_tiles;
    Su2p run = su2p_identity();
    TilePartials next = load_partials(a, b + lane, b + lane < e);
    for (int32_t c0 = b; c0 < e; c0 += 32) {
        const int32_t k = c0 + lane;
        Su2p incl = tile_product_of(next);
        // the next chunk's partials are loaded here and used in the next iteration (in flight meanwhile)
        next = load_partials(a, c0 + 32 + lane, c0 + 32 + lane < e);
#pragma unroll
        for (int s = 1; s < 32; s <<= 1) {  // lane l receives P[l] ... P[0] of the chunk
            const Su2p earlier = shfl_up_su2p(incl, s);
            if (lane >= s) incl = su2p_mul(incl, earlier);
        }
        Su2p excl = shfl_up_su2p(incl, 1);
        if (lane == 0) excl = su2p_identity();
        if (k < e) store_mat<D>(a.tile_prefix + (int64_t)k * kScanMat, su2p_to_mat<D>(su2p_mul(excl, run)));
        run = su2p_mul(shfl_su2p(incl, 31), run);  // lane 31's inclusive product (a full chunk)
    }
    if (a.total != nullptr && lane == 0) store_mat<D>(a.total + (int64_t)i * 2 * D * D, su2p_to_mat<D>(run));
}

#ifdef SPINSIM_SCAN_KERNELS
__global__ void __launch_bounds__(kScanBlock) scan_prefix_kernel(ScanArgs a) {
    grid_dependency_wait();  // the tile products (or partials) of the preceding kernel
    const int32_t i = (int32_t)(((int64_t)blockIdx.x * kScanBlock + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= a.n_instances) return;
    const bool half = scan_instance(a, i).dim == 2;
    if (a.partials) {
        if (half) prefix_warp_su2<2>(a, i, lane);
        else prefix_warp_su2<3>(a, i, lane);
    } else {
        if (half) prefix_warp<2>(a, i, lane);
        else prefix_warp<3>(a, i, lane);
    }
}

#endif

// The group's tile: lane j computes the states of output steps 4j .. 4j + 3 into hist (n of them),
// from the tile's staged operators (su), tile prefix (pre_s, d x d) and psi0 (psi0_s).
template <int D>
SS_D int apply_group(const Tile& tile, int j, const double* su, const double* pre_s, const double* psi0_s,
                     c64 (&hist)[kScanPerLane][D]) {
    constexpr int MD = 2 * D * D;
    Mat<D> m;
    if (tile.count > 0) m = lane_operators<D>(su, tile, j);
    else set_identity(m);
#pragma unroll
    for (int s = 1; s < kScanGroup; s <<= 1) {  // inclusive scan over the group's lanes
        const Mat<D> earlier = shfl_up_mat(m, s);
        if (j >= s) m = matmul(m, earlier);
    }
    Mat<D> excl = shfl_up_mat(m, 1);
    if (j == 0) set_identity(excl);
    const int first = kScanPerLane * j;
    if (tile.count <= first) return 0;
    // psi = (exclusive prefix) (tile prefix) psi0 at output step `first`, then the next three steps
    const Mat<D> pre = shared_mat<D>(pre_s);
    c64 v[D], psi[D];
#pragma unroll
    for (int r = 0; r < D; r++) {
        c64 acc = c64{0.0, 0.0};
#pragma unroll
        for (int c = 0; c < D; c++) acc = cfma(pre.a[r][c], c64{psi0_s[2 * c], psi0_s[2 * c + 1]}, acc);
        v[r] = acc;
    }
#pragma unroll
    for (int r = 0; r < D; r++) {
        c64 acc = excl.a[r][0] * v[0];
#pragma unroll
        for (int c = 1; c < D; c++) acc = cfma(excl.a[r][c], v[c], acc);
        psi[r] = acc;
    }
    const double* u = su + j * ScanShared<D>::kSeg;
    const int n = min(kScanPerLane, tile.count - first);
#pragma unroll
    for (int i = 0; i < kScanPerLane; i++) {
#pragma unroll
        for (int r = 0; r < D; r++) hist[i][r] = psi[r];
        if (i + 1 < n) {
            const Mat<D> op = shared_mat<D>(u + i * MD);
            c64 nx[D];
#pragma unroll
            for (int r = 0; r < D; r++) {
                c64 acc = op.a[r][0] * psi[0];
#pragma unroll
                for (int c = 1; c < D; c++) acc = cfma(op.a[r][c], psi[c], acc);
                nx[r] = acc;
            }
#pragma unroll
            for (int r = 0; r < D; r++) psi[r] = nx[r];
        }
    }
    return n;
}

// apply_group on the tile's staged SU(2) pairs (su: lane j's four pairs at j * seg doubles): the lane
// products and the group's scan are SU(2) products, and each step's d x d operator is formed only
// to advance the state.
template <int D>
SS_D int apply_group_rows(const Tile& tile, int j, const double* su, int seg, const double* pre_s,
                          const double* psi0_s, c64 (&hist)[kScanPerLane][D]) {
    const double2* mine = reinterpret_cast<const double2*>(su + j * seg);
    auto row = [&](int i) {
        const double2 x = mine[2 * i], y = mine[2 * i + 1];
        return Su2p{c64{x.x, x.y}, c64{y.x, y.y}};
    };
    const int first = kScanPerLane * j;
    const int n = min(kScanPerLane, tile.count - first);
    Su2p m = su2p_identity();
#pragma unroll
    for (int i = 0; i < kScanPerLane; i++)
        if (i < n) m = i == 0 ? row(0) : su2p_mul(row(i), m);
#pragma unroll
    for (int s = 1; s < kScanGroup; s <<= 1) {  // inclusive scan over the group's lanes
        const Su2p earlier = shfl_up_su2p(m, s);
        if (j >= s) m = su2p_mul(m, earlier);
    }
    Su2p excl = shfl_up_su2p(m, 1);
    if (j == 0) excl = su2p_identity();
    if (tile.count <= first) return 0;
    // psi = (exclusive prefix) (tile prefix) psi0 at output step `first`, then the next three steps
    const Mat<D> pre = shared_mat<D>(pre_s);
    const Mat<D> e = su2p_to_mat<D>(excl);
    c64 v[D], psi[D];
#pragma unroll
    for (int r = 0; r < D; r++) {
        c64 acc = c64{0.0, 0.0};
#pragma unroll
        for (int c = 0; c < D; c++) acc = cfma(pre.a[r][c], c64{psi0_s[2 * c], psi0_s[2 * c + 1]}, acc);
        v[r] = acc;
    }
#pragma unroll
    for (int r = 0; r < D; r++) {
        c64 acc = e.a[r][0] * v[0];
#pragma unroll
        for (int c = 1; c < D; c++) acc = cfma(e.a[r][c], v[c], acc);
        psi[r] = acc;
    }
#pragma unroll
    for (int i = 0; i < kScanPerLane; i++) {
#pragma unroll
        for (int r = 0; r < D; r++) hist[i][r] = psi[r];
        if (i + 1 < n) {
            const Mat<D> op = su2p_to_mat<D>(row(i));
            c64 nx[D];
#pragma unroll
            for (int r = 0; r < D; r++) {
                c64 acc = op.a[r][0] * psi[0];
#pragma unroll
                for (int c = 1; c < D; c++) acc = cfma(op.a[r][c], psi[c], acc);
                nx[r] = acc;
            }
#pragma unroll
            for (int r = 0; r < D; r++) psi[r] = nx[r];
        }
    }
    return n;
}

// Asynchronous global -> shared copies (cp.async): the apply kernel's two-deep pipeline.
SS_D void cp_async16(void* dst, const void* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
SS_D void cp_async8(void* dst, const void* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
SS_D void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
SS_D void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Shared memory of the apply kernel: per warp kStages buffers (the group being applied and the next
// group in flight; spin one from d x d operators: one, which keeps ten warps resident per SM for its
// longer arithmetic), each with four tiles of staged operators, the tile prefix and psi0.  ROWS: the
// operators are SU(2) pairs (four per lane segment, padded by one 16-byte word), and the area is as
// large as the tile's staged states.  Two warps per CTA: 36 KB and 39 KB from d x d operators, 20 KB
// and 30 KB from SU(2) pairs.
template <int D, bool ROWS = false>
struct ApplyShared {
    static constexpr int kOpWords = ROWS ? 2 * kScanPerLane : ScanShared<D>::kOpWords;  // per lane segment
    static constexpr int kSeg = 2 * (kOpWords + 1);                                     // doubles, padded
    static constexpr int kArea = kScanGroup * kSeg > kScanGroup * ScanShared<D>::kStateSeg
                                     ? kScanGroup * kSeg
                                     : kScanGroup * ScanShared<D>::kStateSeg;
    static constexpr int kStages = (D == 2 || ROWS) ? 2 : 1;
    static constexpr int kWarps = 2;
    static constexpr int kThreads = 32 * kWarps;
    static constexpr int kPrefix = kArea;                     // offset of the tile prefix (2 d^2 doubles)
    static constexpr int kPsi0 = kPrefix + 2 * D * D;         // offset of psi0 (2 d doubles)
    static constexpr int kTileStride = kPsi0 + 2 * D;         // doubles per staged tile (16-byte multiple)
    static constexpr int kBuffer = kScanTilesPerWarp * kTileStride;
    static constexpr size_t kBytes = sizeof(double) * kStages * (size_t)kBuffer * kWarps;
    static_assert(kTileStride % 2 == 0, "16-byte aligned tiles");
    static_assert(kBytes <= 48 * 1024, "the apply kernel uses the default dynamic shared memory limit");
};

// Issue the copies of tiles w0 .. w0 + 3 into buf (operators or SU(2) pairs, tile prefix, psi0),
// warp-cooperatively.
template <int D, bool ROWS>
SS_D void apply_issue(const ScanArgs& a, int64_t w0, int64_t tile_hi, int lane, double* buf) {
    using S = ApplyShared<D, ROWS>;
    constexpr int MD = 2 * D * D;
    constexpr int kWordsPerStep = ROWS ? 2 : D * D;
#pragma unroll
    for (int t = 0; t < kScanTilesPerWarp; t++) {
        const int64_t k = w0 + t;
        const Tile tile = scan_tile(a, k < tile_hi ? k : a.n_tiles);
        if (tile.count <= 0) continue;
        const Instance& inst = scan_instance(a, tile.instance);
        const double2* src = ROWS ? reinterpret_cast<const double2*>(a.rows + 4 * (inst.out_offset + tile.first))
                                  : reinterpret_cast<const double2*>(a.u + inst.u_offset + tile.first * MD);
        double* tb = buf + t * S::kTileStride;
        const int words = tile.count * kWordsPerStep;
#pragma unroll
        for (int r = 0; r < kWordsPerStep; r++) {  // a full tile is kWordsPerStep words per lane
            const int e = lane + 32 * r;
            if (e < words) cp_async16(tb + 2 * (e + e / S::kOpWords), src + e);
        }
        if (lane < D * D) cp_async16(tb + S::kPrefix + 2 * lane, a.tile_prefix + k * kScanMat + 2 * lane);
        if (lane < 2 * D) cp_async8(tb + S::kPsi0 + lane, inst.psi0 + lane);
    }
}

// Apply tiles w0 .. w0 + 3 from buf and write their states (and spins) out, coalesced.
template <int D, bool ROWS>
SS_D void apply_tiles(const ScanArgs& a, int64_t w0, int64_t tile_hi, int lane, double* buf) {
    using S = ApplyShared<D, ROWS>;
    const int t = lane / kScanGroup;
    const int j = lane % kScanGroup;
    const int64_t k = w0 + t;
    double* tb = buf + t * S::kTileStride;
    c64 hist[kScanPerLane][D];
    const Tile tile_k = scan_tile(a, k < tile_hi ? k : a.n_tiles);
    int n;
    if constexpr (ROWS) n = apply_group_rows<D>(tile_k, j, tb, S::kSeg, tb + S::kPrefix, tb + S::kPsi0, hist);
    else n = apply_group<D>(tile_k, j, tb, tb + S::kPrefix, tb + S::kPsi0, hist);
    __syncwarp();  // every lane is done with the operators: the area now takes the states
    double2* st = reinterpret_cast<double2*>(tb + j * ScanShared<D>::kStateSeg);
#pragma unroll
    for (int i = 0; i < kScanPerLane; i++)
        if (i < n)
#pragma unroll
            for (int r = 0; r < D; r++) st[i * D + r] = make_double2(hist[i][r].re, hist[i][r].im);
    __syncwarp();
    // coalesced write-out of the four tiles' states; the spin of step e from its staged state
#pragma unroll
    for (int tt = 0; tt < kScanTilesPerWarp; tt++) {
        const Tile tile = scan_tile(a, w0 + tt < tile_hi ? w0 + tt : a.n_tiles);
        if (tile.count <= 0) continue;
        const Instance& inst = scan_instance(a, tile.instance);
        const double2* from = reinterpret_cast<const double2*>(buf + tt * S::kTileStride);
        double2* to = reinterpret_cast<double2*>(a.state + inst.state_offset) + tile.first * D;
#pragma unroll
        for (int r = 0; r < D; r++) {  // a full tile is D words per lane
            const int e = lane + 32 * r;
            if (e < tile.count * D) to[e] = from[e + e / ScanShared<D>::kStateWords];
        }
        if (a.spin != nullptr && lane < tile.count) {
            const double2* mine = from + lane * D + lane / kScanPerLane;
            c64 psi[D];
#pragma unroll
            for (int r = 0; r < D; r++) psi[r] = c64{mine[r].x, mine[r].y};
            double s3[3];
            spin_of<D>(psi, s3);
            double* sto = a.spin + (inst.out_offset + tile.first + lane) * 3;
            sto[0] = s3[0];
            sto[1] = s3[1];
            sto[2] = s3[2];
        }
    }
}

#ifdef SPINSIM_SCAN_KERNELS
// Tiles [tile_lo, tile_hi) of spin dimension D in groups of four per warp; persistent warps take every
// stride-th group, with kStages groups' copies in flight (spin half: the next group is copied while the
// current one is applied).  after_prefix: the preceding kernel is the prefix kernel, whose results
// this one waits for before it starts; otherwise it follows the other spin's apply kernel, which has
// already waited for them, so it starts at once and waits for that kernel only before it completes.
template <int D, bool ROWS>
__global__ void __launch_bounds__(ApplyShared<D, ROWS>::kThreads) scan_apply_kernel(ScanArgs a, int64_t tile_lo,
                                                                                   int64_t tile_hi, int32_t after_prefix) {
    using S = ApplyShared<D, ROWS>;
    if (after_prefix) grid_dependency_wait();
    grid_dependency_release();  // the other spin's apply kernel may start: the prefixes are complete
    const int lane = threadIdx.x & 31;
    const int64_t groups = (tile_hi - tile_lo + kScanTilesPerWarp - 1) / kScanTilesPerWarp;
    const int64_t stride = (int64_t)gridDim.x * S::kWarps;
    int64_t g = (int64_t)blockIdx.x * S::kWarps + (threadIdx.x >> 5);
    if (g >= groups) {  // warp-uniform
        if (!after_prefix) grid_dependency_wait();
        return;
    }
    double* buf0 = scan_smem + (threadIdx.x >> 5) * S::kStages * S::kBuffer;
#pragma unroll
    for (int st = 0; st < S::kStages; st++) {
        if (g + st * stride < groups)
            apply_issue<D, ROWS>(a, tile_lo + kScanTilesPerWarp * (g + st * stride), tile_hi, lane, buf0 + st * S::kBuffer);
        cp_async_commit();
    }
    for (int it = 0; g < groups; it = (it + 1) % S::kStages, g += stride) {
        double* buf = buf0 + it * S::kBuffer;
        cp_async_wait<S::kStages - 1>();  // this buffer's copies have landed (later ones may be in flight)
        __syncwarp();
        apply_tiles<D, ROWS>(a, tile_lo + kScanTilesPerWarp * g, tile_hi, lane, buf);
        __syncwarp();  // the write-out has read the buffer before it is refilled
        if (g + S::kStages * stride < groups)
            apply_issue<D, ROWS>(a, tile_lo + kScanTilesPerWarp * (g + S::kStages * stride), tile_hi, lane, buf);
        cp_async_commit();
    }
    cp_async_wait<0>();
    if (!after_prefix) grid_dependency_wait();  // complete only after the preceding apply kernel
}
#endif  // SPINSIM_SCAN_KERNELS
#endif

#ifdef SPINSIM_SCAN_KERNELS
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

#endif  // SPINSIM_SCAN_KERNELS

}  // namespace spinsim
