// The time-evolution kernel: the reference's get_time_evolution (spinsim/__init__.py:855-896),
// which maps one CUDA thread to one output interval, rebuilt as a warp-tiled (and, for batches,
// persistent) launch.
//
// A warp takes one Tile (up to 32 / lanes consecutive output intervals of one instance).  Without a
// tile list the launch covers a single instance with one tile per warp.  With a tile list and a
// counter, warps pull tiles from a global atomic queue until it is empty; tiles are ordered
// longest-first on the host, so instances of very different durations share one launch without a
// long tail.  No warp ever waits for another warp.
#pragma once
#include "common.cuh"
#include "evolve32.cuh"
#include "evolve64.cuh"

namespace spinsim {

template <int DIMS, int INTEG, int EXPO_H, int EXPO_O, int FIELD, int PREC>
SS_D void evolve_body(const EvolveArgs& a) {
    // FP32-bulk Magnus CF4 tone fields are synthesised per warp: every lane takes kSynthIntervals
    // intervals (the host sets lanes = 1 for these plans).
    constexpr bool SYNTH = (PREC == PREC_FP32_BULK && FIELD == FIELD_TONES && INTEG == INTEG_CF4);
    const int lane = threadIdx.x & 31;
    const int lanes = a.m.lanes;
    const int group = lane / lanes;
    const int lane_in_group = lane - group * lanes;
    const int per_warp = (SYNTH ? 32 * kSynthIntervals : 32) / lanes;
    const int64_t warp_global = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int64_t tile_id = warp_global;
    for (;;) {
        if (a.tile_counter != nullptr) {
            int t = 0;
            if (lane == 0) t = atomicAdd(a.tile_counter, 1);
            tile_id = __shfl_sync(0xffffffffu, t, 0);
        }
        if (tile_id >= a.n_tiles) return;
        Tile tile;
        if (a.tiles != nullptr) {
            tile = a.tiles[tile_id];
        } else {
            const int64_t n = a.instances[0].n_out;
            const int64_t first = tile_id * per_warp;
            tile.instance = 0;
            tile.first = first;
            tile.count = (int)((n - first) < per_warp ? (n - first) : per_warp);
        }
        const Instance& inst = a.instances[tile.instance];
        const FieldDesc& f = a.fields[inst.field];
        double* time_out = a.time + inst.out_offset;
        double* u_out = a.u + inst.u_offset;
        float* norms_out = a.step_norms != nullptr ? a.step_norms + inst.out_offset : nullptr;
        const int dim = (DIMS == 0) ? inst.dim : DIMS;
        if constexpr (SYNTH) {
            if (DIMS != 2 && dim == 3 && tones_have_quadratic_shift(f)) {
                // spin one with a quadratic shift: 3x3 exponentials, tones sampled directly
#pragma unroll 1
                for (int i = 0; i < kSynthIntervals; i++) {
                    const bool act = lane + 32 * i < tile.count;
                    const int64_t idx = tile.first + (act ? lane + 32 * i : 0);
                    interval32<3, INTEG, EXPO_O, FIELD>(a.m, inst, f, idx, act, 0, time_out, u_out, norms_out);
                }
            } else if (DIMS != 3 && dim == 2) {
                intervals32_synth<2, EXPO_H>(a.m, inst, f, tile, time_out, u_out, norms_out);
            } else if (DIMS != 2) {
                intervals32_synth<3, EXPO_O>(a.m, inst, f, tile, time_out, u_out, norms_out);
            }
        } else {
            const bool active = group < tile.count;
            const int64_t index = tile.first + (active ? group : 0);
            if (DIMS != 3 && dim == 2) {
                if constexpr (PREC == PREC_FP64)
                    interval64<2, INTEG, EXPO_H, FIELD>(a.m, inst, f, index, active, lane_in_group, time_out, u_out);
                else
                    interval32<2, INTEG, EXPO_H, FIELD>(a.m, inst, f, index, active, lane_in_group, time_out, u_out, norms_out);
            } else if (DIMS != 2) {
                if constexpr (PREC == PREC_FP64)
                    interval64<3, INTEG, EXPO_O, FIELD>(a.m, inst, f, index, active, lane_in_group, time_out, u_out);
                else
                    interval32<3, INTEG, EXPO_O, FIELD>(a.m, inst, f, index, active, lane_in_group, time_out, u_out, norms_out);
            }
        }
        if (a.tile_counter == nullptr) return;
    }
}

// MINB = minimum resident CTAs per SM that the register allocation must allow (128-thread CTAs):
// 2 leaves the full register file to one thread (255), 3 caps at 168, 4 at 128 registers.
template <int DIMS, int INTEG, int EXPO_H, int EXPO_O, int FIELD, int PREC, int MINB>
__global__ void __launch_bounds__(kEvolveThreadsMax, MINB) evolve_kernel(EvolveArgs a) {
    evolve_body<DIMS, INTEG, EXPO_H, EXPO_O, FIELD, PREC>(a);
}

}  // namespace spinsim
