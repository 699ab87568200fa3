// FP32-bulk time evolution of one output interval (see interval32 below).
#pragma once
#include "common.cuh"
#include "evolve64.cuh"

namespace spinsim {

template <int D, int INTEG, int EXPO, int FIELD>
SS_D void interval32(const MethodConfig& m, const Instance& inst, const FieldDesc& f, int64_t index, bool active,
                     int lane_in_group, double* time_out, double* u_out) {
    static_assert(D < 0, "FP32-bulk kernels are not built yet");
}

}  // namespace spinsim
