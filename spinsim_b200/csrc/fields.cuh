// Field sources for the time-evolution kernels.
//
//  FIELD_USER   the user's get_field(time_sample, sweep_parameters, field_sample) (the reference's
//               only extension point, spinsim/__init__.py:381-389, :620), compiled by numba to
//               LTO-IR behind a C-ABI shim and linked into the kernel with nvJitLink.
//  FIELD_TABLE  per-channel interpolation tables (the reference's generate_interpolation_sampler,
//               I:1941-2147): zero-order hold, linear or cubic Hermite, zero or held boundaries.
//  FIELD_TONES  per-channel bias + sum of sinusoids A sin(w t + phi).
#pragma once
#include "common.cuh"

#ifdef SPINSIM_USER_FIELD
// Provided by the numba-compiled shim: writes field_sample[0..8) (pre-zeroed by the caller).
extern "C" __device__ void spinsim_user_field(double time_sample, double* sweep_parameters, int64_t n_parameters,
                                              double* field_sample);
#endif

namespace spinsim {

// find_time_index (I:2026-2061): guess the index from equal spacing, bisect if the guess is wrong.
// Returns -1 outside the table (or after `size` bisection steps, as the reference does).
SS_D int64_t table_find(const TableChannel& tb, double ts, double* u) {
    const double* time = tb.time;
    const int64_t size = tb.size;
    *u = 0.0;
    const double first = __ldg(time), last = __ldg(time + size - 1);
    if (!(first <= ts && ts <= last)) return -1;
    int64_t idx = (int64_t)((ts - first) / (__ldg(time + 1) - first));
    bool low_enough = false, high_enough = true;
    if (idx + 1 < size) {
        low_enough = __ldg(time + idx) <= ts;
        high_enough = ts <= __ldg(time + idx + 1);
    } else {
        idx = size;
    }
    if (!(low_enough && high_enough)) {
        int64_t idx_max = size - 1, idx_min = 0, get_out = size;
        while (!(low_enough && high_enough)) {
            if (!low_enough) idx_max = idx;
            else idx_min = idx;
            idx = (int64_t)((double)(idx_max + idx_min) / 2.0);
            low_enough = false;
            high_enough = true;
            if (idx + 1 < size) {
                low_enough = __ldg(time + idx) <= ts;
                high_enough = ts <= __ldg(time + idx + 1);
            }
            if (--get_out == 0) return -1;
        }
    }
    const double t_lo = __ldg(time + idx), t_hi = __ldg(time + idx + 1);
    *u = (ts - t_lo) / (t_hi - t_lo);
    return idx;
}

// Interpolation given the interval index i and parameter u (the sampler bodies of I:2065-2140).
SS_D double table_value(const TableChannel& tb, int64_t i, double u) {
    const double* time = tb.time;
    const double* amp = tb.amplitude;
    const int64_t size = tb.size;
    if (tb.order == 0) return i >= 0 ? __ldg(amp + i) : 0.0;
    if (!(i >= 0 && i + 1 < size)) return 0.0;
    const double a0 = __ldg(amp + i), a1 = __ldg(amp + i + 1);
    if (tb.order == 1) return a0 * (1 - u) + a1 * u;
    const double t0 = __ldg(time + i), t1 = __ldg(time + i + 1);
    const double g_mid = (t0 != t1) ? (a1 - a0) / (t1 - t0) : 0.0;
    double g_left;
    if (i == 0) {
        g_left = g_mid;
    } else {
        const double tm = __ldg(time + i - 1);
        g_left = (tm != t0) ? 0.5 * ((a0 - __ldg(amp + i - 1)) / (t0 - tm) + g_mid) : 0.0;
    }
    g_left *= (t1 - t0);
    double g_right;
    if (i + 2 == size) {
        g_right = g_mid;
    } else {
        const double tp = __ldg(time + i + 2);
        g_right = (t1 != tp) ? 0.5 * ((__ldg(amp + i + 2) - a1) / (tp - t1) + g_mid) : 0.0;
    }
    g_right *= (t1 - t0);
    const double u2 = u * u, u3 = u2 * u;
    return a0 * (2 * u3 - 3 * u2 + 1) + a1 * (-2 * u3 + 3 * u2) + g_left * (u3 - 2 * u2 + u) + g_right * (u3 - u2);
}

// The sampler of I:2065-2140 with the reference's search.
SS_D double table_sample(const TableChannel& tb, double ts) {
    if (!tb.zero_boundary) {
        if (ts <= __ldg(tb.time)) return __ldg(tb.amplitude);
        if (ts >= __ldg(tb.time + tb.size - 1)) return __ldg(tb.amplitude + tb.size - 1);
    }
    double u;
    const int64_t i = table_find(tb, ts, &u);
    return table_value(tb, i, u);
}

// A per-lane cursor over one table for sample times that only increase (the fine steps of an
// output interval).  The interval [time[i], time[i+1]] that holds a sample strictly inside it is
// unique, so advancing the cursor finds the same index as the reference's search; a sample that
// lands exactly on a table time (or outside the table) goes to the reference's search, which picks
// among the touching intervals as the reference does.  Results are therefore identical to
// table_sample; the cursor only removes the bisection's chain of dependent loads.
//
// A cursor also keeps the channel's value while it is constant on (t_lo, t_hi): a zero-order-hold
// table's gain * amplitude[i] + bias, or the bias of a channel without a table (on the whole
// line).  A sample strictly inside that interval then takes the kept value and reads no memory; it
// is the value that the search would give there.
struct TableCursor {
    int32_t i = -1;    // -1: not positioned
    int32_t hold = 0;  // 1: val is the channel's value on (t_lo, t_hi)
    double t_lo = 0.0, t_hi = 0.0;
    double val = 0.0;
};

SS_D double table_sample_cursor(const TableChannel& tb, double ts, TableCursor& cur) {
    if (!tb.zero_boundary) {
        if (ts <= __ldg(tb.time)) return __ldg(tb.amplitude);
        if (ts >= __ldg(tb.time + tb.size - 1)) return __ldg(tb.amplitude + tb.size - 1);
    }
    if (cur.i >= 0) {
        while (ts >= cur.t_hi && cur.i + 2 < tb.size) {
            cur.i++;
            cur.t_lo = cur.t_hi;
            cur.t_hi = __ldg(tb.time + cur.i + 1);
        }
        if (ts > cur.t_lo && ts < cur.t_hi) return table_value(tb, cur.i, (ts - cur.t_lo) / (cur.t_hi - cur.t_lo));
    }
    double u;
    const int64_t i = table_find(tb, ts, &u);
    if (i >= 0 && i + 1 < tb.size && i < INT32_MAX) {
        cur.i = (int32_t)i;
        cur.t_lo = __ldg(tb.time + i);
        cur.t_hi = __ldg(tb.time + i + 1);
    }
    return table_value(tb, i, u);
}

// Sample the field at time t into out[0..NCH) (entries beyond NCH are left untouched).
// The caller pre-zeroes `out` like the reference does before each sample (I:625-642).  `cursors`
// (FIELD_TABLE, optional) hold one TableCursor per channel for increasing sample times.
template <int FIELD, int NCH>
SS_D void sample_field(const FieldDesc& f, double t, double* out, TableCursor* cursors = nullptr) {
    if constexpr (FIELD == FIELD_USER) {
#ifdef SPINSIM_USER_FIELD
        spinsim_user_field(t, const_cast<double*>(f.params), f.n_params, out);
#endif
    } else if constexpr (FIELD == FIELD_TABLE) {
#pragma unroll
        for (int c = 0; c < NCH; c++) {
            if (cursors && cursors[c].hold && t > cursors[c].t_lo && t < cursors[c].t_hi) {
                out[c] = cursors[c].val;
                continue;
            }
            const TableChannel& tb = f.tables[c];
            if (tb.size > 0) {
                const double v = cursors ? table_sample_cursor(tb, t, cursors[c]) : table_sample(tb, t);
                out[c] = fma(f.gain[c], v, f.bias[c]);
                if (cursors && tb.order == 0 && cursors[c].i >= 0) {
                    TableCursor& cu = cursors[c];
                    cu.hold = 1;
                    cu.val = fma(f.gain[c], __ldg(tb.amplitude + cu.i), f.bias[c]);
                }
            } else {
                out[c] = f.bias[c];
                if (cursors) {
                    TableCursor& cu = cursors[c];
                    cu.i = 0;
                    cu.hold = 1;
                    cu.t_lo = -INFINITY;
                    cu.t_hi = INFINITY;
                    cu.val = out[c];
                }
            }
        }
    } else {  // FIELD_TONES
#pragma unroll
        for (int c = 0; c < NCH; c++) {
            double acc = f.bias[c];
            const double* tone = f.tones + 3 * f.tone_start[c];
            const int n = f.tone_count[c];
            const double gain = f.gain[c];
            for (int k = 0; k < n; k++) {
                const double w = __ldg(tone + 3 * k), a = gain * __ldg(tone + 3 * k + 1), ph = __ldg(tone + 3 * k + 2);
                acc = fma(a, sin(fma(w, t, ph)), acc);
            }
            out[c] = acc;
        }
    }
}

}  // namespace spinsim
