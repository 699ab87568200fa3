"""Field sources that need no user code, and the interpolation sampler for user fields.

* ``TabulatedField``: per-channel interpolation tables evaluated inside the kernel (the
  tabulated-field path).  Channel c (x, y, z, q, u1, u2, v1, v2) = bias[c] + gain[c] * table_c(t).
* ``ToneField``: per-channel bias + sum of sinusoids A sin(w t + phi).
* ``generate_interpolation_sampler``: the reference's sampler factory (spinsim/__init__.py:1941-2147)
  returning a numba device function to call from a user ``get_field``.

Tables follow the reference's interpolation rules exactly: zero-order hold (order 0), linear
(order 1) or cubic Hermite with finite-difference gradients (order 3); outside the table the value
is zero (``zero_boundary``) or the end value; the interval is found from the equal-spacing guess
and then by bisection (I:2026-2061), so non-uniform tables work.
"""
import math
from operator import attrgetter, itemgetter, methodcaller

import numpy as np

from . import _lib

CHANNELS = ("x", "y", "z", "q", "u1", "u2", "v1", "v2")


def _channel_index(c):
    if isinstance(c, str):
        return CHANNELS.index(c)
    c = int(c)
    if not 0 <= c < 8:
        raise ValueError("field channel must be in [0, 8)")
    return c


class BuiltinField:
    """Base of the library-evaluated fields: holds a host ``Field`` struct and its device arrays."""

    kind = None

    def device_struct(self, device):
        """Return (ctypes Field, keep-alive list) with device pointers for ``device``."""
        raise NotImplementedError


class TabulatedField(BuiltinField):
    """A field given by sampled time series, interpolated on the device.

    ``channels`` maps a channel (index or name) to ``(time, amplitude)``.  ``order`` and
    ``zero_boundary`` are as in the reference's ``generate_interpolation_sampler``; they may also be
    given per channel as ``(time, amplitude, order, zero_boundary)``.
    """

    kind = 1  # SPINSIM_FIELD_TABLE

    def __init__(self, channels, order=3, zero_boundary=True, bias=None, gain=None):
        if order not in (0, 1, 3):
            raise NotImplementedError(
                f"Interpolation order {order} is not implemented. Try order 0 (zero order hold), 1 (linear) or 3 (cubic).")
        self.tables = {}
        snapshots = {}  # channels given the same time array share one copy (packed once)
        for c, spec in dict(channels).items():
            idx = _channel_index(c)
            t, a = np.asarray(spec[0], np.float64), np.asarray(spec[1], np.float64)
            o = int(spec[2]) if len(spec) > 2 else order
            zb = bool(spec[3]) if len(spec) > 3 else zero_boundary
            if a.ndim != 1:
                raise NotImplementedError("Interpolation sampler does not work with multi-dimensional arrays yet. "
                                          "Try generating a single interpolator for each axis instead.")
            if t.shape != a.shape or t.size < 2:
                raise ValueError("a table needs matching time and amplitude arrays of at least two samples")
            if o not in (0, 1, 3):
                raise NotImplementedError(f"Interpolation order {o} is not implemented.")
            if id(spec[0]) not in snapshots:
                snapshots[id(spec[0])] = (spec[0], t.copy())  # (the input, kept alive so its id stays unique)
            self.tables[idx] = (snapshots[id(spec[0])][1], a.copy(), o, zb)
        self.bias = np.zeros(8)
        self.gain = np.ones(8)
        if bias is not None:
            for c, v in (bias.items() if isinstance(bias, dict) else enumerate(bias)):
                self.bias[_channel_index(c)] = v
        if gain is not None:
            for c, v in (gain.items() if isinstance(gain, dict) else enumerate(gain)):
                self.gain[_channel_index(c)] = v
        self._cplan()  # the packing plan of these snapshots, made once here rather than at each launch

    def device_struct(self, device):
        import torch
        keep = []
        tabs = (_lib.Table * 8)()
        for idx, (t, a, o, zb) in self.tables.items():
            td = torch.from_numpy(t).to(device)
            ad = torch.from_numpy(a).to(device)
            keep += [td, ad]
            tabs[idx] = _lib.Table(td.data_ptr(), ad.data_ptr(), t.size, o, int(zb))
        raw = torch.frombuffer(bytearray(bytes(tabs)), dtype=torch.uint8).to(device)
        keep.append(raw)
        f = _lib.Field()
        f.tables = raw.data_ptr()
        for c in range(8):
            f.bias[c] = self.bias[c]
            f.gain[c] = self.gain[c]
        return f, keep

    def uses_channel(self, c):
        return c in self.tables or self.bias[c] != 0.0

    def packed_doubles(self):
        """float64 entries in a packed field buffer: eight 4-double table descriptors, then the
        times (once per distinct time array) and amplitudes."""
        return 8 * _TABLE_DOUBLES + self._cplan()[1]

    def _cplan(self):
        """The field's rows of a ``spinsim_pack_fields`` plan (host pointers into the field's own
        arrays, which are snapshots) and the doubles of its arrays; computed once."""
        got = self.__dict__.get("_plan")
        if got is None:
            rows, index, n = [], {}, 0
            for k, c in enumerate(sorted(self.tables)):
                t, a, o, z = self.tables[c]
                alias = index.get(id(t), -1)
                if alias < 0:
                    index[id(t)] = k
                    n += t.size
                n += a.size
                rows.append((c, t.ctypes.data, a.ctypes.data, t.size, o, int(z), alias, 0))
            header = (1, len(rows), self.bias.ctypes.data, self.gain.ctypes.data, 0, 0, 0, 0)
            # the arrays the pointers refer to stay referenced by the plan
            keep = (self.bias, self.gain, [v[:2] for v in self.tables.values()])
            got = self._plan = (np.array([header] + rows, np.int64), n, keep)
        return got


class ToneField(BuiltinField):
    """channel c = bias[c] + sum_k A_k sin(w_k t + phi_k).

    ``tones`` maps a channel to an array of shape (n, 3) of (angular frequency, amplitude, phase).
    """

    kind = 2  # SPINSIM_FIELD_TONES

    def __init__(self, tones, bias=None):
        self.tones = {}
        for c, arr in dict(tones).items():
            arr = np.array(arr, np.float64).reshape(-1, 3)  # a snapshot
            self.tones[_channel_index(c)] = arr
        self.bias = np.zeros(8)
        if bias is not None:
            for c, v in (bias.items() if isinstance(bias, dict) else enumerate(bias)):
                self.bias[_channel_index(c)] = v
        self._cplan()  # the packing plan of the tone snapshots, made once here rather than at each launch

    def packed(self):
        """(flat (w, A, phi) array, start[8], count[8]), computed once (the tones are snapshots)."""
        if "_packed" not in self.__dict__:
            self._packed = self._pack()
        return self._packed

    def _pack(self):
        start = np.zeros(8, np.int32)
        count = np.zeros(8, np.int32)
        rows = []
        n = 0
        for c in range(8):
            arr = self.tones.get(c)
            start[c] = n
            if arr is not None:
                rows.append(arr)
                count[c] = arr.shape[0]
                n += arr.shape[0]
        flat = np.concatenate(rows).reshape(-1) if rows else np.zeros(3)
        return np.ascontiguousarray(flat), start, count

    def device_struct(self, device):
        import torch
        flat, start, count = self.packed()
        td = torch.from_numpy(flat).to(device)
        f = _lib.Field()
        f.tones = td.data_ptr()
        for c in range(8):
            f.tone_start[c] = int(start[c])
            f.tone_count[c] = int(count[c])
            f.bias[c] = self.bias[c]
            f.gain[c] = 1.0
        return f, [td]

    def uses_channel(self, c):
        return c in self.tones or self.bias[c] != 0.0

    def packed_doubles(self):
        """float64 entries in a packed field buffer: the (w, A, phi) rows."""
        return self.packed()[0].size

    def _cplan(self):
        """The field's header row of a ``spinsim_pack_fields`` plan (computed once)."""
        got = self.__dict__.get("_plan")
        if got is None:
            flat, start, count = self.packed()
            self._counts = np.concatenate([start, count]).astype(np.int32)
            header = (2, 0, self.bias.ctypes.data, 0, flat.ctypes.data, flat.size, self._counts.ctypes.data, 0)
            got = self._plan = (np.array([header], np.int64), flat.size, (self.bias, flat, self._counts))
        return got

    def sample(self, t):
        """Host evaluation (for plots and checks): array of shape (len(t), 8)."""
        t = np.atleast_1d(np.asarray(t, np.float64))
        out = np.tile(self.bias, (t.size, 1))
        for c, arr in self.tones.items():
            for w, a, ph in arr:
                out[:, c] += a * np.sin(w * t + ph)
        return out


_TABLE_DOUBLES = 4  # one spinsim_table is 32 bytes
FIELD_DTYPE = np.dtype(_lib.Field)
TABLE_DTYPE = np.dtype(_lib.Table)


def _check_fields(fields):
    types = set(map(type, fields))  # one pass at C level; the per-type checks below are few
    if not all(issubclass(t, (TabulatedField, ToneField)) for t in types) or len({t.kind for t in types}) > 1:
        raise TypeError("packed fields must be built-in fields of one kind")


_CPLAN = methodcaller("_cplan")
_PLAN = attrgetter("_plan")  # set by the built-in fields' constructors


def field_plan(fields):
    """The packing plan of a list of built-in fields of one kind (``spinsim_pack_fields`` rows) and
    the float64 entries the packed buffer takes, in one pass over the fields' cached plans."""
    _check_fields(fields)
    if not fields:
        return np.zeros((0, 8), np.int64), 0
    try:
        cps = list(map(_PLAN, fields))
    except AttributeError:
        cps = list(map(_CPLAN, fields))
    plan = np.concatenate(list(map(itemgetter(0), cps))) if len(cps) > 1 else cps[0][0]
    doubles = sum(map(itemgetter(1), cps))
    if fields[0].kind == TabulatedField.kind:  # eight table descriptors per tabulated field
        doubles += 8 * _TABLE_DOUBLES * len(fields)
    return plan, doubles


def pack_plan_into(plan, n, host, base):
    """``pack_fields_into`` from a ``field_plan`` of n fields."""
    out = np.zeros(n, FIELD_DTYPE)
    if not n:
        return out
    if host.dtype != np.float64 or not host.flags["C_CONTIGUOUS"]:
        raise ValueError("host must be a contiguous float64 array")
    lib = _lib.load()
    used = lib.spinsim_pack_fields(n, plan.ctypes.data, plan.shape[0], host.ctypes.data, host.size, int(base),
                                   out.ctypes.data)
    if used < 0:
        _lib.check(int(used))
    return out


def packed_doubles(fields):
    """float64 entries the fields take in a packed field buffer (``pack_fields_into``): per
    tabulated field eight 4-double table descriptors and its times and amplitudes; per tone field its
    (w, A, phi) rows."""
    _check_fields(fields)
    return sum(f.packed_doubles() for f in fields)


def pack_fields_into(fields, host, base):
    """Write the fields' arrays and table descriptors into ``host`` (a contiguous float64 array of
    at least ``packed_doubles(fields)`` entries) for a device copy of ``host`` at address ``base``;
    returns the ``spinsim_field`` structs as a numpy array of ``FIELD_DTYPE``.  Layout (the library's
    ``spinsim_pack_fields``): the tabulated fields' descriptors first, then every field's arrays."""
    plan, _ = field_plan(fields)
    return pack_plan_into(plan, len(fields), host, base)


# ---------------------------------------------------------------------------- sampler factory
def _sampler_body(time, amplitude, order, zero_boundary):
    """Python source-level sampler (compiled by numba for CUDA or CPU).  Restates the reference's
    find_time_index (I:2026-2061) and sampler bodies (I:2065-2140)."""
    size = time.size
    t_first = time[0]
    t_last = time[size - 1]
    spacing = time[1] - time[0]

    def find_time_index(ts):
        if t_first <= ts and ts <= t_last:
            idx = int((ts - t_first) / spacing)
            low_enough = False
            high_enough = True
            if idx + 1 < size:
                low_enough = time[idx] <= ts
                high_enough = ts <= time[idx + 1]
            else:
                idx = size
            if not (low_enough and high_enough):
                idx_max = size - 1
                idx_min = 0
                budget = size
                while not (low_enough and high_enough):
                    if not low_enough:
                        idx_max = idx
                    else:
                        idx_min = idx
                    idx = int(float(idx_max + idx_min) / 2)
                    low_enough = False
                    high_enough = True
                    if idx + 1 < size:
                        low_enough = time[idx] <= ts
                        high_enough = ts <= time[idx + 1]
                    budget -= 1
                    if budget == 0:
                        return -1, 0.0
            return idx, (ts - time[idx]) / (time[idx + 1] - time[idx])
        return -1, 0.0

    def sampler(ts):
        value = 0.0
        if not zero_boundary:
            if ts <= t_first:
                return amplitude[0]
            if ts >= t_last:
                return amplitude[size - 1]
        i, u = find_time_index(ts)
        if order == 0:
            if i >= 0:
                value = amplitude[i]
            return value
        if not (i >= 0 and i + 1 < size):
            return value
        if order == 1:
            return amplitude[i] * (1 - u) + amplitude[i + 1] * u
        t0 = time[i]
        t1 = time[i + 1]
        g_mid = (amplitude[i + 1] - amplitude[i]) / (t1 - t0) if t0 != t1 else 0.0
        if i == 0:
            g_left = g_mid
        elif time[i - 1] != t0:
            g_left = 0.5 * ((amplitude[i] - amplitude[i - 1]) / (t0 - time[i - 1]) + g_mid)
        else:
            g_left = 0.0
        g_left *= (t1 - t0)
        if i + 2 == size:
            g_right = g_mid
        elif t1 != time[i + 2]:
            g_right = 0.5 * ((amplitude[i + 2] - amplitude[i + 1]) / (time[i + 2] - t1) + g_mid)
        else:
            g_right = 0.0
        g_right *= (t1 - t0)
        u2 = u * u
        u3 = u2 * u
        return (amplitude[i] * (2 * u3 - 3 * u2 + 1) + amplitude[i + 1] * (-2 * u3 + 3 * u2)
                + g_left * (u3 - 2 * u2 + u) + g_right * (u3 - u2))

    return find_time_index, sampler


def generate_interpolation_sampler(time, amplitude, order=3, zero_boundary=True, device=None):
    """The reference's ``generate_interpolation_sampler`` (spinsim/__init__.py:1941).

    Returns ``sampler(time_sample) -> float``: a numba CUDA device function (default) to call from a
    user ``get_field``, or a CPU-jitted function when ``device`` is ``Device.CPU`` /
    ``Device.CPU_SINGLE`` (e.g. for plotting), or plain Python for ``Device.PYTHON``.
    """
    time = np.ascontiguousarray(time, np.float64)
    amplitude = np.ascontiguousarray(amplitude, np.float64)
    if amplitude.ndim == 2:
        raise NotImplementedError("Interpolation sampler does not work with multi-dimensional arrays yet. "
                                  "Try generating a single interpolator for each axis instead.")
    if order not in (0, 1, 3):
        raise NotImplementedError(
            f"Interpolation order {order} is not implemented. Try order 0 (zero order hold), 1 (linear) or 3 (cubic).")
    from . import Device
    device = device or Device.CUDA
    find, samp = _sampler_body(time, amplitude, order, bool(zero_boundary))
    if device == Device.PYTHON:
        return samp
    import numba
    if device in (Device.CPU, Device.CPU_SINGLE):
        find_j = numba.njit(find)
        return numba.njit(_rebind(samp, find_time_index=find_j))
    from numba import cuda
    find_j = cuda.jit(device=True, inline=True)(find)
    return cuda.jit(device=True, inline=True)(_rebind(samp, find_time_index=find_j))


def _rebind(fn, **names):
    """Copy of closure ``fn`` with the free variables in ``names`` replaced."""
    import types
    cells = []
    for name, cell in zip(fn.__code__.co_freevars, fn.__closure__ or ()):
        cells.append(types.CellType(names[name]) if name in names else cell)
    return types.FunctionType(fn.__code__, fn.__globals__, fn.__name__, fn.__defaults__, tuple(cells))


def table_sample(time, amplitude, order, zero_boundary, t):
    """Host evaluation of one table at the times ``t`` (pure Python; for checks and plots)."""
    _, samp = _sampler_body(np.asarray(time, np.float64), np.asarray(amplitude, np.float64), order,
                            bool(zero_boundary))
    return np.array([samp(float(x)) for x in np.ravel(t)])


TAU = 2 * math.pi
