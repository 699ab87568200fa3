"""Python side of the oracle: the reference's evaluate() host logic around the C restatement.

TEST INFRASTRUCTURE ONLY.  Imported by tests/, by ``__graft_entry__.smoke()`` (as the checker) and
by bench.py's CPU-baseline leg.  The product package ``spinsim_b200`` never imports it.

``evaluate`` restates Simulator.evaluate (spinsim/__init__.py:993-1085): the integration-step
normalisation (I:1025-1028), N = int((t1 - t0) / dt_out) (I:1034), the time-evolution call
(I:1043), get_state (I:1081-1082) and the spin calculation (I:961-988).
"""
import ctypes
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libspinsim_oracle.so")

INTEG = {"magnus_cf4": 0, "euler": 1, "heun": 2}
EXPO = {"analytic": 0, "lie_trotter": 1, "lie_trotter_8": 2}


class _Config(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("integration", ctypes.c_int), ("expo", ctypes.c_int),
                ("rotating", ctypes.c_int), ("n_squares", ctypes.c_int)]


class _Table(ctypes.Structure):
    _fields_ = [("time", ctypes.POINTER(ctypes.c_double)), ("amplitude", ctypes.POINTER(ctypes.c_double)),
                ("size", ctypes.c_int64), ("order", ctypes.c_int), ("zero_boundary", ctypes.c_int)]


class _Field(ctypes.Structure):
    _fields_ = [("code", ctypes.c_int), ("tables", ctypes.POINTER(_Table)), ("n_tables", ctypes.c_int)]


def build():
    """Compile the C restatement (make -C oracle)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = ctypes.CDLL(LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        _lib.oracle_time_evolution.argtypes = [ctypes.POINTER(_Config), ctypes.POINTER(_Field), dp, ctypes.c_int64,
                                               ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int64,
                                               ctypes.c_int64, ctypes.c_int64, dp, dp, ctypes.c_int]
        _lib.oracle_time_evolution.restype = ctypes.c_int
        _lib.oracle_state.argtypes = [ctypes.c_int, dp, dp, ctypes.c_int64, dp]
        _lib.oracle_spin.argtypes = [ctypes.c_int, dp, ctypes.c_int64, dp]
        _lib.oracle_interpolate.argtypes = [ctypes.POINTER(_Table), ctypes.c_double]
        _lib.oracle_interpolate.restype = ctypes.c_double
        _lib.oracle_max_threads.restype = ctypes.c_int
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Field:
    """A field for the oracle: an integer code of tests/golden/fields.py plus optional tables.

    ``tables``: list of (time, amplitude, order, zero_boundary) for the tabulated code (9)."""

    def __init__(self, code, tables=None):
        self.code = code
        self._keep = []
        self.tables = None
        n = 0
        if tables:
            n = len(tables)
            arr = (_Table * n)()
            for i, (t, a, order, zb) in enumerate(tables):
                t = np.ascontiguousarray(t, np.float64)
                a = np.ascontiguousarray(a, np.float64)
                self._keep += [t, a]
                arr[i] = _Table(_dp(t), _dp(a), t.size, int(order), int(bool(zb)))
            self.tables = arr
            self._keep.append(arr)
        self.struct = _Field(code, self.tables if self.tables is not None else None, n)


def resolve_expo(spin_dim, expo):
    """Default exponentiator (I:529-533) and the analytic-on-spin-one switch (I:556-559)."""
    if expo is None:
        expo = "analytic" if spin_dim == 2 else "lie_trotter"
    if expo == "analytic" and spin_dim == 3:
        expo = "lie_trotter"
    return expo


def normalise_steps(t0, t1, dt_int, dt_out):
    """I:1025-1034: returns (dt_int', N, K, warned)."""
    old = dt_int
    dt_int = dt_out / round(max(dt_out / dt_int, 1))
    warned = math.fabs(dt_out / old - round(dt_out / old)) > 1e-6
    n = int((np.float64(t1) - np.float64(t0)) / dt_out)
    k = math.floor(dt_out / dt_int + 0.5)
    return dt_int, n, k, warned


def time_evolution(spin_dim, field, sweep, t0, dt_int, dt_out, n, integration="magnus_cf4", expo=None,
                   rotating=True, n_squares=24, first=0, count=None, n_threads=0):
    """get_time_evolution over output intervals [first, first + count) of an N-interval run."""
    expo = resolve_expo(spin_dim, expo)
    cfg = _Config(spin_dim, INTEG[integration], EXPO[expo], int(bool(rotating)), int(n_squares))
    sweep = np.ascontiguousarray(sweep, np.float64).reshape(-1)
    if sweep.size == 0:
        sweep = np.zeros(1)
    count = n - first if count is None else count
    time = np.zeros(n, np.float64)
    u = np.zeros((n, spin_dim, spin_dim), np.complex128)
    rc = lib().oracle_time_evolution(ctypes.byref(cfg), ctypes.byref(field.struct), _dp(sweep), sweep.size,
                                     float(t0), float(dt_int), float(dt_out), int(n), int(first), int(count),
                                     _dp(time), _dp(u.view(np.float64)), int(n_threads))
    if rc != 0:
        raise ValueError("oracle_time_evolution rejected its arguments")
    return time, u


def state(u, psi0):
    n, d = u.shape[0], u.shape[1]
    u = np.ascontiguousarray(u, np.complex128)
    psi0 = np.ascontiguousarray(psi0, np.complex128)
    out = np.zeros((n, d), np.complex128)
    lib().oracle_state(d, _dp(u.view(np.float64)), _dp(psi0.view(np.float64)), n, _dp(out.view(np.float64)))
    return out


def spin(st):
    st = np.ascontiguousarray(st, np.complex128)
    n, d = st.shape
    out = np.zeros((n, 3), np.float64)
    lib().oracle_spin(d, _dp(st.view(np.float64)), n, _dp(out))
    return out


def evaluate(spin_dim, field, sweep, t0, t1, dt_int, dt_out, psi0, integration="magnus_cf4", expo=None,
             rotating=True, n_squares=24, n_threads=0):
    """The reference's evaluate(): returns (time, time_evolution, state, spin)."""
    dt_int, n, _, _ = normalise_steps(t0, t1, dt_int, dt_out)
    time, u = time_evolution(spin_dim, field, sweep, t0, dt_int, dt_out, n, integration, expo, rotating, n_squares,
                             n_threads=n_threads)
    st = state(u, psi0)
    return time, u, st, spin(st)


def interpolate(time, amplitude, order, zero_boundary, t):
    """The reference's interpolation sampler (I:1941-2147) evaluated at the times in ``t``."""
    time = np.ascontiguousarray(time, np.float64)
    amplitude = np.ascontiguousarray(amplitude, np.float64)
    tb = _Table(_dp(time), _dp(amplitude), time.size, int(order), int(bool(zero_boundary)))
    return np.array([lib().oracle_interpolate(ctypes.byref(tb), float(x)) for x in np.ravel(t)])


def max_threads():
    return lib().oracle_max_threads()
