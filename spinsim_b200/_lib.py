"""ctypes binding of libspinsim_b200.so (the C ABI declared in include/spinsim_b200.h).

The library is built in-tree by ``spinsim_b200.build``.  There is no CPU fallback: if the library
is missing or fails to load, every entry point raises.
"""
import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("SPINSIM_LIB", os.path.join(HERE, "libspinsim_b200.so"))

OK = 0
ERR_INVALID = -1
ERR_CUDA = -2
ERR_LINK = -3
ERR_UNSUPPORTED = -4
ERR_WORKSPACE = -5

c_i32 = ctypes.c_int32
c_i64 = ctypes.c_int64
c_dbl = ctypes.c_double
c_vp = ctypes.c_void_p


class PlanDesc(ctypes.Structure):
    _fields_ = [("spin_dim", c_i32), ("integration", c_i32), ("expo_half", c_i32), ("expo_one", c_i32),
                ("rotating", c_i32), ("number_of_squares", c_i32), ("field_kind", c_i32), ("precision", c_i32),
                ("threads_per_block", c_i32), ("max_registers", c_i32), ("lanes", c_i32), ("variant", c_i32)]


class Table(ctypes.Structure):
    _fields_ = [("time", c_vp), ("amplitude", c_vp), ("size", c_i64), ("order", c_i32), ("zero_boundary", c_i32)]


class Field(ctypes.Structure):
    _fields_ = [("params", c_vp), ("n_params", c_i64), ("tables", c_vp), ("tones", c_vp),
                ("tone_start", c_i32 * 8), ("tone_count", c_i32 * 8), ("bias", c_dbl * 8), ("gain", c_dbl * 8)]


class Instance(ctypes.Structure):
    _fields_ = [("t0", c_dbl), ("dt_int", c_dbl), ("dt_out", c_dbl), ("n_out", c_i64), ("out_offset", c_i64),
                ("u_offset", c_i64), ("state_offset", c_i64), ("n_fine", c_i32), ("dim", c_i32), ("field", c_i32),
                ("interval0", c_i32), ("psi0", c_dbl * 6)]


class PlanInfo(ctypes.Structure):
    _fields_ = [("registers_per_thread", c_i32), ("threads_per_block", c_i32), ("blocks_per_sm", c_i32),
                ("sm_count", c_i32), ("lanes", c_i32), ("linked", c_i32), ("variant", c_i32),
                ("tile_intervals", c_i32)]


class BatchInfo(ctypes.Structure):
    _fields_ = [("tiles", c_i64), ("scan_tiles", c_i64), ("lanes", c_i32), ("tile_intervals", c_i32),
                ("scan_partials", c_i32), ("reserved", c_i32)]


class SpinsimError(RuntimeError):
    """A failure reported by the CUDA library (message from spinsim_last_error)."""

    def __init__(self, code, message):
        super().__init__(message)
        self.code = code


_lib = None
_lock = threading.Lock()

# (name, restype, argtypes)
_SIGNATURES = [
    ("spinsim_version", ctypes.c_char_p, []),
    ("spinsim_last_error", ctypes.c_int, [ctypes.c_char_p, ctypes.c_size_t]),
    ("spinsim_normalise_steps", ctypes.c_int,
     [c_dbl, c_dbl, c_dbl, c_dbl, ctypes.POINTER(c_dbl), ctypes.POINTER(c_i64), ctypes.POINTER(c_i32),
      ctypes.POINTER(c_i32)]),
    ("spinsim_plan_create", ctypes.c_int, [ctypes.POINTER(PlanDesc), c_vp, ctypes.c_size_t, ctypes.POINTER(c_vp)]),
    ("spinsim_plan_destroy", ctypes.c_int, [c_vp]),
    ("spinsim_plan_get_info", ctypes.c_int, [c_vp, ctypes.POINTER(PlanInfo)]),
    ("spinsim_evaluate_workspace_size", ctypes.c_size_t, [c_vp, c_i64]),
    ("spinsim_evaluate", ctypes.c_int,
     [c_vp, ctypes.POINTER(Field), c_dbl, c_dbl, c_dbl, c_i64, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, ctypes.c_size_t,
      c_vp]),
    ("spinsim_evaluate_with_norms", ctypes.c_int,
     [c_vp, ctypes.POINTER(Field), c_dbl, c_dbl, c_dbl, c_i64, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp,
      ctypes.c_size_t, c_vp]),
    ("spinsim_time_evolution", ctypes.c_int,
     [c_vp, ctypes.POINTER(Field), c_dbl, c_dbl, c_dbl, c_i64, c_vp, c_vp, c_vp, ctypes.c_size_t, c_vp]),
    ("spinsim_state_workspace_size", ctypes.c_size_t, [c_i32, c_i64]),
    ("spinsim_state", ctypes.c_int, [c_i32, c_vp, c_i64, c_vp, c_vp, c_vp, c_vp, ctypes.c_size_t, c_vp]),
    ("spinsim_spin", ctypes.c_int, [c_i32, c_vp, c_i64, c_vp, c_vp]),
    ("spinsim_batch_describe", ctypes.c_int,
     [c_i32, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, ctypes.POINTER(Instance), ctypes.POINTER(c_i64)]),
    ("spinsim_batch_workspace_size", ctypes.c_size_t, [c_vp, ctypes.POINTER(Instance), c_i32, c_i32]),
    ("spinsim_batch_prepare", ctypes.c_int,
     [c_vp, ctypes.POINTER(Instance), c_i32, c_vp, c_i32, c_vp, ctypes.c_size_t, c_vp, ctypes.POINTER(c_vp)]),
    ("spinsim_pack_fields", c_i64, [c_i32, c_vp, c_i64, c_vp, c_i64, ctypes.c_uint64, c_vp]),
    ("spinsim_spin_mean_workspace_size", ctypes.c_size_t, [c_i32, c_i64]),
    ("spinsim_spin_mean", ctypes.c_int, [c_vp, c_i64, c_i64, c_i32, c_i64, c_vp, c_vp, ctypes.c_size_t, c_vp]),
    ("spinsim_piece_product", ctypes.c_int, [c_i32, c_vp, c_i64, c_vp, c_vp, ctypes.c_size_t, c_vp]),
    ("spinsim_piece_states", ctypes.c_int, [c_i32, c_vp, c_i64, c_vp, c_vp, c_vp, c_vp, ctypes.c_size_t, c_vp]),
    ("spinsim_batch_staging_size", ctypes.c_size_t, [c_vp, ctypes.POINTER(Instance), c_i32, c_i32]),
    ("spinsim_batch_prepare_staged", ctypes.c_int,
     [c_vp, ctypes.POINTER(Instance), c_i32, c_vp, c_i32, c_vp, ctypes.c_size_t, c_vp, ctypes.c_size_t, c_vp,
      ctypes.POINTER(c_vp)]),
    ("spinsim_batch_launch", ctypes.c_int, [c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    ("spinsim_batch_destroy", ctypes.c_int, [c_vp]),
    ("spinsim_batch_get_info", ctypes.c_int, [c_vp, ctypes.POINTER(BatchInfo)]),
    ("spinsim_batch_set_step_norms", ctypes.c_int, [c_vp, c_vp]),
    ("spinsim_fma_peak", ctypes.c_int, [c_i32, ctypes.POINTER(c_dbl), c_vp]),
    ("spinsim_state_static_max_steps", c_i64, []),
    ("spinsim_state_static", ctypes.c_int, [c_i32, c_vp, c_i64, c_vp, c_vp, c_vp, c_vp]),
]

EXPORTED = [name for name, _, _ in _SIGNATURES]


def load(path=LIB_PATH):
    """Load (once) and return the library; raises if it is missing."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(path):
            raise ImportError(f"spinsim_b200 CUDA library not built: {path} is missing "
                              "(run `python -m spinsim_b200.build`)")
        lib = ctypes.CDLL(path)
        for name, restype, argtypes in _SIGNATURES:
            fn = getattr(lib, name)
            fn.restype = restype
            fn.argtypes = argtypes
        _lib = lib
        return lib


def last_error():
    buf = ctypes.create_string_buffer(1024)
    load().spinsim_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(rc):
    if rc != OK:
        msg = last_error()
        if rc == ERR_INVALID or rc == ERR_WORKSPACE:
            raise ValueError(msg)
        if rc == ERR_UNSUPPORTED:
            raise NotImplementedError(msg)
        raise SpinsimError(rc, msg)
    return rc


def normalise_steps(t0, t1, dt_int, dt_out):
    """(dt_int', N, K, warned) of Simulator.evaluate's step normalisation (spinsim/__init__.py:1025-1034)."""
    d = c_dbl()
    n = c_i64()
    k = c_i32()
    w = c_i32()
    check(load().spinsim_normalise_steps(float(t0), float(t1), float(dt_int), float(dt_out), ctypes.byref(d),
                                         ctypes.byref(n), ctypes.byref(k), ctypes.byref(w)))
    return d.value, n.value, k.value, bool(w.value)
