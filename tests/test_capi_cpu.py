"""The C ABI library without a GPU: it loads, exports every entry point of include/*.h, and its
host logic (step normalisation, workspace sizing, argument checks) follows the reference."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

from spinsim_b200 import _lib
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(spinsim_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_library_loads_and_exports_every_header_symbol():
    lib = _lib.load()
    declared = header_functions()
    assert len(declared) >= 15
    for name in declared:
        assert hasattr(lib, name), f"{name} declared in include/ but not exported"
    assert set(declared) <= set(_lib.EXPORTED) | set(declared)
    assert b"sm_100a" in lib.spinsim_version()


@pytest.mark.parametrize("t0,t1,dti,dto", [
    (0, 0.1, 100e-9, 500e-9), (0, 10e-3, 10e-9, 100e-9), (0, 1e-3, 20e-9, 1e-6), (1e-3, 1.2e-3, 100e-9, 1e-6),
    (0, 1e-3, 3e-7, 1e-6), (0, 1e-3, 2e-6, 1e-6), (-5.0, 7.0, 0.01, 2.0), (0, 0.5e-6, 100e-9, 1e-6),
    (0, 1e-3, 0.4e-6, 1e-6), (0, 1e-3, 2.5e-7, 1e-6)])
def test_normalise_steps_matches_reference(t0, t1, dti, dto):
    """I:1025-1034 (Python round() is half-to-even: dt_out/dt_int = 2.5 rounds to 2)."""
    a = _lib.normalise_steps(t0, t1, dti, dto)
    b = O.normalise_steps(t0, t1, dti, dto)
    assert a[0] == b[0] and a[1] == b[1] and a[2] == b[2] and a[3] == b[3]


def test_invalid_arguments_raise():
    with pytest.raises(ValueError):
        _lib.normalise_steps(0, 1, 0.0, 1e-6)
    lib = _lib.load()
    plan = ctypes.c_void_p()
    desc = _lib.PlanDesc()
    desc.spin_dim = 5
    rc = lib.spinsim_plan_create(ctypes.byref(desc), None, 0, ctypes.byref(plan))
    assert rc == _lib.ERR_INVALID and "spin_dim" in _lib.last_error()
    desc.spin_dim = 2
    desc.expo_half = 2  # eight-generator exponential on spin half
    rc = lib.spinsim_plan_create(ctypes.byref(desc), None, 0, ctypes.byref(plan))
    assert rc == _lib.ERR_INVALID
    desc.expo_half = 0
    desc.field_kind = 0  # user field without LTO-IR
    rc = lib.spinsim_plan_create(ctypes.byref(desc), None, 0, ctypes.byref(plan))
    assert rc == _lib.ERR_INVALID and "field_ltoir" in _lib.last_error()


def test_workspace_sizes():
    lib = _lib.load()
    assert lib.spinsim_state_workspace_size(2, 0) > 0
    a = lib.spinsim_state_workspace_size(2, 200_000)
    b = lib.spinsim_state_workspace_size(3, 200_000)
    assert 0 < a <= b
    assert lib.spinsim_state_workspace_size(4, 10) == 0
    # two stored operators (tile product and prefix, 3 x 3 complex slots) per scan tile of 32 steps
    assert a >= (200_000 // 32) * 2 * 144
    assert lib.spinsim_state_workspace_size(2, 33) > lib.spinsim_state_workspace_size(2, 32)
    # the fixed scratch of spinsim_state_static holds the scan of its largest input
    assert lib.spinsim_state_workspace_size(3, lib.spinsim_state_static_max_steps()) <= 5 << 20


def test_state_entry_points_check_arguments_without_a_gpu():
    lib = _lib.load()
    psi = np.zeros(4)
    rc = lib.spinsim_state(2, None, 10, psi.ctypes.data_as(ctypes.c_void_p), None, None, None, 0, None)
    assert rc == _lib.ERR_INVALID
    assert lib.spinsim_state(2, None, 0, None, None, None, None, 0, None) == _lib.OK  # empty is a no-op
    assert lib.spinsim_spin(7, None, 1, None, None) == _lib.ERR_INVALID
