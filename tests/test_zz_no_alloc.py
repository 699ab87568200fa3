"""The allocation-free state propagation entry point (spinsim_state_static).

Some callers of this library may not allocate device memory: a plugin that only receives buffers
from a host application owning every allocation, or a loop that cannot pay cudaMalloc's device-wide
synchronisation.  spinsim_state_static serves them with scratch held inside the library.  This test
calls it through the C ABI twice in a row and checks both results against spinsim_state (which takes
a caller-allocated workspace), within the tolerance of the other scan tests; it also checks that
sizes beyond the stated maximum are rejected.  The file is named to run last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _random_unitaries(n, dim, seed):
    rng = np.random.default_rng(seed)
    a = rng.normal(size=(n, dim, dim)) + 1j * rng.normal(size=(n, dim, dim))
    q, _ = np.linalg.qr(a)
    psi0 = rng.normal(size=dim) + 1j * rng.normal(size=dim)
    return np.ascontiguousarray(q), np.ascontiguousarray(psi0 / np.linalg.norm(psi0))


@pytest.mark.parametrize("dim,n", [(2, 200_000), (3, 262_144), (3, 5)])
def test_static_scratch_state_matches_workspace_state(cuda, dim, n):
    import torch
    from spinsim_b200 import _lib
    lib = _lib.load()
    stream = torch.cuda.current_stream().cuda_stream
    q, psi0 = _random_unitaries(n, dim, seed=dim * 7 + n % 97)
    u = torch.from_numpy(q).to(cuda)
    p0 = psi0.ctypes.data_as(ctypes.c_void_p)

    ref_state = torch.empty((n, dim), dtype=torch.complex128, device=cuda)
    ref_spin = torch.empty((n, 3), dtype=torch.float64, device=cuda)
    ws_bytes = lib.spinsim_state_workspace_size(dim, n)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=cuda)
    _lib.check(lib.spinsim_state(dim, u.data_ptr(), n, p0, ref_state.data_ptr(), ref_spin.data_ptr(),
                                 ws.data_ptr(), ws_bytes, stream))

    for _ in range(2):  # two calls in a row share the library's scratch
        state = torch.full((n, dim), float("nan"), dtype=torch.complex128, device=cuda)
        spin = torch.full((n, 3), float("nan"), dtype=torch.float64, device=cuda)
        _lib.check(lib.spinsim_state_static(dim, u.data_ptr(), n, p0, state.data_ptr(), spin.data_ptr(), stream))
        torch.cuda.synchronize()
        assert (state - ref_state).abs().max().item() < 1e-11
        assert (spin - ref_spin).abs().max().item() < 1e-11


def test_static_scratch_rejects_oversized_input(cuda):
    from spinsim_b200 import _lib
    lib = _lib.load()
    limit = lib.spinsim_state_static_max_steps()
    assert limit == 262_144
    psi0 = np.zeros(3, np.complex128)
    rc = lib.spinsim_state_static(3, 1, limit + 1, psi0.ctypes.data_as(ctypes.c_void_p), 1, None, None)
    assert rc == _lib.ERR_INVALID
    assert "at most" in _lib.last_error()
