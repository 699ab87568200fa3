"""Single-instance entry points are stream-ordered and capturable: spinsim_state and spinsim_evaluate
take their instance, field and scan tiles as launch arguments (no host-to-device copy), so a CUDA
graph captured around them replays the same launches on whatever the device buffers hold at replay
time.  Also: the allocation-free state scan and the on-device ensemble mean checked directly against
the oracle."""
import ctypes

import numpy as np
import pytest

import fields as F
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _unitaries(n, dim, seed):
    rng = np.random.default_rng(seed)
    a = rng.normal(size=(n, dim, dim)) + 1j * rng.normal(size=(n, dim, dim))
    q, _ = np.linalg.qr(a)
    psi0 = rng.normal(size=dim) + 1j * rng.normal(size=dim)
    return np.ascontiguousarray(q), np.ascontiguousarray(psi0 / np.linalg.norm(psi0))


@pytest.mark.parametrize("dim", [2, 3])
def test_state_scan_captured_in_a_cuda_graph(cuda, dim):
    import torch
    from spinsim_b200 import _lib
    lib = _lib.load()
    n = 5000
    q1, psi0 = _unitaries(n, dim, seed=1)
    q2, _ = _unitaries(n, dim, seed=2)
    u = torch.from_numpy(q1).to(cuda)
    state = torch.empty((n, dim), dtype=torch.complex128, device=cuda)
    spin = torch.empty((n, 3), dtype=torch.float64, device=cuda)
    ws_bytes = lib.spinsim_state_workspace_size(dim, n)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=cuda)
    p0 = psi0.ctypes.data_as(ctypes.c_void_p)

    graph = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        with torch.cuda.graph(graph, stream=side):
            _lib.check(lib.spinsim_state(dim, u.data_ptr(), n, p0, state.data_ptr(), spin.data_ptr(),
                                         ws.data_ptr(), ws_bytes, side.cuda_stream))
    torch.cuda.synchronize()
    for q in (q1, q2):  # new operators in the same buffer, then replay
        u.copy_(torch.from_numpy(q))
        state.fill_(float("nan"))
        graph.replay()
        torch.cuda.synchronize()
        ref = O.state(q, psi0)
        assert np.abs(state.cpu().numpy() - ref).max() < 1e-11
        assert np.abs(spin.cpu().numpy() - O.spin(ref)).max() < 1e-11


def test_evaluate_captured_in_a_cuda_graph(cuda):
    """spinsim_evaluate with a user field (the detuned spin-one Rabi drive) captured once; replays
    with new sweep parameters in the captured device buffer match direct evaluations and the oracle."""
    import torch
    import spinsim_b200 as ss
    from spinsim_b200 import _lib
    sim = ss.Simulator(F.detuned_rabi, ss.SpinQuantumNumber.ONE, ss.IntegrationMethod.MAGNUS_CF4,
                       ss.ExponentiationMethod.LIE_TROTTER, True, 28)
    t0, t1, dti, dto = 0.0, 400e-6, 10e-9, 100e-9
    psi0 = np.ascontiguousarray(ss.SpinQuantumNumber.ONE.plus_z, np.complex128)
    dt_int, n, _, _ = _lib.normalise_steps(t0, t1, dti, dto)
    sweep = torch.tensor([1500.0], dtype=torch.float64, device=cuda)
    time = torch.empty(n, dtype=torch.float64, device=cuda)
    u = torch.empty((n, 3, 3), dtype=torch.complex128, device=cuda)
    state = torch.empty((n, 3), dtype=torch.complex128, device=cuda)
    spin = torch.empty((n, 3), dtype=torch.float64, device=cuda)
    ws_bytes = sim._lib.spinsim_evaluate_workspace_size(sim._plan, n)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=cuda)
    field = sim._field_struct(sweep)
    graph = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        with torch.cuda.graph(graph, stream=side):
            _lib.check(sim._lib.spinsim_evaluate(
                sim._plan, ctypes.byref(field), t0, float(dt_int), dto, n, psi0.ctypes.data_as(ctypes.c_void_p),
                time.data_ptr(), u.data_ptr(), state.data_ptr(), spin.data_ptr(), ws.data_ptr(), ws_bytes,
                side.cuda_stream))
    torch.cuda.synchronize()
    for delta in (1500.0, -3200.0):
        sweep.fill_(delta)
        graph.replay()
        torch.cuda.synchronize()
        direct = sim.evaluate(t0, t1, dti, dto, psi0, [delta])
        assert np.array_equal(state.cpu().numpy(), direct.state)
        assert np.array_equal(u.cpu().numpy(), direct.time_evolution)
        tt, uu, st, sp = O.evaluate(3, O.Field(4), [delta], t0, t1, dti, dto, psi0, expo="lie_trotter", n_squares=28)
        assert np.abs(state.cpu().numpy() - st).max() < 1e-10


@pytest.mark.parametrize("dim,n", [(2, 1000), (3, 70_001)])
def test_static_scratch_state_matches_oracle(cuda, dim, n):
    import torch
    from spinsim_b200 import _lib
    lib = _lib.load()
    q, psi0 = _unitaries(n, dim, seed=5 + dim)
    u = torch.from_numpy(q).to(cuda)
    state = torch.empty((n, dim), dtype=torch.complex128, device=cuda)
    spin = torch.empty((n, 3), dtype=torch.float64, device=cuda)
    _lib.check(lib.spinsim_state_static(dim, u.data_ptr(), n, psi0.ctypes.data_as(ctypes.c_void_p),
                                        state.data_ptr(), spin.data_ptr(), torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    ref = O.state(q, psi0)
    assert np.abs(state.cpu().numpy() - ref).max() < 1e-11
    assert np.abs(spin.cpu().numpy() - O.spin(ref)).max() < 1e-11


def test_ensemble_spin_mean_matches_oracle(cuda):
    """The on-device ensemble mean of the Gaussian-pulse members against the mean of the oracle's
    spins (each member evaluated by the oracle)."""
    import spinsim_b200 as ss
    import spinsim_b200.batch as B
    members = np.random.default_rng(seed=2).normal(0.0, 500.0, 24)
    half = ss.SpinQuantumNumber.HALF
    insts = [B.Instance(half, 0.0, 200e-6, 20e-9, 1e-6, half.plus_z, sweep_parameters=[m]) for m in members]
    b = B.Batch(insts, get_field=F.gaussian_ensemble)
    b.run()
    mean = b.spin_mean().cpu().numpy()
    ref = np.mean([O.evaluate(2, O.Field(5), [m], 0.0, 200e-6, 20e-9, 1e-6, half.plus_z)[3] for m in members], axis=0)
    assert mean.shape == ref.shape == (200, 3)
    assert np.abs(mean - ref).max() < 1e-10
