"""Batched persistent launches: a mixed spin-half / spin-one batch with uneven durations against the
oracle, and alone-vs-in-the-mix identity."""
import numpy as np
import pytest

import fields as F
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def tone_field(p):
    import spinsim_b200 as ss
    tones = {a: np.array([(p[4 + 24 * a + 3 * k], p[5 + 24 * a + 3 * k], p[6 + 24 * a + 3 * k]) for k in range(8)])
             for a in range(3)}
    return ss.ToneField(tones, bias=list(p[:4]))


def make_instances(n, seed=3, max_duration=200e-6):
    import spinsim_b200 as ss
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        spin = ss.SpinQuantumNumber.HALF if rng.uniform() < 0.7 else ss.SpinQuantumNumber.ONE
        dur = float(np.exp(rng.uniform(np.log(10e-6), np.log(max_duration))))
        p = F.tone_parameters(np.random.default_rng(1000 + k))
        out.append(ss.batch.Instance(spin, 0.0, dur, 10e-9, 1e-6, spin.plus_z if spin.dimension == 2 else spin.plus_x,
                                     sweep_parameters=p, field=tone_field(p)))
    return out


def test_mixed_batch_matches_oracle(cuda):
    import spinsim_b200.batch as B
    insts = make_instances(24)
    b = B.Batch(insts)
    b.run()
    for k, inst in enumerate(insts):
        r = b.result(k)
        d = inst.spin.dimension
        t, u, s, sp = O.evaluate(d, O.Field(8), inst.sweep_parameters, inst.time_start, inst.time_end,
                                 inst.time_step_integration, inst.time_step_output, inst.state_init)
        assert np.array_equal(r.time, t)
        assert np.abs(r.time_evolution - u).max() < 1e-10
        assert np.abs(r.state - s).max() < 1e-10
        assert np.abs(r.spin - sp).max() < 1e-10


def test_user_field_batch_matches_oracle(cuda):
    """One user get_field shared by the batch, per-instance sweep parameters."""
    import spinsim_b200 as ss
    import spinsim_b200.batch as B
    members = np.random.default_rng(seed=2).normal(0.0, 500.0, 16)
    insts = [B.Instance(ss.SpinQuantumNumber.HALF, 0.0, 100e-6, 20e-9, 1e-6, ss.SpinQuantumNumber.HALF.plus_z,
                        sweep_parameters=[m]) for m in members]
    b = B.Batch(insts, get_field=F.gaussian_ensemble)
    b.run()
    for k, m in enumerate(members):
        t, u, s, sp = O.evaluate(2, O.Field(5), [m], 0.0, 100e-6, 20e-9, 1e-6, ss.SpinQuantumNumber.HALF.plus_z)
        r = b.result(k)
        assert np.abs(r.state - s).max() < 1e-10


def test_result_alone_equals_result_in_mix(cuda):
    """Per-instance arithmetic does not depend on what else runs in the launch."""
    import spinsim_b200.batch as B
    insts = make_instances(16, seed=5)
    mix = B.Batch(insts, lanes=1)
    mix.run()
    for k in (0, 7, 15):
        alone = B.Batch([insts[k]], lanes=1)
        alone.run()
        a, m = alone.result(0), mix.result(k)
        assert np.array_equal(a.time_evolution, m.time_evolution)
        assert np.array_equal(a.state, m.state)


def test_graph_replay_reproduces(cuda):
    import torch
    import spinsim_b200.batch as B
    insts = make_instances(8, seed=9)
    b = B.Batch(insts)
    b.run()
    torch.cuda.synchronize()
    first = b.state.clone()
    b.state.zero_()
    b.capture()
    b.replay()
    torch.cuda.synchronize()
    assert torch.equal(first, b.state)


def final_state_errors(a, b):
    return np.array([np.abs(x - y).max() if x.size else 0.0 for x, y in zip(a.final_states(), b.final_states())])


@pytest.mark.parametrize("variant", [0, 1])
def test_fp32_bulk_tones_error_vs_fp64(cuda, variant):
    """The batched FP32-bulk form (tensor-path kernel, variant 0, and warp synthesis, variant 1)
    against the plain FP64 form: final-state error <= 1e-6 (uneven spin-half / spin-one tone batch,
    durations up to 2 ms)."""
    import spinsim_b200 as ss
    import spinsim_b200.batch as B
    insts = make_instances(64, seed=11, max_duration=2e-3)
    plans = {}
    bulk = B.Batch(insts, precision=ss.Precision.FP32_BULK, plan_cache=plans, variant=variant)
    assert bulk.plan_info()["variant"] == variant
    plain = B.Batch(insts, precision=ss.Precision.FP64, plan_cache=plans)
    bulk.run()
    plain.run()
    errs = final_state_errors(bulk, plain)
    assert errs.max() < 1e-6, errs.max()
    du = (bulk.u - plain.u).abs().max().item()
    assert du < 1e-8, du


def test_fp32_bulk_quadratic_shift_and_lie_trotter_half(cuda):
    """Spin one with a quadratic shift (Taylor-series exponential) and spin half with the
    Lie-Trotter exponentiator selected, against FP64."""
    import spinsim_b200 as ss
    import spinsim_b200.batch as B
    rng = np.random.default_rng(21)
    insts = []
    for k in range(12):
        spin = ss.SpinQuantumNumber.ONE
        p = F.tone_parameters(np.random.default_rng(500 + k))
        fld = tone_field(p)
        fld.bias[3] = ss.fields.TAU * rng.uniform(-20e3, 20e3)
        fld.tones[3] = np.array([(ss.fields.TAU * 3e5, ss.fields.TAU * 5e3, 0.3)])
        insts.append(B.Instance(spin, 0.0, 500e-6, 10e-9, 1e-6, spin.plus_x, field=fld))
    plans = {}
    bulk = B.Batch(insts, precision=ss.Precision.FP32_BULK, plan_cache=plans)
    plain = B.Batch(insts, precision=ss.Precision.FP64, plan_cache=plans)
    bulk.run()
    plain.run()
    assert final_state_errors(bulk, plain).max() < 1e-6
    half = make_instances(24, seed=4, max_duration=1e-3)
    half = [i for i in half if i.spin.dimension == 2]
    bulk = B.Batch(half, precision=ss.Precision.FP32_BULK, exponentiation_half=ss.ExponentiationMethod.LIE_TROTTER)
    plain = B.Batch(half, precision=ss.Precision.FP64, exponentiation_half=ss.ExponentiationMethod.LIE_TROTTER)
    bulk.run()
    plain.run()
    assert final_state_errors(bulk, plain).max() < 1e-6


def test_fp32_bulk_gaussian_ensemble_members(cuda):
    """Spin-half Gaussian-pulse ensemble (user field) in FP32-bulk, per-member error against FP64."""
    import spinsim_b200 as ss
    import spinsim_b200.batch as B
    members = np.random.default_rng(seed=2).normal(0.0, 500.0, 256)
    insts = [B.Instance(ss.SpinQuantumNumber.HALF, 0.0, 1e-3, 20e-9, 1e-6, ss.SpinQuantumNumber.HALF.plus_z,
                        sweep_parameters=[m]) for m in members]
    bulk = B.Batch(insts, get_field=F.gaussian_ensemble, precision=ss.Precision.FP32_BULK)
    plain = B.Batch(insts, get_field=F.gaussian_ensemble, precision=ss.Precision.FP64)
    bulk.run()
    plain.run()
    errs = final_state_errors(bulk, plain)
    assert errs.max() < 1e-6, errs.max()


def test_fp32_bulk_simulator_single_instance(cuda):
    import spinsim_b200 as ss
    sim32 = ss.Simulator(F.detuned_rabi, ss.SpinQuantumNumber.ONE, precision=ss.Precision.FP32_BULK)
    sim64 = ss.Simulator(F.detuned_rabi, ss.SpinQuantumNumber.ONE)
    a = sim32.evaluate(0, 1e-3, 10e-9, 100e-9, ss.SpinQuantumNumber.ONE.plus_z, [250.0])
    b = sim64.evaluate(0, 1e-3, 10e-9, 100e-9, ss.SpinQuantumNumber.ONE.plus_z, [250.0])
    assert np.abs(a.state - b.state).max() < 1e-6


@pytest.mark.parametrize("chunks", [1, 3, 5])
def test_evaluator_to_host_equals_batch(cuda, chunks):
    """The overlapped host path (staged uploads, per-chunk launches, copies on a second stream) gives
    the batch's results bit for bit."""
    import torch
    import spinsim_b200.batch as B
    insts = make_instances(40, seed=12, max_duration=300e-6)
    ref = B.Batch(insts, lanes=1, force_mixed=True)
    ref.run()
    torch.cuda.synchronize()
    ev = B.Evaluator(chunks=chunks, lanes=1, force_mixed=True)
    res = ev.evaluate(insts)
    assert len(res) == len(insts)
    # one copy per group of its time, U, state and spin pieces, with the alignment gaps between them
    tensor_bytes = sum(t.numel() * t.element_size() for t in (ref.time, ref.u, ref.state, ref.spin))
    assert tensor_bytes <= ev.d2h_bytes <= tensor_bytes + 3 * 256 * chunks
    for k in range(len(insts)):
        r = ref.result(k)
        for name in ("time", "time_evolution", "state", "spin"):
            assert np.array_equal(getattr(res[k], name), getattr(r, name)), (k, name)


def test_evaluator_default_split_agrees_to_rounding(cuda):
    import spinsim_b200.batch as B
    insts = make_instances(30, seed=14, max_duration=300e-6)
    ref = B.Batch(insts)
    ref.run()
    res = B.evaluate_many(insts, chunks=4)
    for k in range(len(insts)):
        assert np.abs(res[k].state - ref.result(k).state).max() < 1e-12


def test_staged_batch_equals_pageable_batch(cuda):
    import torch
    import spinsim_b200.batch as B
    insts = make_instances(12, seed=13)
    plain = B.Batch(insts)
    staged = B.Batch(insts, staging=lambda n: torch.empty(n, dtype=torch.uint8, pin_memory=True))
    assert staged._staging is not None
    plain.run()
    staged.run()
    torch.cuda.synchronize()
    assert torch.equal(plain.u, staged.u) and torch.equal(plain.state, staged.state)


def test_evaluate_many_user_field(cuda):
    import spinsim_b200 as ss
    import spinsim_b200.batch as B
    members = np.random.default_rng(seed=4).normal(0.0, 500.0, 9)
    insts = [B.Instance(ss.SpinQuantumNumber.HALF, 0.0, 50e-6, 20e-9, 1e-6, ss.SpinQuantumNumber.HALF.plus_z,
                        sweep_parameters=[m]) for m in members]
    res = B.evaluate_many(insts, chunks=2, get_field=F.gaussian_ensemble)
    for m, r in zip(members, res):
        t, u, s, sp = O.evaluate(2, O.Field(5), [m], 0.0, 50e-6, 20e-9, 1e-6, ss.SpinQuantumNumber.HALF.plus_z)
        assert np.abs(r.state - s).max() < 1e-10


def test_ensemble_spin_mean_on_device(cuda):
    """The Gaussian-pulse ensemble's mean spin reduced on the device equals the host mean of the
    members' spins; final states gathered on the device equal the slices of the full state."""
    import torch
    import spinsim_b200 as ss
    import spinsim_b200.batch as B
    members = np.random.default_rng(seed=2).normal(0.0, 500.0, 200)
    insts = [B.Instance(ss.SpinQuantumNumber.HALF, 0.0, 300e-6, 20e-9, 1e-6, ss.SpinQuantumNumber.HALF.plus_z,
                        sweep_parameters=[m]) for m in members]
    b = B.Batch(insts, get_field=F.gaussian_ensemble)
    b.run()
    mean = b.spin_mean().cpu().numpy()
    host = np.mean([b.result(k).spin for k in range(len(insts))], axis=0)
    assert mean.shape == host.shape == (300, 3)
    assert np.abs(mean - host).max() < 1e-13
    part = b.spin_mean(10, 50).cpu().numpy()
    assert np.abs(part - np.mean([b.result(k).spin for k in range(10, 60)], axis=0)).max() < 1e-13
    finals = b.final_states()
    for k in (0, 7, 199):
        assert np.array_equal(finals[k], b.result(k).state[-1])
    # zero-copy interop: the device arrays export through DLPack without a copy
    st = b.result(3).device_arrays["state"]
    again = torch.from_dlpack(st)
    assert again.data_ptr() == st.data_ptr()


def test_spin_mean_rejects_unequal_members(cuda):
    import spinsim_b200.batch as B
    insts = make_instances(6, seed=41)
    b = B.Batch(insts)
    b.run()
    with pytest.raises(ValueError):
        b.spin_mean()


def test_tensor_path_step_counts_and_tile_edges(cuda):
    """The tensor-path tone kernel with every split of K fine steps over its four time segments
    (K = 1 .. 9, 33, 100, 137: empty and uneven segments) and instance lengths that end inside a
    CTA tile or a warp's rows, against the oracle and the warp-synthesis kernel."""
    import spinsim_b200 as ss
    import spinsim_b200.batch as B
    H, O1 = ss.SpinQuantumNumber.HALF, ss.SpinQuantumNumber.ONE
    specs = []
    for j, k in enumerate([1, 2, 3, 4, 5, 6, 7, 8, 9, 33, 100, 137]):
        n = [1, 7, 8, 9, 31, 32, 33, 40, 65, 3, 12, 20][j]
        specs.append((H if j % 3 else O1, 0.25e-6 * j, 0.25e-6 * j + n * 1e-6, 1e-6 / k, 1e-6))
    insts = []
    for j, (s, t0, t1, dti, dto) in enumerate(specs):
        p = F.tone_parameters(np.random.default_rng(900 + j))
        insts.append(B.Instance(s, t0, t1, dti, dto, s.plus_x, sweep_parameters=p, field=tone_field(p)))
    plans = {}
    tensor = B.Batch(insts, precision=ss.Precision.FP32_BULK, plan_cache=plans, variant=0)
    synth = B.Batch(insts, precision=ss.Precision.FP32_BULK, plan_cache=plans, variant=1)
    tensor.run()
    synth.run()
    for k, (s, t0, t1, dti, dto) in enumerate(specs):
        r, r1 = tensor.result(k), synth.result(k)
        t, u, st, sp = O.evaluate(s.dimension, O.Field(8), insts[k].sweep_parameters, t0, t1, dti, dto, s.plus_x)
        assert np.array_equal(r.time, t)
        assert np.abs(r.time_evolution - u).max() < 1e-7, k
        assert np.abs(r.state - st).max() < 1e-6, k
        assert np.abs(r.state - r1.state).max() < 1e-6, k


def _operator_scan(u, psi0):
    """The state scan of the given operators through spinsim_state (the tile products kernels)."""
    import ctypes
    import torch
    from spinsim_b200 import _lib
    lib = _lib.load()
    n, dim = u.shape[0], u.shape[1]
    ud = torch.from_numpy(np.ascontiguousarray(u)).cuda()
    state = torch.empty((n, dim), dtype=torch.complex128, device="cuda")
    ws_bytes = lib.spinsim_state_workspace_size(dim, n)
    ws = torch.empty(max(ws_bytes, 1), dtype=torch.uint8, device="cuda")
    p0 = np.ascontiguousarray(psi0, dtype=np.complex128)
    _lib.check(lib.spinsim_state(dim, ud.data_ptr(), n, p0.ctypes.data_as(ctypes.c_void_p), state.data_ptr(), None,
                                 ws.data_ptr(), ws_bytes, torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return state.cpu().numpy()


def test_tensor_path_partials_scan_equals_operator_scan(cuda):
    """On the tensor path the time evolution writes each scan tile's warp partials (SU(2) pairs) and
    the scan skips its tile products: the states equal the scan of the returned operators through
    spinsim_state to FP64 rounding, for tiles that end inside a warp's rows, instances of more than
    one prefix chunk (32 tiles) and both spins, in a batch and in single Simulator calls."""
    import spinsim_b200 as ss
    import spinsim_b200.batch as B
    H, O1 = ss.SpinQuantumNumber.HALF, ss.SpinQuantumNumber.ONE
    lengths = [1, 5, 8, 9, 31, 32, 33, 100, 1023, 1024, 1025, 2100]
    insts = []
    for j, n in enumerate(lengths):
        s = H if j % 3 else O1
        p = F.tone_parameters(np.random.default_rng(1300 + j))
        insts.append(B.Instance(s, 0.0, n * 1e-6, 50e-9, 1e-6, s.plus_x, sweep_parameters=p, field=tone_field(p)))
    b = B.Batch(insts, precision=ss.Precision.FP32_BULK, variant=0)
    info = b.launch_info()
    assert info["variant"] == 0 and info["scan_partials"] == 1
    b.run()
    for k, inst in enumerate(insts):
        r = b.result(k)
        assert r.state.shape[0] == lengths[k]
        ref = _operator_scan(r.time_evolution, inst.spin.plus_x)
        assert np.abs(r.state - ref).max() < 1e-12, k
    plain = B.Batch(insts[:4], precision=ss.Precision.FP64)
    assert plain.launch_info()["scan_partials"] == 0
    plain.run()
    for k in range(4):
        r = plain.result(k)
        assert np.abs(r.state - _operator_scan(r.time_evolution, insts[k].spin.plus_x)).max() < 1e-12, k
    for j, s in enumerate([H, O1]):
        p = F.tone_parameters(np.random.default_rng(1400 + j))
        sim = ss.Simulator(tone_field(p), s, precision=ss.Precision.FP32_BULK)
        r = sim.evaluate(0.0, 1500e-6, 50e-9, 1e-6, s.plus_x)
        ref = _operator_scan(r.time_evolution, s.plus_x)
        assert np.abs(r.state - ref).max() < 1e-12, s


def test_ragged_batch_edge_instances(cuda):
    """A batch mixing an empty instance (t1 == t0), a single output step, K = 1 (dt_int = dt_out), a
    non-integer step ratio (dt_int reset as the reference does) and fewer steps than a warp, against
    the oracle; the empty instance yields empty arrays."""
    import spinsim_b200 as ss
    import spinsim_b200.batch as B
    H, O1 = ss.SpinQuantumNumber.HALF, ss.SpinQuantumNumber.ONE
    p = F.tone_parameters(np.random.default_rng(77))
    specs = [(H, 0.0, 0.0, 10e-9, 1e-6), (H, 0.0, 1e-6, 10e-9, 1e-6), (O1, 0.0, 20e-6, 1e-6, 1e-6),
             (H, 1e-6, 31e-6, 30e-9, 1e-6), (O1, 0.0, 7e-6, 10e-9, 1e-6), (H, 0.0, 200e-6, 10e-9, 1e-6)]
    insts = [B.Instance(s, t0, t1, dti, dto, s.plus_x, sweep_parameters=p, field=tone_field(p))
             for s, t0, t1, dti, dto in specs]
    for prec in (ss.Precision.FP64, ss.Precision.FP32_BULK):
        b = B.Batch(insts, precision=prec)
        b.run()
        for k, (s, t0, t1, dti, dto) in enumerate(specs):
            r = b.result(k)
            t, u, st, sp = O.evaluate(s.dimension, O.Field(8), p, t0, t1, dti, dto, s.plus_x)
            assert r.time.shape == t.shape and r.state.shape == st.shape
            assert np.array_equal(r.time, t)
            if t.size:
                tol = 1e-10 if prec == ss.Precision.FP64 else 1e-6
                assert np.abs(r.state - st).max() < tol, (prec, k)
        finals = b.final_states()  # the empty instance has none to gather
        assert np.array_equal(finals[0], np.zeros(2, complex))
        for k in range(1, len(specs)):
            assert np.array_equal(finals[k], b.result(k).state[-1])


def test_full_uneven_tone_batch_properties(cuda):
    """The full 1024-instance uneven tone batch (durations 10 us - 10 ms, 1.4e8 steps) at its real
    size, through size-independent properties: every time grid is t0 + dt_out * i exactly, every
    operator is unitary, every state has unit norm, the FP32-bulk final states are within 1e-6 of
    the FP64 form's, and an instance sampled at random matches the oracle."""
    import torch
    import spinsim_b200 as ss
    import spinsim_b200.batch as B
    rng = np.random.default_rng(3)
    insts = []
    for k in range(1024):
        spin = ss.SpinQuantumNumber.HALF if rng.uniform() < 0.7 else ss.SpinQuantumNumber.ONE
        dur = float(np.exp(rng.uniform(np.log(10e-6), np.log(10e-3))))
        p = F.tone_parameters(np.random.default_rng(10_000 + k))
        insts.append(B.Instance(spin, 0.0, dur, 10e-9, 1e-6, spin.plus_z if spin.dimension == 2 else spin.plus_x,
                                sweep_parameters=p, field=tone_field(p)))
    plans = {}
    bulk = B.Batch(insts, precision=ss.Precision.FP32_BULK, plan_cache=plans)
    plain = B.Batch(insts, precision=ss.Precision.FP64, plan_cache=plans)
    assert bulk.total_steps > 1e8
    bulk.run()
    plain.run()
    torch.cuda.synchronize()
    for b, tol in ((plain, 1e-10), (bulk, 1e-6)):
        worst_u = worst_norm = 0.0
        for k, inst in enumerate(insts):
            r = b.result(k)
            n = r.time.shape[0]
            assert np.array_equal(r.time, 0.0 + 1e-6 * np.arange(n))
            u = r.time_evolution
            d = u.shape[1]
            eye = np.eye(d)
            worst_u = max(worst_u, np.abs(np.einsum("nij,nkj->nik", u, u.conj()) - eye).max())
            worst_norm = max(worst_norm, np.abs(np.linalg.norm(r.state, axis=1) - 1.0).max())
        assert worst_u < tol and worst_norm < tol, (tol, worst_u, worst_norm)
    fb, fp = bulk.final_states(), plain.final_states()
    assert max(np.abs(a - c).max() for a, c in zip(fb, fp)) < 1e-6
    for k in rng.choice(1024, 3, replace=False):
        inst = insts[k]
        d = inst.spin.dimension
        t, u, s, sp = O.evaluate(d, O.Field(8), inst.sweep_parameters, 0.0, inst.time_end, 10e-9, 1e-6, inst.state_init)
        assert np.abs(plain.result(int(k)).state - s).max() < 1e-10


def test_fp32_bulk_uneven_tone_counts(cuda):
    """Tone synthesis with channels of different tone counts: more tones than the per-channel
    synthesis slots (the rest sampled directly), none, and a few with a bias; spin half and spin one,
    against the FP64 form."""
    import spinsim_b200 as ss
    import spinsim_b200.batch as B
    rng = np.random.default_rng(21)

    def tones(n):
        return np.column_stack([ss.fields.TAU * rng.uniform(0, 1e6, n), rng.uniform(0, ss.fields.TAU * 10e3, n),
                                rng.uniform(0, ss.fields.TAU, n)]) if n else None

    insts = []
    for k in range(12):
        chans = {c: tones(n) for c, n in zip((0, 1, 2), (11, 0, 2)) if n}
        f = ss.ToneField(chans, bias=[0.0, 3e3, ss.fields.TAU * 2e3])
        spin = ss.SpinQuantumNumber.HALF if k % 2 else ss.SpinQuantumNumber.ONE
        insts.append(B.Instance(spin, 0.0, float(rng.uniform(50e-6, 400e-6)), 10e-9, 1e-6, spin.plus_x, field=f))
    plans = {}
    bulk = B.Batch(insts, precision=ss.Precision.FP32_BULK, plan_cache=plans)
    plain = B.Batch(insts, precision=ss.Precision.FP64, plan_cache=plans)
    bulk.run()
    plain.run()
    for k in range(len(insts)):
        assert np.abs(bulk.result(k).state - plain.result(k).state).max() < 1e-6, k
        assert np.array_equal(bulk.result(k).time, plain.result(k).time)
