"""FP32-bulk results state their error against the FP64 form (Results.error_estimate,
Batch.error_estimates): checked to bound the measured error on every member of the reference
workloads the FP32-bulk form serves, and not to be vacuous (within a fixed factor of the largest
measured error)."""
import numpy as np
import pytest

import fields as F

pytestmark = pytest.mark.gpu


def _max_state_error(bulk, plain):
    """Per instance: max over output steps and entries of |state_bulk - state_fp64| (on the device)."""
    import torch
    out = []
    for k in range(len(bulk.instances)):
        a = bulk.result(k).device_arrays["state"]
        b = plain.result(k).device_arrays["state"]
        out.append((a - b).abs().max().item() if a.numel() else 0.0)
    return np.array(out)


def _check(stated, true, slack=1e4):
    assert stated.shape == true.shape
    assert np.all(stated >= true), (np.max(true / stated), np.argmax(true / stated))
    assert stated.max() <= slack * max(true.max(), 1e-12)


def test_gaussian_ensemble_members(cuda):
    import spinsim_b200 as ss
    import spinsim_b200.batch as B
    members = np.random.default_rng(seed=2).normal(0.0, 500.0, 4096)
    half = ss.SpinQuantumNumber.HALF
    insts = [B.Instance(half, 0, 1e-3, 20e-9, 1e-6, half.plus_z, [m]) for m in members]
    plans = {}
    bulk = B.Batch(insts, get_field=F.gaussian_ensemble, precision=ss.Precision.FP32_BULK, plan_cache=plans)
    plain = B.Batch(insts, get_field=F.gaussian_ensemble, precision=ss.Precision.FP64, plan_cache=plans)
    bulk.run()
    plain.run()
    stated = bulk.error_estimates()
    _check(stated, _max_state_error(bulk, plain))
    assert np.all(plain.error_estimates() == 0.0)
    assert bulk.result(17).error_estimate == pytest.approx(stated[17], rel=1e-12)


def test_uneven_tone_batch_members(cuda):
    """The 1024-instance uneven tone batch of the benchmark (durations up to 10 ms): tensor-path
    kernel (Magnus step) and warp synthesis (CF4)."""
    import sys
    import os
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    import spinsim_b200 as ss
    import spinsim_b200.batch as B
    insts = bench.instances(ss, bench.workload())
    plans = {}
    plain = B.Batch(insts, precision=ss.Precision.FP64, plan_cache=plans, max_registers=128)
    plain.run()
    fp = plain.final_states()
    for variant in (0, 1):
        bulk = B.Batch(insts, precision=ss.Precision.FP32_BULK, plan_cache=plans, variant=variant)
        bulk.run()
        true = np.array([np.abs(a - b).max() if a.size else 0.0 for a, b in zip(bulk.final_states(), fp)])
        _check(bulk.error_estimates(), true)
        del bulk


def test_detuned_rabi_sweep_and_simulator(cuda):
    import spinsim_b200 as ss
    import spinsim_b200.batch as B
    one = ss.SpinQuantumNumber.ONE
    deltas = np.random.default_rng(seed=1).uniform(-5e3, 5e3, 64)
    insts = [B.Instance(one, 0, 2e-3, 10e-9, 100e-9, one.plus_z, [d]) for d in deltas]
    plans = {}
    kw = dict(get_field=F.detuned_rabi, number_of_squares=28, plan_cache=plans)
    bulk = B.Batch(insts, precision=ss.Precision.FP32_BULK, **kw)
    plain = B.Batch(insts, precision=ss.Precision.FP64, **kw)
    bulk.run()
    plain.run()
    _check(bulk.error_estimates(), _max_state_error(bulk, plain))
    sim32 = ss.Simulator(F.detuned_rabi, one, ss.IntegrationMethod.MAGNUS_CF4, ss.ExponentiationMethod.LIE_TROTTER,
                         True, 28, precision=ss.Precision.FP32_BULK)
    sim64 = ss.Simulator(F.detuned_rabi, one, ss.IntegrationMethod.MAGNUS_CF4, ss.ExponentiationMethod.LIE_TROTTER,
                         True, 28)
    r32 = sim32.evaluate(0, 2e-3, 10e-9, 100e-9, one.plus_z, [deltas[0]])
    r64 = sim64.evaluate(0, 2e-3, 10e-9, 100e-9, one.plus_z, [deltas[0]])
    assert r64.error_estimate == 0.0
    assert r32.error_estimate >= np.abs(r32.state - r64.state).max()


def _tone_field(p):
    import spinsim_b200 as ss
    tones = {a: np.array([(p[4 + 24 * a + 3 * k], p[5 + 24 * a + 3 * k], p[6 + 24 * a + 3 * k]) for k in range(8)])
             for a in range(3)}
    return ss.ToneField(tones, bias=list(p[:4]))


@pytest.mark.parametrize("integration", ["EULER", "HEUN"])
def test_euler_and_heun_fp32_bulk(cuda, integration):
    """FP32-bulk with the Euler and Heun integrators (the generic per-interval kernel: one midpoint
    exponential, or two half-step exponentials at the step's ends, each with its linear part in
    FP64): within 1e-6 of the FP64 form of the same integrator and within the stated error, on tone
    batches of both spins (uneven durations) and on user fields through Simulator."""
    import spinsim_b200 as ss
    import spinsim_b200.batch as B
    integ = getattr(ss.IntegrationMethod, integration)
    half, one = ss.SpinQuantumNumber.HALF, ss.SpinQuantumNumber.ONE
    plans = {}
    for spin in (half, one):
        insts = []
        for k in range(48):
            p = F.tone_parameters(np.random.default_rng(2000 + k))
            dur = float(np.exp(np.random.default_rng(3000 + k).uniform(np.log(5e-6), np.log(300e-6))))
            insts.append(B.Instance(spin, 0.0, dur, 10e-9, 1e-6, spin.plus_x, sweep_parameters=p, field=_tone_field(p)))
        kw = dict(integration_method=integ, plan_cache=plans)
        bulk = B.Batch(insts, precision=ss.Precision.FP32_BULK, **kw)
        plain = B.Batch(insts, precision=ss.Precision.FP64, **kw)
        assert bulk.launch_info()["variant"] == -1  # the generic kernel (no tone synthesis for this integrator)
        bulk.run()
        plain.run()
        true = _max_state_error(bulk, plain)
        assert true.max() < 1e-6, (spin.dimension, true.max())
        _check(bulk.error_estimates(), true)
    for spin, field, sweep in ((half, F.gaussian_ensemble, [250.0]), (one, F.detuned_rabi, [1500.0])):
        sim32 = ss.Simulator(field, spin, integ, precision=ss.Precision.FP32_BULK)
        sim64 = ss.Simulator(field, spin, integ)
        r32 = sim32.evaluate(0, 200e-6, 10e-9, 100e-9, spin.plus_z, sweep)
        r64 = sim64.evaluate(0, 200e-6, 10e-9, 100e-9, spin.plus_z, sweep)
        err = np.abs(r32.state - r64.state).max()
        assert err < 1e-6, (spin.dimension, err)
        assert r32.error_estimate >= err
