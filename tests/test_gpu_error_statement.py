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
