"""Whole sweeps against the oracle: every detuning of the spin-one Rabi sweep (64, full 10 ms) and
every member of the Gaussian-pulse ensemble (4096, full 1 ms), as the reference's examples evaluate
them one sweep value at a time (example.py:33-45, gaussian_example.py:11-49).  The GPU side runs
each sweep as one batched launch of the plain FP64 form; the final state of every member must match
the oracle's (the reference's algorithm, pinned to its own outputs) to 1e-10, and the FP32-bulk form
of the same batch must stay within 1e-6 of it."""
import numpy as np
import pytest

import fields as F
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _final_states(batch):
    batch.run()
    return batch.final_states()


def test_detuned_rabi_all_64_detunings(cuda):
    """Spin one, Lie-Trotter with 28 squarings, 0-10 ms at 10 ns / 100 ns, start +1 z: all 64 seeded
    detunings uniform in [-5, 5] kHz in one launch, against the oracle run per detuning."""
    import spinsim_b200 as ss
    import spinsim_b200.batch as B
    one = ss.SpinQuantumNumber.ONE
    deltas = np.random.default_rng(seed=1).uniform(-5e3, 5e3, 64)
    insts = [B.Instance(one, 0.0, 10e-3, 10e-9, 100e-9, one.plus_z, sweep_parameters=[d]) for d in deltas]
    kw = dict(get_field=F.detuned_rabi, integration_method=ss.IntegrationMethod.MAGNUS_CF4,
              exponentiation_one=ss.ExponentiationMethod.LIE_TROTTER, number_of_squares=28)
    plain = _final_states(B.Batch(insts, **kw))
    bulk = _final_states(B.Batch(insts, precision=ss.Precision.FP32_BULK, **kw))
    errs = []
    for k, d in enumerate(deltas):
        _, _, s, _ = O.evaluate(3, O.Field(4), [d], 0.0, 10e-3, 10e-9, 100e-9, one.plus_z, expo="lie_trotter",
                                n_squares=28)
        errs.append(np.abs(plain[k] - s[-1]).max())
        assert np.abs(bulk[k] - plain[k]).max() < 1e-6, k
    assert max(errs) < TOL, (int(np.argmax(errs)), max(errs))


def test_gaussian_ensemble_all_4096_members(cuda):
    """Spin half, Bz = 2 pi delta_i with delta_i ~ N(0, 500 Hz), the Gaussian pulse on x, 0-1 ms at
    20 ns / 1 us, start +z: all 4096 seeded members in one launch, against the oracle per member."""
    import spinsim_b200 as ss
    import spinsim_b200.batch as B
    half = ss.SpinQuantumNumber.HALF
    members = np.random.default_rng(seed=2).normal(0.0, 500.0, 4096)
    insts = [B.Instance(half, 0.0, 1e-3, 20e-9, 1e-6, half.plus_z, sweep_parameters=[m]) for m in members]
    plain = _final_states(B.Batch(insts, get_field=F.gaussian_ensemble))
    bulk = _final_states(B.Batch(insts, get_field=F.gaussian_ensemble, precision=ss.Precision.FP32_BULK))
    errs, bulk_errs = np.zeros(members.size), np.zeros(members.size)
    for k, m in enumerate(members):
        _, _, s, _ = O.evaluate(2, O.Field(5), [m], 0.0, 1e-3, 20e-9, 1e-6, half.plus_z)
        errs[k] = np.abs(plain[k] - s[-1]).max()
        bulk_errs[k] = np.abs(bulk[k] - s[-1]).max()
    assert errs.max() < TOL, (int(np.argmax(errs)), errs.max())
    assert bulk_errs.max() < 1e-6, (int(np.argmax(bulk_errs)), bulk_errs.max())
