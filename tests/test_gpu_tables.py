"""Zero-order-hold tables whose knots fall exactly on sample times, against the oracle.

The table path keeps a per-lane cursor: a sample strictly inside the cursor's interval takes the
kept value, and a sample on a knot goes to the reference's search (find_time_index,
spinsim/__init__.py:2026-2061), which decides between the two touching intervals.  With dyadic step
sizes the sample times are exact binary fractions, so Heun's step-end samples and the rotating
frame's mid-interval samples land exactly on knots; Euler's and CF4's samples fall between them.
Tolerances: 1e-10 for the plain FP64 form, 1e-6 (the FP32-bulk contract) on the final state.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

DT_INT = 2.0 ** -24          # about 60 ns; every sample time below is an exact binary fraction
DT_OUT = 8 * DT_INT
N_OUT = 96
KNOT = 2 * DT_INT            # a knot at every second step boundary


def tables(seed):
    rng = np.random.default_rng(seed)
    n = int(N_OUT * DT_OUT / KNOT) + 1
    t = np.arange(n, dtype=np.float64) * KNOT
    out = []
    for c in range(3):
        scale = 2 * np.pi * (2e5 if c < 2 else 5e4)
        amp = rng.uniform(-1.0, 1.0, n) * scale
        # channel y's knots are shifted by one step, so its knots fall on the other step boundaries
        out.append((t + (DT_INT if c == 1 else 0.0), amp))
    return out


@pytest.mark.parametrize("zero_boundary", [False, True])
@pytest.mark.parametrize("integration", ["heun", "euler", "magnus_cf4"])
@pytest.mark.parametrize("spin", ["half", "one"])
def test_zero_order_hold_knots_on_sample_times(cuda, spin, integration, zero_boundary):
    import spinsim_b200 as ss
    tabs = tables(seed={"half": 5, "one": 6}[spin] + 10 * len(integration))
    sq = ss.SpinQuantumNumber.HALF if spin == "half" else ss.SpinQuantumNumber.ONE
    fld = ss.TabulatedField({c: tabs[c] for c in range(3)}, order=0, zero_boundary=zero_boundary)
    psi0 = sq.plus_x
    t1 = N_OUT * DT_OUT
    ref_field = O.Field(9, [(t, a, 0, zero_boundary) for t, a in tabs])
    _, u_ref, st_ref, _ = O.evaluate(sq.dimension, ref_field, [1.0, 1.0, 0.0, 1.0], 0.0, t1, DT_INT, DT_OUT, psi0,
                                     integration=integration)
    for precision, tol in ((ss.Precision.FP64, 1e-10), (ss.Precision.FP32_BULK, 1e-6)):
        sim = ss.Simulator(fld, sq, integration_method=ss.IntegrationMethod(integration), precision=precision)
        res = sim.evaluate(0.0, t1, DT_INT, DT_OUT, psi0)
        assert res.time_evolution.shape == u_ref.shape
        if precision == ss.Precision.FP64:
            assert np.abs(res.time_evolution - u_ref).max() < tol
            assert np.abs(res.state - st_ref).max() < tol
        else:
            assert np.abs(res.state[-1] - st_ref[-1]).max() < tol
