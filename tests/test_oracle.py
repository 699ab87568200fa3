"""The oracle (C restatement of the reference) against the reference's own outputs and known answers."""
import math

import numpy as np
import pytest

import golden_cases as G
from oracle import oracle as O


def oracle_field(c):
    if c["field"] == "table":
        return O.Field(9, G.table_channels(c))
    return O.Field(G.F.ORACLE_FIELD_CODE[c["field"]])


def run_case(c, n_threads=0):
    e = G.expected(c["name"])
    d = G.SPIN_DIM[c["spin"]]
    return O.evaluate(d, oracle_field(c), c["sweep"], c["t0"], c["t1"], c["dt_int"], c["dt_out"], e["psi0"],
                      c["integration"], c["exponentiation"], c["rotating"], c["n_squares"], n_threads=n_threads)


@pytest.mark.parametrize("name", [c["name"] for c in G.cases()])
def test_oracle_matches_reference(name):
    """Every golden case (produced by the reference, tests/golden/make_golden.py) to 1e-12."""
    c = G.case(name)
    e = G.expected(name)
    t, u, s, sp = run_case(c)
    assert t.shape == e["time"].shape
    assert np.array_equal(t, e["time"])
    if t.size:
        assert np.abs(u - e["time_evolution"]).max() < 1e-14
        assert np.abs(s - e["state"]).max() < 1e-12
        assert np.abs(sp - e["spin"]).max() < 1e-12


def test_oracle_threads_do_not_change_results():
    c = G.case("one_magnus_cf4_lie_trotter_rf")
    a = run_case(c, n_threads=1)
    b = run_case(c, n_threads=4)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_oracle_larmor_analytic():
    """Larmor precession (example.py:7-15): psi(t) = (exp(-i w t/2), exp(i w t/2))/sqrt2."""
    c = G.case("larmor")
    t, u, s, sp = run_case(c)
    w = math.tau * 1000
    ana = np.stack([np.exp(-0.5j * w * t), np.exp(0.5j * w * t)], 1) / math.sqrt(2)
    assert np.abs(s - ana).max() < 1e-11


def test_oracle_gaussian_pulse_analytic():
    """gaussian_example.py:22-26: a pi pulse; the error falls with the step (doc claim < 1e-6 at small steps)."""
    def cumulative(t):
        return 0.5 * (1 + math.erf(t / math.sqrt(2.0))) - 0.5 * (1 + math.erf(-5.0 / math.sqrt(2.0)))
    errs = []
    for dt in (0.1, 0.01):
        t, u, s, sp = O.evaluate(2, O.Field(7), [0.0], -5.0, 7.0, dt, 2.0, [1.0, 0.0])
        ana = np.array([[math.cos(0.5 * math.pi * cumulative(x)), -1j * math.sin(0.5 * math.pi * cumulative(x))]
                        for x in t])
        errs.append(np.sqrt(np.sum(np.abs(s - ana) ** 2)) / 5)
    assert errs[1] < errs[0]
    assert errs[1] < 1e-6


def test_oracle_norm_preserved():
    c = G.case("one_magnus_cf4_lie_trotter_rf")
    t, u, s, sp = run_case(c)
    assert np.abs(np.linalg.norm(s, axis=1) - 1).max() < 1e-12


def test_oracle_reproduces_lie_trotter_8_norm_loss():
    """The reference's eight-generator exponential (I:1810-1925) is not unitary (its third block
    reuses a stale sin term); the oracle reproduces the reference's ~3% norm drift on this case."""
    c = G.case("one_magnus_cf4_lie_trotter_8_rf")
    t, u, s, sp = run_case(c)
    e = G.expected(c["name"])["state"]
    drift = np.abs(np.linalg.norm(s, axis=1) - 1).max()
    assert 0.01 < drift < 0.1
    assert abs(drift - np.abs(np.linalg.norm(e, axis=1) - 1).max()) < 1e-12


def test_oracle_step_normalisation():
    # I:1025-1034: dt_int reset to dt_out / round(dt_out / dt_int); N truncates.
    assert O.normalise_steps(0, 1e-3, 3e-7, 1e-6)[:3] == (1e-6 / 3, 1000, 3)
    assert O.normalise_steps(1e-3, 1.2e-3, 100e-9, 1e-6)[1] == 199
    assert O.normalise_steps(0, 1e-3, 2e-6, 1e-6)[:3] == (1e-6, 1000, 1)
    assert O.normalise_steps(0, 1e-3, 100e-9, 1e-6)[3] is False
    assert O.normalise_steps(0, 1e-3, 3e-7, 1e-6)[3] is True


def test_oracle_interpolation_matches_reference_rules():
    tb = G.tables()
    t = np.linspace(-10e-6, 215e-6, 997)
    for order in (0, 1, 3):
        for zb in (True, False):
            for key in ("x", "y"):
                from spinsim_b200.fields import table_sample
                a = O.interpolate(tb["t" + key], tb["a" + key], order, zb, t)
                b = table_sample(tb["t" + key], tb["a" + key], order, zb, t)
                assert np.array_equal(a, b)
