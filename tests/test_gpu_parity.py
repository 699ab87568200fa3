"""Parity of the sm_100a kernels with the reference, through the drop-in API and the C ABI.

Tolerance (plain FP64 form): 1e-10 max-abs on time_evolution and state, the reference's own CPU
path being the ground truth (golden fixtures made by running it, tests/golden/make_golden.py), and
the oracle (C restatement) for sizes beyond the fixtures.
"""
import math

import numpy as np
import pytest

import golden_cases as G
import fields as F
from oracle import oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-10

_sims = {}


def spin_of(name):
    import spinsim_b200 as ss
    return ss.SpinQuantumNumber.HALF if name == "half" else ss.SpinQuantumNumber.ONE


def user_table_field(c):
    """The golden table field rebuilt on this package's device samplers."""
    import spinsim_b200 as ss
    t = G.tables()
    sx = ss.generate_interpolation_sampler(t["tx"], t["ax"], c["order"], c["zero_boundary"])
    sy = ss.generate_interpolation_sampler(t["ty"], t["ay"], c["order"], c["zero_boundary"])
    sz = ss.generate_interpolation_sampler(t["tz"], t["az"], c["order"], c["zero_boundary"])

    def field(time_sample, sweep_parameters, field_sample):
        field_sample[0] = sweep_parameters[0] * sx(time_sample)
        field_sample[1] = sweep_parameters[1] * sy(time_sample)
        field_sample[2] = sweep_parameters[2] + sweep_parameters[3] * sz(time_sample)
    return field


def simulator(c, field=None, **kw):
    import spinsim_b200 as ss
    key = (c["field"], c.get("order"), c.get("zero_boundary"), c["spin"], c["integration"], c["exponentiation"],
           c["rotating"], c["n_squares"], id(field), tuple(sorted(kw.items())))
    if key not in _sims:
        if field is None:
            field = user_table_field(c) if c["field"] == "table" else F.FIELDS[c["field"]]
        expo = {m.value: m for m in ss.ExponentiationMethod}[c["exponentiation"]] if c["exponentiation"] else None
        _sims[key] = ss.Simulator(field, spin_of(c["spin"]), exponentiation_method=expo,
                                  use_rotating_frame=c["rotating"],
                                  integration_method=ss.IntegrationMethod(c["integration"]),
                                  number_of_squares=c["n_squares"], **kw)
    return _sims[key]


def check(res, e, tol=TOL):
    assert res.time.shape == e["time"].shape
    assert np.array_equal(res.time, e["time"])
    if e["time"].size:
        assert np.abs(res.time_evolution - e["time_evolution"]).max() < tol
        assert np.abs(res.state - e["state"]).max() < tol
        assert np.abs(res.spin - e["spin"]).max() < tol


@pytest.mark.parametrize("name", [c["name"] for c in G.cases()])
def test_user_field_matches_reference(cuda, name):
    """Every golden case through Simulator(get_field, ...) with the field linked from numba LTO-IR."""
    c = G.case(name)
    e = G.expected(name)
    sim = simulator(c)
    res = sim.evaluate(c["t0"], c["t1"], c["dt_int"], c["dt_out"], e["psi0"], c["sweep"])
    check(res, e)


@pytest.mark.parametrize("name", [c["name"] for c in G.cases() if c["field"] == "table"])
def test_tabulated_field_matches_reference(cuda, name):
    """The library's tabulated-field path (no user code) against the reference's interpolated fields."""
    import spinsim_b200 as ss
    c = G.case(name)
    e = G.expected(name)
    t = G.tables()
    p = c["sweep"]
    fld = ss.TabulatedField({0: (t["tx"], t["ax"]), 1: (t["ty"], t["ay"]), 2: (t["tz"], t["az"])},
                            order=c["order"], zero_boundary=c["zero_boundary"], bias={2: p[2]},
                            gain={0: p[0], 1: p[1], 2: p[3]})
    sim = simulator(c, field=fld)
    res = sim.evaluate(c["t0"], c["t1"], c["dt_int"], c["dt_out"], e["psi0"], c["sweep"])
    check(res, e)


def tone_field(p):
    import spinsim_b200 as ss
    tones = {}
    for axis in range(3):
        rows = []
        for k in range(8):
            b = 4 + 24 * axis + 3 * k
            rows.append((p[b], p[b + 1], p[b + 2]))
        tones[axis] = np.array(rows)
    return ss.ToneField(tones, bias=list(p[:4]))


@pytest.mark.parametrize("name", [c["name"] for c in G.cases() if c["field"] == "tones"])
def test_tone_field_matches_reference(cuda, name):
    c = G.case(name)
    e = G.expected(name)
    sim = simulator(c, field=tone_field(c["sweep"]))
    res = sim.evaluate(c["t0"], c["t1"], c["dt_int"], c["dt_out"], e["psi0"], c["sweep"])
    check(res, e)


@pytest.mark.parametrize("lanes", [1, 2, 4, 8, 32])
def test_lane_split_matches_reference(cuda, lanes):
    """Fine steps of one output interval shared by several lanes (warp-shuffle product) give the same
    operators as one lane."""
    c = G.case("one_magnus_cf4_lie_trotter_rf")
    e = G.expected(c["name"])
    sim = simulator(c, lanes=lanes)
    res = sim.evaluate(c["t0"], c["t1"], c["dt_int"], c["dt_out"], e["psi0"], c["sweep"])
    check(res, e)


def test_larmor_full_size(cuda):
    """Larmor precession at full size: 0-100 ms, 100 ns / 500 ns (200,000 output steps)."""
    import spinsim_b200 as ss
    sim = ss.Simulator(F.larmor, ss.SpinQuantumNumber.HALF)
    res = sim.evaluate(0e-3, 100e-3, 100e-9, 500e-9, ss.SpinQuantumNumber.HALF.plus_x)
    t, u, s, sp = O.evaluate(2, O.Field(1), [0.0], 0e-3, 100e-3, 100e-9, 500e-9, ss.SpinQuantumNumber.HALF.plus_x)
    assert res.time.size == 200_000
    assert np.array_equal(res.time, t)
    assert np.abs(res.time_evolution - u).max() < TOL
    assert np.abs(res.state - s).max() < TOL
    w = math.tau * 1000
    ana = np.stack([np.exp(-0.5j * w * res.time), np.exp(0.5j * w * res.time)], 1) / math.sqrt(2)
    assert np.abs(res.state - ana).max() < 1e-10


def test_detuned_rabi_spin_one_full_length(cuda):
    """Spin-one detuned Rabi, Lie-Trotter with 28 squarings, full 10 ms at 10 ns / 100 ns for two
    detunings of the seeded sweep (the other 62 only change the detuning)."""
    import spinsim_b200 as ss
    deltas = np.random.default_rng(seed=1).uniform(-5e3, 5e3, 64)
    sim = ss.Simulator(F.detuned_rabi, ss.SpinQuantumNumber.ONE, ss.IntegrationMethod.MAGNUS_CF4,
                       ss.ExponentiationMethod.LIE_TROTTER, True, 28)
    for delta in deltas[:2]:
        res = sim.evaluate(0, 10e-3, 10e-9, 100e-9, state_start=ss.SpinQuantumNumber.ONE.plus_z,
                           sweep_parameters=[delta])
        t, u, s, sp = O.evaluate(3, O.Field(4), [delta], 0, 10e-3, 10e-9, 100e-9, ss.SpinQuantumNumber.ONE.plus_z,
                                 expo="lie_trotter", n_squares=28)
        assert res.time.size == 100_000
        assert np.abs(res.time_evolution - u).max() < TOL
        assert np.abs(res.state - s).max() < TOL


def test_gaussian_ensemble_members_full_length(cuda):
    import spinsim_b200 as ss
    members = np.random.default_rng(seed=2).normal(0.0, 500.0, 4096)
    sim = ss.Simulator(F.gaussian_ensemble, ss.SpinQuantumNumber.HALF)
    for m in members[:3]:
        res = sim.evaluate(0, 1e-3, 20e-9, 1e-6, ss.SpinQuantumNumber.HALF.plus_z, [m])
        t, u, s, sp = O.evaluate(2, O.Field(5), [m], 0, 1e-3, 20e-9, 1e-6, ss.SpinQuantumNumber.HALF.plus_z)
        assert np.abs(res.state - s).max() < TOL
        assert np.abs(res.time_evolution - u).max() < TOL


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("n", [1, 2, 31, 32, 33, 1023, 1024, 1025, 32_769, 300_001])
def test_state_scan_matches_serial_propagation(cuda, dim, n):
    """get_state as a prefix scan against the reference's serial loop (I:1089-1111) on random
    unitaries, across scan-tile boundaries."""
    import spinsim_b200 as ss
    rng = np.random.default_rng(n + dim)
    a = rng.normal(size=(n, dim, dim)) + 1j * rng.normal(size=(n, dim, dim))
    q, _ = np.linalg.qr(a)
    psi0 = rng.normal(size=dim) + 1j * rng.normal(size=dim)
    psi0 /= np.linalg.norm(psi0)
    state = np.zeros((n, dim), np.complex128)
    ss.Simulator.get_state(psi0, state, q)
    ref = O.state(q, psi0)
    assert np.abs(state - ref).max() < 1e-11


@pytest.mark.parametrize("dim", [2, 3])
def test_spin_kernel_matches_reference(cuda, dim):
    import spinsim_b200 as ss
    rng = np.random.default_rng(dim)
    st = rng.normal(size=(1000, dim)) + 1j * rng.normal(size=(1000, dim))
    sim = ss.Simulator(F.larmor if dim == 2 else F.rabi_one, spin_of("half" if dim == 2 else "one"))
    got = sim.spin_calculator(st)
    assert np.abs(got - O.spin(st)).max() < 1e-12


def test_empty_and_single_step(cuda):
    import spinsim_b200 as ss
    sim = ss.Simulator(F.rabi, ss.SpinQuantumNumber.HALF)
    r = sim.evaluate(0, 0.5e-6, 100e-9, 1e-6, ss.SpinQuantumNumber.HALF.plus_x, [1.0, 1.0])
    assert r.time.shape == (0,) and r.state.shape == (0, 2) and r.spin.shape == (0, 3)
    r = sim.evaluate(0, 1e-6, 100e-9, 1e-6, ss.SpinQuantumNumber.HALF.plus_x, [1.0, 1.0])
    assert r.state.shape == (1, 2) and np.array_equal(r.state[0], ss.SpinQuantumNumber.HALF.plus_x)


def test_gaussian_pi_pulse_known_answer(cuda):
    """gaussian_example.py:22-26 on the device: a Gaussian pi pulse against its closed form (the
    rotation angle is pi times the pulse's cumulative area; error below 1e-6 at dt = 0.01, the
    reference documentation's figure) and against the oracle to 1e-10."""
    import spinsim_b200 as ss

    def cumulative(t):
        return 0.5 * (1 + math.erf(t / math.sqrt(2.0))) - 0.5 * (1 + math.erf(-5.0 / math.sqrt(2.0)))

    sim = ss.Simulator(F.gaussian_pulse, ss.SpinQuantumNumber.HALF)
    res = sim.evaluate(-5.0, 7.0, 0.01, 2.0, [1.0, 0.0])
    ana = np.array([[math.cos(0.5 * math.pi * cumulative(x)), -1j * math.sin(0.5 * math.pi * cumulative(x))]
                    for x in res.time])
    assert np.sqrt(np.sum(np.abs(res.state - ana) ** 2)) / 5 < 1e-6
    t, u, s, sp = O.evaluate(2, O.Field(7), [0.0], -5.0, 7.0, 0.01, 2.0, [1.0, 0.0])
    assert np.array_equal(res.time, t)
    assert np.abs(res.state - s).max() < TOL


@pytest.mark.parametrize("spin_name", ["HALF", "ONE"])
def test_rabi_rotating_wave_limit(cuda, spin_name):
    """example.py:33-45's dressed Rabi drive in the rotating-wave limit (drive 2 kHz, bias 1 MHz):
    the spin's z component follows cos(Omega t) (times 1/2 for spin half) to the size of the
    counter-rotating corrections, Omega / omega = 2e-3."""
    import spinsim_b200 as ss
    spin = getattr(ss.SpinQuantumNumber, spin_name)
    omega, rabi = math.tau * 1e6, math.tau * 2e3
    field = F.rabi if spin == ss.SpinQuantumNumber.HALF else F.rabi_one
    sim = ss.Simulator(field, spin)
    res = sim.evaluate(0.0, 1e-3, 10e-9, 1e-6, spin.plus_z, [omega, rabi])
    scale = 0.5 if spin == ss.SpinQuantumNumber.HALF else 1.0
    z = res.spin[:, 2] / scale
    assert np.abs(z - np.cos(rabi * res.time)).max() < 1e-2
    assert np.abs(np.linalg.norm(res.state, axis=1) - 1.0).max() < 1e-10
