"""Generate the golden fixtures in ``tests/golden/golden.npz`` by running the reference itself.

The reference (alexander-tritt-monash/spinsim, one Python file on numba) is imported from the
directory given by ``--reference`` (or the ``SPINSIM_REFERENCE`` environment variable) with a stub
``numba.roc`` module: the reference's top-level ``from numba import roc`` (spinsim/__init__.py:8)
is the only thing that fails on the numba in this image, and the ROC branches are dead code on the
CPU device.  Every case runs ``Simulator(..., device=Device.CPU)``
(spinsim/__init__.py:375, :993) and stores ``time``, ``time_evolution``, ``state`` and ``spin``.

Usage: ``python tests/golden/make_golden.py --reference <path to the reference checkout>``.  Only this
script reads the reference; the tests read the committed ``golden.npz``.
"""
import argparse
import json
import math
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import fields as F  # noqa: E402


def import_reference(path):
    import numba
    stub = types.ModuleType("numba.roc")
    sys.modules["numba.roc"] = stub
    numba.roc = stub
    sys.path.insert(0, path)
    import spinsim
    return spinsim


def table_cases(rng):
    """Interpolation tables for the tabulated cases: one uniform and one jittered (non-uniform)
    time grid, so that both the guessed-index and the bisection branches of the reference's
    find_time_index (spinsim/__init__.py:2026-2061) are exercised."""
    m = 41
    t_uniform = np.linspace(-5e-6, 205e-6, m)
    t_jitter = np.sort(np.concatenate([[0.0], rng.uniform(0.0, 190e-6, m - 2), [190e-6]]))
    amp_x = rng.normal(0.0, 1.0, m)
    amp_y = rng.normal(0.0, 1.0, m)
    amp_z = rng.normal(0.0, 1.0, m)
    return dict(tx=t_uniform, ax=amp_x, ty=t_jitter, ay=amp_y, tz=t_uniform.copy(), az=amp_z)


def build_cases():
    rng = np.random.default_rng(12345)
    cases = []

    def add(name, spin, field, sweep, t0, t1, dti, dto, psi0, integ="magnus_cf4", expo=None, rf=True, nsq=24, **extra):
        cases.append(dict(name=name, spin=spin, field=field, sweep=list(map(float, sweep)), t0=t0, t1=t1,
                          dt_int=dti, dt_out=dto, psi0=psi0, integration=integ, exponentiation=expo,
                          rotating=rf, n_squares=nsq, **extra))

    # Method matrix, spin half: integrator x exponentiator x frame.
    for integ in ("magnus_cf4", "euler", "heun"):
        for expo in ("analytic", "lie_trotter"):
            for rf in (True, False):
                add(f"half_{integ}_{expo}_{'rf' if rf else 'lab'}", "half", "rabi",
                    [math.tau * 20e3, math.tau * 1e3], 0.0, 200e-6, 100e-9, 1e-6, "plus_x", integ, expo, rf)
    # Method matrix, spin one.
    for integ in ("magnus_cf4", "euler", "heun"):
        for rf in (True, False):
            add(f"one_{integ}_lie_trotter_{'rf' if rf else 'lab'}", "one", "rabi_one",
                [math.tau * 20e3, math.tau * 1e3], 0.0, 200e-6, 100e-9, 1e-6, "plus_z", integ, "lie_trotter", rf)
            add(f"one_{integ}_lie_trotter_8_{'rf' if rf else 'lab'}", "one", "full_su3",
                [math.tau * 20e3], 0.0, 200e-6, 100e-9, 1e-6, "plus_z", integ, "lie_trotter_8", rf)
    # Number of squares (trotter cutoff) variants: 0, odd, the spin-one workload's 28.
    for nsq in (0, 1, 5, 28):
        add(f"half_lt_nsq{nsq}", "half", "rabi", [math.tau * 20e3, math.tau * 1e3], 0.0, 100e-6, 100e-9, 1e-6,
            "plus_y", "magnus_cf4", "lie_trotter", True, nsq)
        add(f"one_lt_nsq{nsq}", "one", "rabi_one", [math.tau * 20e3, math.tau * 1e3], 0.0, 100e-6, 100e-9, 1e-6,
            "zero_x", "magnus_cf4", "lie_trotter", True, nsq)
    # Larmor precession (shortened): analytic state known.
    add("larmor", "half", "larmor", [0.0], 0.0, 2e-3, 100e-9, 500e-9, "plus_x")
    # Spin-one detuned Rabi, LT 28 squarings (shortened), two detunings from seed 1.
    deltas = np.random.default_rng(seed=1).uniform(-5e3, 5e3, 64)
    for k in range(2):
        add(f"detuned_rabi_{k}", "one", "detuned_rabi", [deltas[k]], 0.0, 100e-6, 10e-9, 100e-9, "plus_z",
            "magnus_cf4", "lie_trotter", True, 28)
    # Gaussian-pulse ensemble (shortened), members from seed 2.
    members = np.random.default_rng(seed=2).normal(0.0, 500.0, 4096)
    for k in range(3):
        add(f"gaussian_ensemble_{k}", "half", "gaussian_ensemble", [members[k]], 0.0, 40e-6, 20e-9, 1e-6, "plus_z")
    # Multi-tone fields, both spins.
    for k, spin in enumerate(("half", "one", "half")):
        p = F.tone_parameters(np.random.default_rng(100 + k))
        add(f"tones_{spin}_{k}", spin, "tones", p, 0.0, 20e-6, 10e-9, 1e-6,
            "plus_z" if spin == "half" else "plus_x", "magnus_cf4", None, True, 24)
    # Offset start time and a non-integer output/integration ratio (the reference resets dt_int).
    add("offset_start", "half", "rabi", [math.tau * 20e3, math.tau * 1e3], 1e-3, 1.2e-3, 100e-9, 1e-6, "minus_x")
    add("non_integer_ratio", "half", "rabi", [math.tau * 20e3, math.tau * 1e3], 0.0, 100e-6, 3e-7, 1e-6, "plus_x")
    add("ratio_below_one", "one", "rabi_one", [math.tau * 20e3, math.tau * 1e3], 0.0, 50e-6, 2e-6, 1e-6, "plus_x")
    # The reference's Gaussian pi-pulse example (dimensionless time), analytic answer known.
    for dt in (0.01, 0.1):
        add(f"gaussian_pulse_{dt}", "half", "gaussian_pulse", [0.0], -5.0, 7.0, dt, 2.0, [1.0, 0.0])
    # Edge sizes: a single output step and no output steps.
    add("single_step", "half", "rabi", [math.tau * 20e3, math.tau * 1e3], 0.0, 1e-6, 100e-9, 1e-6, "plus_x")
    add("empty", "one", "rabi_one", [math.tau * 20e3, math.tau * 1e3], 0.0, 0.5e-6, 100e-9, 1e-6, "plus_x")
    # Tabulated channels through the reference's interpolation sampler (orders 0, 1, 3; both boundaries).
    tables = table_cases(rng)
    for order in (0, 1, 3):
        for zb in (True, False):
            add(f"table_half_o{order}_{'zb' if zb else 'hold'}", "half", "table",
                [math.tau * 25e3, math.tau * 10e3, math.tau * 2e3, math.tau * 5e3], 0.0, 200e-6, 50e-9, 1e-6,
                "plus_z", "magnus_cf4", None, True, 24, order=order, zero_boundary=zb)
    add("table_one_o3_zb", "one", "table", [math.tau * 25e3, math.tau * 10e3, math.tau * 2e3, math.tau * 5e3],
        0.0, 200e-6, 50e-9, 1e-6, "plus_z", "magnus_cf4", None, True, 24, order=3, zero_boundary=True)
    return cases, tables


def make_table_field(spinsim, tables, order, zero_boundary, spin):
    """A user field over three reference interpolation samplers: x = p0 sx(t), y = p1 sy(t),
    z = p2 + p3 sz(t) (and q = 0 for spin one)."""
    dev = spinsim.Device.CPU
    sx = spinsim.generate_interpolation_sampler(tables["tx"], tables["ax"], order, zero_boundary, dev)
    sy = spinsim.generate_interpolation_sampler(tables["ty"], tables["ay"], order, zero_boundary, dev)
    sz = spinsim.generate_interpolation_sampler(tables["tz"], tables["az"], order, zero_boundary, dev)
    if spin == "half":
        def field(time_sample, sweep_parameters, field_sample):
            field_sample[0] = sweep_parameters[0] * sx(time_sample)
            field_sample[1] = sweep_parameters[1] * sy(time_sample)
            field_sample[2] = sweep_parameters[2] + sweep_parameters[3] * sz(time_sample)
    else:
        def field(time_sample, sweep_parameters, field_sample):
            field_sample[0] = sweep_parameters[0] * sx(time_sample)
            field_sample[1] = sweep_parameters[1] * sy(time_sample)
            field_sample[2] = sweep_parameters[2] + sweep_parameters[3] * sz(time_sample)
            field_sample[3] = 0
    return field


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("SPINSIM_REFERENCE"),
                    help="directory holding the reference's spinsim/ package (or set SPINSIM_REFERENCE)")
    ap.add_argument("--out", default=os.path.join(HERE, "golden.npz"))
    args = ap.parse_args()
    if not args.reference:
        ap.error("give --reference or set SPINSIM_REFERENCE")
    spinsim = import_reference(args.reference)
    cases, tables = build_cases()
    spins = {"half": spinsim.SpinQuantumNumber.HALF, "one": spinsim.SpinQuantumNumber.ONE}
    integs = {m.value: m for m in spinsim.IntegrationMethod}
    expos = {m.value: m for m in spinsim.ExponentiationMethod}
    arrays = {}
    for key, value in tables.items():
        arrays[f"table/{key}"] = value
    sims = {}
    meta = []
    for case in cases:
        spin = spins[case["spin"]]
        if case["field"] == "table":
            fkey = ("table", case["order"], case["zero_boundary"], case["spin"])
            field = make_table_field(spinsim, tables, case["order"], case["zero_boundary"], case["spin"])
        else:
            fkey = case["field"]
            field = F.FIELDS[case["field"]]
        key = (fkey, case["spin"], case["integration"], case["exponentiation"], case["rotating"], case["n_squares"])
        if key not in sims:
            sims[key] = spinsim.Simulator(
                field, spin, device=spinsim.Device.CPU,
                exponentiation_method=expos[case["exponentiation"]] if case["exponentiation"] else None,
                use_rotating_frame=case["rotating"], integration_method=integs[case["integration"]],
                number_of_squares=case["n_squares"])
        sim = sims[key]
        psi0 = getattr(spin, case["psi0"]) if isinstance(case["psi0"], str) else np.asarray(case["psi0"], np.complex128)
        res = sim.evaluate(case["t0"], case["t1"], case["dt_int"], case["dt_out"], psi0, np.asarray(case["sweep"]))
        name = case["name"]
        arrays[f"{name}/time"] = res.time
        arrays[f"{name}/time_evolution"] = res.time_evolution
        arrays[f"{name}/state"] = res.state
        arrays[f"{name}/spin"] = res.spin
        arrays[f"{name}/psi0"] = np.asarray(psi0, np.complex128)
        meta.append(case)
        print(f"{name:40s} N={res.time.size:6d}", flush=True)
    arrays["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(args.out, **arrays)
    print("wrote", args.out, os.path.getsize(args.out), "bytes")


if __name__ == "__main__":
    main()
