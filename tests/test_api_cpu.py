"""The drop-in Python API without a GPU: enums, constructor argument handling, the interpolation
sampler and the user-field LTO-IR compilation."""
import math

import numpy as np
import pytest

import spinsim_b200 as ss
import fields as F


def test_enums_match_reference_values():
    # I:58-66, I:78-93, I:111-129, I:229-261
    assert ss.SpinQuantumNumber.HALF.value == 0.5 and ss.SpinQuantumNumber.HALF.dimension == 2
    assert ss.SpinQuantumNumber.ONE.value == 1 and ss.SpinQuantumNumber.ONE.dimension == 3
    assert ss.SpinQuantumNumber.HALF.label == "half" and ss.SpinQuantumNumber.ONE.label == "one"
    assert [m.value for m in ss.IntegrationMethod] == ["magnus_cf4", "euler", "heun"]
    assert [(m.value, m.index) for m in ss.ExponentiationMethod] == [("analytic", 0), ("lie_trotter", 1),
                                                                      ("lie_trotter_8", 2)]
    assert ss.Device.CUDA.index == 1 and ss.Device.CPU.value == "cpu"


def test_basis_states_match_reference():
    import golden_cases as G
    h, o = ss.SpinQuantumNumber.HALF, ss.SpinQuantumNumber.ONE
    assert np.array_equal(h.plus_x, np.array([1, 1]) / math.sqrt(2))
    assert np.array_equal(o.plus_y, np.array([-1, -1j * math.sqrt(2), 1]) / 2)
    for c in G.cases():
        if isinstance(c["psi0"], str):
            spin = h if c["spin"] == "half" else o
            assert np.array_equal(getattr(spin, c["psi0"]), G.expected(c["name"])["psi0"])


def test_spin_half_lie_trotter_8_is_rejected():
    with pytest.raises(ValueError):
        ss.Simulator(F.larmor, ss.SpinQuantumNumber.HALF,
                     exponentiation_method=ss.ExponentiationMethod.LIE_TROTTER_8)


def test_non_cuda_device_is_rejected():
    with pytest.raises(ValueError):
        ss.Simulator(F.larmor, ss.SpinQuantumNumber.HALF, ss.Device.CPU)


def test_no_cpu_fallback():
    """Without a GPU the simulator refuses to run instead of computing on the host."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(RuntimeError):
        ss.Simulator(F.larmor, ss.SpinQuantumNumber.HALF)


def test_user_field_compiles_to_ltoir():
    from spinsim_b200.user_field import compile_ltoir
    for f in (F.larmor, F.rabi_one, F.tones, F.full_su3):
        blob = compile_ltoir(f)
        assert isinstance(blob, bytes) and len(blob) > 1000
    assert compile_ltoir(F.larmor) is compile_ltoir(F.larmor)


def test_sampler_in_user_field_compiles():
    from spinsim_b200.user_field import compile_ltoir
    t = np.linspace(0, 1e-3, 11)
    s = ss.generate_interpolation_sampler(t, np.sin(t * 1e4), order=3)

    def field(time_sample, sweep_parameters, field_sample):
        field_sample[2] = sweep_parameters[0] * s(time_sample)

    assert len(compile_ltoir(field)) > 1000


@pytest.mark.parametrize("order", [0, 1, 3])
@pytest.mark.parametrize("zb", [True, False])
def test_cpu_sampler_matches_oracle(order, zb):
    from oracle import oracle as O
    rng = np.random.default_rng(order)
    t = np.sort(rng.uniform(0, 1, 25))
    a = rng.normal(size=25)
    samp = ss.generate_interpolation_sampler(t, a, order, zb, device=ss.Device.CPU)
    x = np.linspace(-0.1, 1.1, 301)
    got = np.array([samp(v) for v in x])
    assert np.array_equal(got, O.interpolate(t, a, order, zb, x))


def test_sampler_rejects_bad_order():
    with pytest.raises(NotImplementedError):
        ss.generate_interpolation_sampler(np.arange(3.0), np.arange(3.0), order=2)
    with pytest.raises(NotImplementedError):
        ss.generate_interpolation_sampler(np.arange(3.0), np.zeros((3, 2)))
