"""Field functions shared by the golden-fixture generator, the oracle tests and the GPU tests.

Each function has the reference's plugin signature
``get_field(time_sample, sweep_parameters, field_sample)`` (spinsim/__init__.py:381-389, :620)
and writes the field in place.  The same Python source is compiled three ways:

* by the reference's numba CPU path when ``make_golden.py`` produces the fixtures;
* by numba's CUDA target to LTO-IR and linked into the sm_100a kernels by ``spinsim_b200``;
* restated in C inside the oracle (``oracle/spinsim_oracle.c``, ``field_eval``), selected by the
  integer code in ``ORACLE_FIELD_CODE``.

Fields taken from the reference's examples cite the example file and line.
"""
import math

TAU = 2.0 * math.pi


def larmor(time_sample, sweep_parameters, field_sample):
    """Constant 1 kHz z field: example.py:7-10 (the Larmor configuration)."""
    field_sample[0] = 0
    field_sample[1] = 0
    field_sample[2] = math.tau * 1000


def rabi(time_sample, sweep_parameters, field_sample):
    """Dressed Rabi flopping, parameters (bias, Rabi): example.py:33-38 (spin one; spin half uses the first three)."""
    field_sample[0] = 2 * sweep_parameters[1] * math.cos(sweep_parameters[0] * time_sample)
    field_sample[1] = 0
    field_sample[2] = sweep_parameters[0]


def rabi_one(time_sample, sweep_parameters, field_sample):
    """example.py:33-38 verbatim, including the quadratic shift entry written for spin one."""
    field_sample[0] = 2 * sweep_parameters[1] * math.cos(sweep_parameters[0] * time_sample)
    field_sample[1] = 0
    field_sample[2] = sweep_parameters[0]
    field_sample[3] = 0


def detuned_rabi(time_sample, sweep_parameters, field_sample):
    """Spin-one detuned Rabi workload: Bz = 2pi(840 kHz + delta), Bx = 2pi 2 kHz cos(2pi 840 kHz t), Bq = 0."""
    field_sample[0] = math.tau * 2e3 * math.cos(math.tau * 840e3 * time_sample)
    field_sample[1] = 0
    field_sample[2] = math.tau * (840e3 + sweep_parameters[0])
    field_sample[3] = 0


def gaussian_ensemble(time_sample, sweep_parameters, field_sample):
    """Spin-half ensemble member: Bz = 2pi delta, Bx = 2pi 50 kHz Gaussian (sigma 2 us, centre 10 us)."""
    field_sample[0] = math.tau * 50e3 * math.exp(-0.5 * ((time_sample - 10e-6) / 2e-6) ** 2)
    field_sample[1] = 0
    field_sample[2] = math.tau * sweep_parameters[0]


def full_su3(time_sample, sweep_parameters, field_sample):
    """All eight su(3) components: full_algebra_example.py:6-15."""
    field_sample[0] = math.tau * 2000 * math.cos(sweep_parameters[0] * time_sample)
    field_sample[1] = 0
    field_sample[2] = sweep_parameters[0]
    field_sample[3] = math.tau * 1000
    field_sample[4] = math.tau * 1000
    field_sample[5] = math.tau * 1000
    field_sample[6] = math.tau * 1000
    field_sample[7] = math.tau * 1000


def gaussian_pulse(time_sample, sweep_parameters, field_sample):
    """Unit-area Gaussian pi pulse in dimensionless time: gaussian_example.py:11-14."""
    field_sample[0] = math.pi / math.sqrt(math.tau) * math.exp(-0.5 * (time_sample ** 2))
    field_sample[1] = 0.0
    field_sample[2] = 0.0


def tones(time_sample, sweep_parameters, field_sample):
    """Eight-tone sum per spatial axis with a bias per channel.

    ``sweep_parameters`` = [bias x, bias y, bias z, bias q, then for each axis x, y, z and each of
    8 tones: angular frequency, amplitude, phase].  Axis a is ``bias[a] + sum A sin(w t + phi)``.
    """
    for axis in range(3):
        value = sweep_parameters[axis]
        for tone in range(8):
            base = 4 + 24 * axis + 3 * tone
            value += sweep_parameters[base + 1] * math.sin(sweep_parameters[base] * time_sample + sweep_parameters[base + 2])
        field_sample[axis] = value
    field_sample[3] = sweep_parameters[3]


ORACLE_FIELD_CODE = {
    "larmor": 1,
    "rabi": 2,
    "rabi_one": 3,
    "detuned_rabi": 4,
    "gaussian_ensemble": 5,
    "full_su3": 6,
    "gaussian_pulse": 7,
    "tones": 8,
    # 9: tabulated channels (see oracle field_eval), built from interpolation tables
}

FIELDS = {
    "larmor": larmor,
    "rabi": rabi,
    "rabi_one": rabi_one,
    "detuned_rabi": detuned_rabi,
    "gaussian_ensemble": gaussian_ensemble,
    "full_su3": full_su3,
    "gaussian_pulse": gaussian_pulse,
    "tones": tones,
}


def tone_parameters(rng, max_frequency=1e6, max_amplitude=TAU * 10e3, bias=(0.0, 0.0, 0.0, 0.0)):
    """Draw the 8-tones-per-axis parameter vector used by ``tones`` (frequency U[0, f_max], amplitude
    U[0, A_max], phase U[0, 2pi)) from a numpy Generator."""
    import numpy as np
    p = np.zeros(4 + 72, np.float64)
    p[:4] = bias
    for axis in range(3):
        for tone in range(8):
            base = 4 + 24 * axis + 3 * tone
            p[base] = TAU * rng.uniform(0.0, max_frequency)
            p[base + 1] = rng.uniform(0.0, max_amplitude)
            p[base + 2] = rng.uniform(0.0, TAU)
    return p
