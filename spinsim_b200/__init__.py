"""spinsim_b200: spinsim's evaluation path on NVIDIA B200 (sm_100a).

A drop-in for the reference's public API (alexander-tritt-monash/spinsim, spinsim/__init__.py):

    Simulator(get_field, spin_quantum_number, ...).evaluate(time_start, time_end,
        time_step_integration, time_step_output, state_init, sweep_parameters) -> Results

with ``Results.time``, ``.time_evolution``, ``.state`` and ``.spin`` as numpy arrays (copied from the
device on first access; ``Results.device_arrays`` keeps the torch device tensors).  The enums,
their values and the basis states are the reference's (I:15-269).  The computation runs in
hand-written CUDA kernels behind a C ABI (include/spinsim_b200.h); there is no CPU path.

Both argument spellings of the constructor are accepted: the reference's
``Simulator(get_field, spin, device, exponentiation_method, use_rotating_frame,
integration_method, number_of_squares, threads_per_block, max_registers, number_of_threads)`` and
``Simulator(get_field, spin, integration_method, exponentiation_method, use_rotating_frame,
trotter_cutoff)``; ``trotter_cutoff`` is ``number_of_squares``.  ``evaluate`` accepts
``state_start`` for ``state_init``.
"""
import ctypes
import math
from enum import Enum

import numpy as np

from . import _lib
from .fields import BuiltinField, TabulatedField, ToneField, generate_interpolation_sampler  # noqa: F401

__all__ = ["SpinQuantumNumber", "IntegrationMethod", "ExponentiationMethod", "Device", "Results", "Simulator",
           "generate_interpolation_sampler", "TabulatedField", "ToneField", "Precision"]

sqrt2 = math.sqrt(2)
sqrt3 = math.sqrt(3)


class SpinQuantumNumber(Enum):
    """Spin quantum number (I:15-66): ``value``, Hilbert-space ``dimension``, ``label`` and the spin
    projection eigenstates ``plus_x`` ... ``minus_z`` as complex128 vectors."""

    def __init__(self, value, dimension, label):
        super().__init__()
        self._value_ = value
        self.dimension = dimension
        self.label = label
        if self.label == "half":
            self.plus_x = np.array([1, 1], np.complex128) / math.sqrt(2)
            self.minus_x = np.array([-1, 1], np.complex128) / math.sqrt(2)
            self.plus_y = np.array([1, 1j], np.complex128) / math.sqrt(2)
            self.minus_y = np.array([1, -1j], np.complex128) / math.sqrt(2)
            self.plus_z = np.array([1, 0], np.complex128)
            self.minus_z = np.array([0, 1], np.complex128)
        else:
            self.plus_x = np.array([1, math.sqrt(2), 1], np.complex128) / 2
            self.zero_x = np.array([-1, 0, 1], np.complex128) / math.sqrt(2)
            self.minus_x = np.array([1, -math.sqrt(2), 1], np.complex128) / 2
            self.plus_y = np.array([-1, -1j * math.sqrt(2), 1], np.complex128) / 2
            self.zero_y = np.array([1, 0, 1], np.complex128) / math.sqrt(2)
            self.minus_y = np.array([1, -1j * math.sqrt(2), 1], np.complex128) / 2
            self.plus_z = np.array([1, 0, 0], np.complex128)
            self.zero_z = np.array([0, 1, 0], np.complex128)
            self.minus_z = np.array([0, 0, 1], np.complex128)

    HALF = (1 / 2, 2, "half")
    ONE = (1, 3, "one")


class IntegrationMethod(Enum):
    """Integrator (I:68-93)."""
    MAGNUS_CF4 = "magnus_cf4"
    EULER = "euler"
    HEUN = "heun"


class ExponentiationMethod(Enum):
    """Matrix exponential (I:95-129): ``value`` label and ``index``."""

    def __init__(self, value, index):
        super().__init__()
        self._value_ = value
        self.index = index

    ANALYTIC = ("analytic", 0)
    LIE_TROTTER = ("lie_trotter", 1)
    LIE_TROTTER_8 = ("lie_trotter_8", 2)


class Device(Enum):
    """Target device names of the reference (I:131-269).  This package evaluates on CUDA only; the
    CPU members remain for ``generate_interpolation_sampler`` (host samplers for plotting)."""

    def __init__(self, value, index):
        super().__init__()
        self._value_ = value
        self.index = index

    PYTHON = ("python", 0)
    CPU_SINGLE = ("cpu_single", 0)
    CPU = ("cpu", 0)
    CUDA = ("cuda", 1)
    ROC = ("roc", 2)


class Precision(Enum):
    """Arithmetic of the time-evolution kernel.  ``FP64``: the reference's arithmetic in double
    precision.  ``FP32_BULK``: single precision for the per-step generators and exponentials, double
    precision for fields, phases and every product across steps (batched form); its results state
    their error against the FP64 form (``Results.error_estimate``)."""
    FP64 = 0
    FP32_BULK = 1


# Error statement of FP32-bulk results against the FP64 form.  Every fine step keeps the linear part
# of its exponential, -i g.J with g the step generator, in FP64; only its O(|g|^2) remainder (and the
# Magnus commutator, the quadratic part of the CF4 product) is computed in FP32, so a step's FP32
# rounding error is at most about 2^-24 |g|^2 (four times that for the sincos branch at |g| > 1/2;
# twice for spin one, whose operator is the spin-one image of an SU(2) element).  Summed over the
# steps without any cancellation this gives ERROR_KAPPA[d] 2^-24 sum |g|^2, a bound that holds even
# when the rounding errors of consecutive steps repeat (slowly varying fields); the kernels accumulate
# sum |g|^2 on the device (step norms).  Added to it: the FP64 form's Lie-Trotter approximant differs
# from the exact exponential the FP32-bulk form applies by at most |g|^2 / 4^h per step (h = number of
# squarings / 2; spin one, and spin half when Lie-Trotter is chosen); tone instances that took the
# one-exponential Magnus step differ from CF4 by at most MAGNUS_PER_STEP theta^5 per step; and both
# forms round in FP64, FP64_PER_STEP per step.  The GPU tests check the statement against the
# measured error on every member of the Gaussian-pulse ensemble (4096 members), the uneven
# 1024-instance tone batch and the spin-one detuned Rabi sweep.
FP32_UNIT = 2.0 ** -24
ERROR_KAPPA = {2: 4.0, 3: 8.0}
MAGNUS_PER_STEP = 3e-10
MAGNUS_THETA = 0.1
FP64_PER_STEP = 2.0 ** -47


def bulk_error_estimate(sum_sq, dim, method_bound=0.0, steps=0, lie_trotter_hypercubes=None):
    """Stated error of an FP32-bulk result against the FP64 form, from the sum over its steps of |g|^2
    (``sum_sq``), its spin dimension, the Magnus step's bound, its number of fine steps and, when the
    FP64 form uses Lie-Trotter, its number of hypercubes h (number of squarings / 2)."""
    sum_sq = max(float(sum_sq), 0.0)
    err = ERROR_KAPPA[int(dim)] * FP32_UNIT * sum_sq + float(method_bound) + FP64_PER_STEP * float(steps)
    if lie_trotter_hypercubes is not None:
        err += sum_sq / 4.0 ** int(lie_trotter_hypercubes)
    return err


def magnus_method_bound(field, time_step_integration, steps):
    """Bound on the one-exponential Magnus step's difference from CF4 for a tone field instance on the
    tensor-path kernel (zero when the kernel keeps CF4: theta = h (|B|max + w_max) above MAGNUS_THETA,
    or any other field)."""
    if not isinstance(field, ToneField):
        return 0.0
    bsq, wmax = 0.0, 0.0
    for c in range(3):
        tones = field.tones.get(c)
        bc = abs(float(field.bias[c]))
        if tones is not None and len(tones):
            t = np.asarray(tones, np.float64).reshape(-1, 3)
            if t.shape[0] > 8:  # more tones than the tensor path takes: the per-interval CF4 path
                return 0.0
            bc += float(np.abs(t[:, 1]).sum())
            wmax = max(wmax, float(np.abs(t[:, 0]).max()))
        bsq += bc * bc
    theta = float(time_step_integration) * (math.sqrt(bsq) + wmax)
    return MAGNUS_PER_STEP * theta ** 5 * steps if theta <= MAGNUS_THETA else 0.0


_INTEGRATION_CODE = {IntegrationMethod.MAGNUS_CF4: 0, IntegrationMethod.EULER: 1, IntegrationMethod.HEUN: 2}
_RED = "\033[31m"
_YELLOW = "\033[33m"
_RESET = "\033[0m"


# ---------------------------------------------------------------------------------------- Results
class Results:
    """Results of an evaluation (I:271-332): ``time`` (N,), ``time_evolution`` (N, d, d),
    ``state`` (N, d) and ``spin`` (N, 3).

    Constructed by ``Simulator.evaluate`` from device tensors (copied to numpy on first access), or
    as in the reference from arrays and a ``spin_calculator`` that computes ``spin`` on first access.
    """

    _ARRAYS = ("time", "time_evolution", "state", "spin")

    def __init__(self, time, time_evolution, state, spin_calculator=None, *, spin=None, keep=None, error=None):
        self.__dict__["_dev"] = {"time": time, "time_evolution": time_evolution, "state": state}
        if spin is not None:
            self.__dict__["_dev"]["spin"] = spin
        self.__dict__["spin_calculator"] = spin_calculator
        self.__dict__["_keep"] = keep
        self.__dict__["_error"] = error

    @property
    def error_estimate(self):
        """Stated error of ``state`` against the FP64 form (max over entries and output steps of the
        difference; the FP64 form itself matches the reference to 1e-10): 0.0 for FP64 results, the
        FP32-bulk error statement (``bulk_error_estimate``) for FP32-bulk results, None when unknown
        (results built from host arrays)."""
        err = self.__dict__["_error"]
        if callable(err):
            err = err()
            self.__dict__["_error"] = err
        return err

    @property
    def device_arrays(self):
        """The torch device tensors behind the results (no copy)."""
        return dict(self.__dict__["_dev"])

    def __getattr__(self, name):
        dev = self.__dict__["_dev"]
        if name in Results._ARRAYS:
            if name in dev:
                value = _to_numpy(dev[name])
            elif name == "spin":
                calc = self.__dict__["spin_calculator"]
                if calc is None:
                    raise AttributeError("no spin calculator")
                value = _to_numpy(calc(self.state))
            else:
                raise AttributeError(name)
            self.__dict__[name] = value
            return value
        raise AttributeError("{} has no attribute called {}.".format(self, name))


def _to_numpy(x):
    if isinstance(x, np.ndarray):
        return x
    try:
        import torch
        if isinstance(x, torch.Tensor):
            return x.detach().cpu().numpy()
    except ImportError:
        pass
    return np.asarray(x)


# -------------------------------------------------------------------------------------- Simulator
def _cuda_device():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("spinsim_b200 evaluates on a CUDA device and none is available")
    return torch.device("cuda", torch.cuda.current_device())


class Simulator:
    """The reference's Simulator (I:334-1111) on sm_100a kernels.

    ``get_field`` is a Python function ``get_field(time_sample, sweep_parameters, field_sample)``
    (compiled by numba to LTO-IR and linked into the kernel), or a built-in ``TabulatedField`` /
    ``ToneField`` evaluated by the library.  Extra keyword options: ``precision`` (``Precision``),
    ``lanes`` (lanes per output step; 0 = automatic).
    """

    def __init__(self, get_field, spin_quantum_number, *args, device=None, exponentiation_method=None,
                 use_rotating_frame=True, integration_method=IntegrationMethod.MAGNUS_CF4, number_of_squares=None,
                 threads_per_block=64, max_registers=None, number_of_threads=None, trotter_cutoff=None,
                 precision=Precision.FP64, lanes=0):
        opts = dict(device=device, exponentiation_method=exponentiation_method,
                    use_rotating_frame=use_rotating_frame, integration_method=integration_method,
                    number_of_squares=number_of_squares, threads_per_block=threads_per_block,
                    max_registers=max_registers, number_of_threads=number_of_threads)
        if args:
            # Positional form: the reference's order (device third) or the (integration_method,
            # exponentiation_method, use_rotating_frame, trotter_cutoff) order, told apart by type.
            if isinstance(args[0], IntegrationMethod):
                names = ["integration_method", "exponentiation_method", "use_rotating_frame", "number_of_squares"]
            else:
                names = ["device", "exponentiation_method", "use_rotating_frame", "integration_method",
                         "number_of_squares", "threads_per_block", "max_registers", "number_of_threads"]
            if len(args) > len(names):
                raise TypeError("too many positional arguments")
            for n, v in zip(names, args):
                opts[n] = v
        if trotter_cutoff is not None:
            if opts["number_of_squares"] is not None and opts["number_of_squares"] != trotter_cutoff:
                raise TypeError("give number_of_squares or trotter_cutoff, not both")
            opts["number_of_squares"] = trotter_cutoff
        if opts["number_of_squares"] is None:
            opts["number_of_squares"] = 24
        device = opts["device"] or Device.CUDA
        if device != Device.CUDA:
            raise ValueError(f"spinsim_b200 evaluates on Device.CUDA only (got {device})")
        if not isinstance(spin_quantum_number, SpinQuantumNumber):
            raise TypeError("spin_quantum_number must be a SpinQuantumNumber")
        integration_method = opts["integration_method"]
        if not isinstance(integration_method, IntegrationMethod):
            raise TypeError("integration_method must be an IntegrationMethod")
        expo = opts["exponentiation_method"]
        # Default exponentiator, I:529-533
        if not expo:
            expo = ExponentiationMethod.LIE_TROTTER if spin_quantum_number == SpinQuantumNumber.ONE \
                else ExponentiationMethod.ANALYTIC
        # I:556-559 (the reference prints this and then fails to compile; the intent, switching to
        # Lie-Trotter, is what happens here)
        if expo == ExponentiationMethod.ANALYTIC and spin_quantum_number != SpinQuantumNumber.HALF:
            print(f"{_RED}spinsim warning!!!\n_attempting to use an analytic exponentiation method outside of "
                  f"spin-half. Switching to a Lie Trotter method.{_RESET}")
            expo = ExponentiationMethod.LIE_TROTTER
        if expo == ExponentiationMethod.LIE_TROTTER_8 and spin_quantum_number == SpinQuantumNumber.HALF:
            print(f"{_RED}spinsim error!!!\nnumba could not jit get_field() function into a device function.{_RESET}\n")
            raise ValueError("ExponentiationMethod.LIE_TROTTER_8 is defined for spin one only")
        nsq = int(opts["number_of_squares"])
        tpb = int(opts["threads_per_block"] or 0)

        self.spin_quantum_number = spin_quantum_number
        self.device = device
        self.threads_per_block = tpb
        self.number_of_threads = opts["number_of_threads"]
        self.integration_method = integration_method
        self.exponentiation_method = expo
        self.use_rotating_frame = bool(opts["use_rotating_frame"])
        self.number_of_squares = nsq
        self.precision = Precision(precision)
        self.get_field = get_field
        dim = spin_quantum_number.dimension

        if isinstance(get_field, BuiltinField):
            field_kind = get_field.kind
            ltoir = None
        else:
            field_kind = 0
            from .user_field import compile_ltoir
            try:
                ltoir = compile_ltoir(get_field)
            except Exception:
                print(f"{_RED}spinsim error!!!\nnumba could not jit get_field() function into a device function."
                      f"{_RESET}\n")
                raise
        self._torch_device = _cuda_device()
        desc = _lib.PlanDesc()
        desc.spin_dim = dim
        desc.integration = _INTEGRATION_CODE[integration_method]
        desc.expo_half = expo.index if dim == 2 else 0
        desc.expo_one = expo.index if dim == 3 else 1
        desc.rotating = int(self.use_rotating_frame)
        desc.number_of_squares = nsq
        desc.field_kind = field_kind
        desc.precision = self.precision.value
        # threads_per_block (a tuning knob of the reference, I:375) is honoured up to the kernel's 128
        desc.threads_per_block = max(32, min(128, tpb // 32 * 32)) if tpb else 0
        desc.max_registers = int(opts["max_registers"] or 0)
        desc.lanes = int(lanes)
        lib = _lib.load()
        plan = ctypes.c_void_p()
        buf = ctypes.create_string_buffer(ltoir) if ltoir else None
        _lib.check(lib.spinsim_plan_create(ctypes.byref(desc), buf, len(ltoir) if ltoir else 0, ctypes.byref(plan)))
        self._plan = plan
        self._lib = lib
        self._builtin = None
        if isinstance(get_field, BuiltinField):
            self._builtin = get_field.device_struct(self._torch_device)

    def __del__(self):
        plan = getattr(self, "_plan", None)
        if plan is not None and plan.value:
            try:
                self._lib.spinsim_plan_destroy(plan)
            except Exception:
                pass
            self._plan = None

    @property
    def plan_info(self):
        info = _lib.PlanInfo()
        _lib.check(self._lib.spinsim_plan_get_info(self._plan, ctypes.byref(info)))
        return {k: getattr(info, k) for k, _ in _lib.PlanInfo._fields_}

    def _lie_trotter_hypercubes(self):
        """h = ceil(number_of_squares / 2) when this simulator's FP64 form uses Lie-Trotter, else None."""
        d = self.spin_quantum_number.dimension
        if d == 3 or self.exponentiation_method == ExponentiationMethod.LIE_TROTTER:
            return (int(self.number_of_squares) + 1) // 2
        return None

    def _field_struct(self, sweep_dev):
        if self._builtin is not None:
            return self._builtin[0]
        f = _lib.Field()
        f.params = sweep_dev.data_ptr()
        f.n_params = sweep_dev.numel()
        return f

    def evaluate(self, time_start, time_end, time_step_integration, time_step_output, state_init=None,
                 sweep_parameters=(0,), *, state_start=None):
        """Simulator.evaluate (I:993-1085).  Returns Results(time, time_evolution, state, spin)."""
        import torch
        if state_init is None:
            state_init = state_start
        elif state_start is not None:
            raise TypeError("give state_init or state_start, not both")
        if state_init is None:
            raise TypeError("evaluate() needs an initial state")
        dt_int, n, _, warned = _lib.normalise_steps(time_start, time_end, time_step_integration, time_step_output)
        if warned:
            print(f"{_YELLOW}spinsim warning!!!\ntime_step_output ({time_step_output:8.4e}) not an integer multiple "
                  f"of time_step_integration ({time_step_integration:8.4e}). Resetting time_step_integration to "
                  f"{dt_int:8.4e}.{_RESET}\n")
        if (float(time_end) - float(time_start)) / float(time_step_output) <= -1:
            raise ValueError("negative dimensions are not allowed")
        d = self.spin_quantum_number.dimension
        psi0 = np.ascontiguousarray(np.asarray(state_init, np.complex128).reshape(-1))
        if psi0.size != d:
            raise ValueError(f"state_init must have {d} entries")
        dev = self._torch_device
        sweep = torch.as_tensor(np.asarray(sweep_parameters, np.float64).reshape(-1), device=dev)
        if sweep.numel() == 0:
            sweep = torch.zeros(1, dtype=torch.float64, device=dev)
        time = torch.empty(n, dtype=torch.float64, device=dev)
        u = torch.empty((n, d, d), dtype=torch.complex128, device=dev)
        state = torch.empty((n, d), dtype=torch.complex128, device=dev)
        spin = torch.empty((n, 3), dtype=torch.float64, device=dev)
        ws_bytes = self._lib.spinsim_evaluate_workspace_size(self._plan, n)
        ws = torch.empty(max(ws_bytes, 256), dtype=torch.uint8, device=dev)
        field = self._field_struct(sweep)
        stream = torch.cuda.current_stream(dev).cuda_stream
        if self.precision == Precision.FP32_BULK:
            norms = torch.zeros(max(n, 1), dtype=torch.float32, device=dev)
            _lib.check(self._lib.spinsim_evaluate_with_norms(
                self._plan, ctypes.byref(field), float(time_start), float(dt_int), float(time_step_output), n,
                psi0.ctypes.data_as(ctypes.c_void_p), time.data_ptr(), u.data_ptr(), state.data_ptr(),
                spin.data_ptr(), norms.data_ptr(), ws.data_ptr(), ws.numel(), stream))
            steps = n * int(math.floor(float(time_step_output) / float(dt_int) + 0.5))
            bound = magnus_method_bound(self.get_field, dt_int, steps)
            lt = self._lie_trotter_hypercubes()

            def error():
                return bulk_error_estimate(norms[:n].double().sum().item(), d, bound, steps, lt)
        else:
            _lib.check(self._lib.spinsim_evaluate(
                self._plan, ctypes.byref(field), float(time_start), float(dt_int), float(time_step_output), n,
                psi0.ctypes.data_as(ctypes.c_void_p), time.data_ptr(), u.data_ptr(), state.data_ptr(),
                spin.data_ptr(), ws.data_ptr(), ws.numel(), stream))
            error = 0.0
        return Results(time, u, state, self.spin_calculator, spin=spin, keep=(sweep, ws, self._builtin), error=error)

    def spin_calculator(self, state):
        """get_spin / spin_calculator (I:899-988): Bloch vector of a state series, on the device."""
        import torch
        d = self.spin_quantum_number.dimension
        st = torch.as_tensor(np.asarray(state, np.complex128) if not isinstance(state, torch.Tensor) else state,
                             device=self._torch_device).to(torch.complex128).contiguous()
        n = st.shape[0]
        spin = torch.empty((n, 3), dtype=torch.float64, device=self._torch_device)
        stream = torch.cuda.current_stream(self._torch_device).cuda_stream
        _lib.check(self._lib.spinsim_spin(d, st.data_ptr(), n, spin.data_ptr(), stream))
        return spin.cpu().numpy()

    @staticmethod
    def get_state(state_init, state, time_evolution):
        """get_state (I:1089-1111) on the device: fills ``state`` (numpy, (N, d)) from ``time_evolution``."""
        import torch
        u = torch.as_tensor(np.ascontiguousarray(time_evolution, np.complex128)).cuda()
        n, d = u.shape[0], u.shape[1]
        psi0 = np.ascontiguousarray(np.asarray(state_init, np.complex128).reshape(-1))
        out = torch.empty((n, d), dtype=torch.complex128, device=u.device)
        lib = _lib.load()
        ws_bytes = lib.spinsim_state_workspace_size(d, n)
        ws = torch.empty(max(ws_bytes, 256), dtype=torch.uint8, device=u.device)
        stream = torch.cuda.current_stream(u.device).cuda_stream
        _lib.check(lib.spinsim_state(d, u.data_ptr(), n, psi0.ctypes.data_as(ctypes.c_void_p), out.data_ptr(), None,
                                     ws.data_ptr(), ws.numel(), stream))
        state[...] = out.cpu().numpy()

from . import batch  # noqa: E402,F401  (batched persistent launches)
