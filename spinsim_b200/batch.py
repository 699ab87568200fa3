"""Batched evaluation: many evaluate() calls in one persistent launch.

The reference runs one ``evaluate`` per sweep value and per duration (spinsim/__init__.py:993); a
sweep is a Python loop of kernel launches (example.py:41-45).  ``Batch`` runs a whole list of
instances (different spin, duration, step sizes, sweep parameters or fields) as one persistent
time-evolution launch over a longest-first tile queue, followed by the segmented state scan, with
all descriptors resident on the device.  ``Batch.run`` can be captured once into a CUDA graph and
replayed.  Every instance's arithmetic is independent of what else is in the batch (fixed tiles,
fixed scan tree), so a result is the same alone and in a mix.
"""
import ctypes
from dataclasses import dataclass, field as dc_field
from typing import Any, Optional, Sequence

import numpy as np

from . import _lib
from . import (BuiltinField, ExponentiationMethod, IntegrationMethod, Precision, Results, SpinQuantumNumber,
               _INTEGRATION_CODE, _cuda_device)


@dataclass
class Instance:
    """One evaluate() call: the reference's evaluate arguments (I:993) plus its field.

    ``field`` is a built-in field (TabulatedField / ToneField) when the batch has no user field;
    with a user ``get_field`` it is ignored and ``sweep_parameters`` go to get_field."""
    spin: SpinQuantumNumber
    time_start: float
    time_end: float
    time_step_integration: float
    time_step_output: float
    state_init: Any
    sweep_parameters: Sequence[float] = (0.0,)
    field: Optional[BuiltinField] = None
    meta: dict = dc_field(default_factory=dict)


class Batch:
    """A fixed list of instances prepared for repeated launches.

    Parameters mirror Simulator: ``get_field`` (a user function shared by all instances, or None for
    per-instance built-in fields), ``integration_method``, ``exponentiation_half`` /
    ``exponentiation_one`` (defaults: analytic for spin half, Lie-Trotter for spin one, I:529-533),
    ``use_rotating_frame``, ``number_of_squares``, ``precision``, ``lanes``, ``threads_per_block``,
    ``max_registers`` (the last three are picked by ``spinsim_b200.autotune.tune``), ``force_mixed``
    (use the mixed-spin kernel even for a single-spin batch).
    """

    def __init__(self, instances, get_field=None, integration_method=IntegrationMethod.MAGNUS_CF4,
                 exponentiation_half=ExponentiationMethod.ANALYTIC, exponentiation_one=ExponentiationMethod.LIE_TROTTER,
                 use_rotating_frame=True, number_of_squares=24, precision=Precision.FP64, lanes=0,
                 threads_per_block=0, max_registers=0, plan_cache=None, force_mixed=False):
        import torch
        self.instances = list(instances)
        if not self.instances:
            raise ValueError("empty batch")
        dev = _cuda_device()
        self.device = dev
        dims = sorted({i.spin.dimension for i in self.instances})
        # force_mixed: always the mixed-spin kernel, so results do not depend on the batch's spin mix
        spin_dim = dims[0] if (len(dims) == 1 and not force_mixed) else 0
        if exponentiation_one == ExponentiationMethod.ANALYTIC:
            exponentiation_one = ExponentiationMethod.LIE_TROTTER
        if get_field is None:
            kinds = {type(i.field).kind if i.field is not None else None for i in self.instances}
            if len(kinds) != 1 or None in kinds:
                raise ValueError("without a user get_field every instance needs a built-in field of one kind")
            field_kind = kinds.pop()
            ltoir = None
        else:
            field_kind = 0
            from .user_field import compile_ltoir
            ltoir = compile_ltoir(get_field)
        desc = _lib.PlanDesc()
        desc.spin_dim = spin_dim
        desc.integration = _INTEGRATION_CODE[integration_method]
        desc.expo_half = exponentiation_half.index if spin_dim != 3 else 0
        desc.expo_one = exponentiation_one.index if spin_dim != 2 else 1
        desc.rotating = int(bool(use_rotating_frame))
        desc.number_of_squares = int(number_of_squares)
        desc.field_kind = field_kind
        desc.precision = Precision(precision).value
        desc.threads_per_block = int(threads_per_block)
        desc.lanes = int(lanes)
        desc.max_registers = int(max_registers)
        self.config = {"lanes": int(lanes), "threads_per_block": int(threads_per_block),
                       "max_registers": int(max_registers)}
        self.lib = lib = _lib.load()
        key = bytes(desc) + (ltoir or b"")
        if plan_cache is not None and key in plan_cache:
            self._plan, self._owns_plan = plan_cache[key], False
        else:
            plan = ctypes.c_void_p()
            buf = ctypes.create_string_buffer(ltoir) if ltoir else None
            _lib.check(lib.spinsim_plan_create(ctypes.byref(desc), buf, len(ltoir) if ltoir else 0, ctypes.byref(plan)))
            self._plan, self._owns_plan = plan, plan_cache is None
            if plan_cache is not None:
                plan_cache[key] = plan

        # Descriptors and output layout.
        n = len(self.instances)
        insts = (_lib.Instance * n)()
        fields = []
        keep = []
        params_host = []
        self.layout = []
        out_off = u_off = st_off = 0
        self.total_steps = 0
        for k, inst in enumerate(self.instances):
            d = inst.spin.dimension
            dt_int, n_out, n_fine, _ = _lib.normalise_steps(inst.time_start, inst.time_end,
                                                            inst.time_step_integration, inst.time_step_output)
            s = insts[k]
            s.t0 = float(inst.time_start)
            s.dt_int = dt_int
            s.dt_out = float(inst.time_step_output)
            s.n_out = n_out
            s.n_fine = n_fine
            s.dim = d
            s.out_offset = out_off
            s.u_offset = u_off
            s.state_offset = st_off
            s.field = k
            psi0 = np.asarray(inst.state_init, np.complex128).reshape(-1)
            if psi0.size != d:
                raise ValueError(f"instance {k}: state_init must have {d} entries")
            for j in range(d):
                s.psi0[2 * j] = psi0[j].real
                s.psi0[2 * j + 1] = psi0[j].imag
            self.layout.append((out_off, u_off, st_off, n_out, d))
            out_off += n_out
            u_off += 2 * d * d * n_out
            st_off += 2 * d * n_out
            self.total_steps += n_out * n_fine
            if get_field is not None:
                params_host.append(np.asarray(inst.sweep_parameters, np.float64).reshape(-1))
        self.h2d_bytes = 0
        if get_field is None:
            from .fields import pack_fields
            fields, kp, nbytes = pack_fields([i.field for i in self.instances], dev)
            keep += kp
            self.h2d_bytes += nbytes
        if get_field is not None:
            sizes = [max(1, p.size) for p in params_host]
            flat = np.zeros(sum(sizes))
            offs = np.cumsum([0] + sizes[:-1])
            for p, o in zip(params_host, offs):
                flat[o:o + p.size] = p
            params_dev = torch.from_numpy(flat).to(dev)
            keep.append(params_dev)
            self.h2d_bytes += flat.nbytes
            for p, o in zip(params_host, offs):
                f = _lib.Field()
                f.params = params_dev.data_ptr() + 8 * int(o)
                f.n_params = p.size
                fields.append(f)
        self.n_intervals = out_off
        fields_arr = (_lib.Field * n)(*fields)
        self.h2d_bytes += ctypes.sizeof(insts) + ctypes.sizeof(fields_arr)
        self._insts, self._fields, self._keep = insts, fields_arr, keep
        self.time = torch.empty(max(1, out_off), dtype=torch.float64, device=dev)
        self.u = torch.empty(max(1, u_off // 2), dtype=torch.complex128, device=dev)
        self.state = torch.empty(max(1, st_off // 2), dtype=torch.complex128, device=dev)
        self.spin = torch.empty((max(1, out_off), 3), dtype=torch.float64, device=dev)
        ws_bytes = lib.spinsim_batch_workspace_size(self._plan, insts, n, n)
        if ws_bytes == 0:
            raise ValueError(_lib.last_error() or "batch layout rejected")
        self.workspace = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
        handle = ctypes.c_void_p()
        stream = torch.cuda.current_stream(dev).cuda_stream
        _lib.check(lib.spinsim_batch_prepare(self._plan, insts, n, fields_arr, n, self.workspace.data_ptr(), ws_bytes,
                                             stream, ctypes.byref(handle)))
        self._handle = handle
        self._graph = None

    def run(self, stream=None, with_state=True, with_spin=True):
        """Launch the batch (time evolution + state scan + spin) on ``stream`` (default: current)."""
        import torch
        if stream is None:
            stream = torch.cuda.current_stream(self.device).cuda_stream
        _lib.check(self.lib.spinsim_batch_launch(self._handle, self.time.data_ptr(), self.u.data_ptr(),
                                                 self.state.data_ptr() if with_state else None,
                                                 self.spin.data_ptr() if (with_state and with_spin) else None, stream))

    def capture(self):
        """Capture ``run`` into a CUDA graph; ``replay()`` then relaunches it."""
        import torch
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(s):
            self.run()  # warm-up outside the graph (module loads, lazy init)
        torch.cuda.current_stream(self.device).wait_stream(s)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.run()
        self._graph = g
        return g

    def replay(self):
        if self._graph is None:
            self.capture()
        self._graph.replay()

    def plan_info(self):
        info = _lib.PlanInfo()
        _lib.check(self.lib.spinsim_plan_get_info(self._plan, ctypes.byref(info)))
        return {k: getattr(info, k) for k, _ in _lib.PlanInfo._fields_}

    def result(self, k):
        """Results of instance k (views of the batch's device arrays)."""
        out_off, u_off, st_off, n_out, d = self.layout[k]
        time = self.time[out_off:out_off + n_out]
        u = self.u[u_off // 2:u_off // 2 + n_out * d * d].view(n_out, d, d)
        st = self.state[st_off // 2:st_off // 2 + n_out * d].view(n_out, d)
        sp = self.spin[out_off:out_off + n_out]
        return Results(time, u, st, None, spin=sp)

    def final_states(self):
        """state[N-1] of every instance as a list of numpy arrays."""
        st = self.state.cpu().numpy()
        out = []
        for out_off, u_off, st_off, n_out, d in self.layout:
            out.append(st[st_off // 2 + (n_out - 1) * d: st_off // 2 + n_out * d] if n_out else np.zeros(d, complex))
        return out

    def __del__(self):
        try:
            if getattr(self, "_handle", None) is not None and self._handle.value:
                self.lib.spinsim_batch_destroy(self._handle)
            if getattr(self, "_owns_plan", False) and self._plan.value:
                self.lib.spinsim_plan_destroy(self._plan)
        except Exception:
            pass
