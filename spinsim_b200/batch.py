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
    (use the mixed-spin kernel even for a single-spin batch), ``memory`` (a callable taking a byte
    count and returning a 256-byte aligned uint8 CUDA tensor of at least that size; default
    ``torch.empty``).  All device buffers of the batch (outputs, workspace, fields, sweep
    parameters) are carved from that one allocation, ``device_bytes`` long; the uploads run on the
    current stream.  ``staging`` (optional): a pinned float64 host tensor the field arrays are
    packed into for an asynchronous upload; the caller must not reuse it before that upload has
    completed on the current stream.
    """

    def __init__(self, instances, get_field=None, integration_method=IntegrationMethod.MAGNUS_CF4,
                 exponentiation_half=ExponentiationMethod.ANALYTIC, exponentiation_one=ExponentiationMethod.LIE_TROTTER,
                 use_rotating_frame=True, number_of_squares=24, precision=Precision.FP64, lanes=0,
                 threads_per_block=0, max_registers=0, plan_cache=None, force_mixed=False, memory=None,
                 staging=None):
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

        # Descriptors and output layout (step normalisation and offsets in the library).
        n = len(self.instances)
        insts = (_lib.Instance * n)()
        psi0 = np.zeros((n, 6))
        dims = np.empty(n, np.int32)
        for k, inst in enumerate(self.instances):
            d = dims[k] = inst.spin.dimension
            p = np.asarray(inst.state_init, np.complex128).reshape(-1)
            if p.size != d:
                raise ValueError(f"instance {k}: state_init must have {d} entries")
            psi0[k, 0:2 * d:2] = p.real
            psi0[k, 1:2 * d:2] = p.imag
        t0 = np.fromiter((float(i.time_start) for i in self.instances), np.float64, n)
        t1 = np.fromiter((float(i.time_end) for i in self.instances), np.float64, n)
        dti = np.fromiter((float(i.time_step_integration) for i in self.instances), np.float64, n)
        dto = np.fromiter((float(i.time_step_output) for i in self.instances), np.float64, n)
        totals = (ctypes.c_int64 * 4)()
        _lib.check(lib.spinsim_batch_describe(n, t0.ctypes.data, t1.ctypes.data, dti.ctypes.data, dto.ctypes.data,
                                              dims.ctypes.data, psi0.ctypes.data, insts, totals))
        out_off, u_off, st_off, self.total_steps = (int(v) for v in totals)
        self._inst_np = np.frombuffer(insts, dtype=np.dtype(_lib.Instance))
        keep = []
        params_host = []
        if get_field is not None:
            params_host = [np.asarray(i.sweep_parameters, np.float64).reshape(-1) for i in self.instances]
        self.n_intervals = out_off
        ws_bytes = lib.spinsim_batch_workspace_size(self._plan, insts, n, n)
        if ws_bytes == 0:
            raise ValueError(_lib.last_error() or "batch layout rejected")
        if get_field is None:
            from .fields import packed_doubles
            field_list = [i.field for i in self.instances]
            field_doubles = max(4, packed_doubles(field_list))
        else:
            sizes = [max(1, p.size) for p in params_host]
            offs = np.cumsum([0] + sizes[:-1]).astype(np.int64)
            field_doubles = sum(sizes)
        # one device allocation, 256-byte aligned pieces
        pieces = {"time": 8 * max(1, out_off), "u": 8 * max(2, u_off), "state": 8 * max(2, st_off),
                  "spin": 24 * max(1, out_off), "workspace": ws_bytes, "fields": 8 * field_doubles}
        offsets, total = {}, 0
        for name, nbytes in pieces.items():
            offsets[name] = total
            total += (nbytes + 255) // 256 * 256
        self.device_bytes = total
        if memory is None:
            buf = torch.empty(total, dtype=torch.uint8, device=dev)
        else:
            buf = memory(total)
            if buf.dtype != torch.uint8 or buf.numel() < total or buf.data_ptr() % 256:
                raise ValueError("memory() must return a 256-byte aligned uint8 tensor of the requested size")
        self.memory = buf

        def piece(name, dtype):
            o = offsets[name]
            return buf[o:o + pieces[name]].view(dtype)

        self.time = piece("time", torch.float64)
        self.u = piece("u", torch.complex128)
        self.state = piece("state", torch.complex128)
        self.spin = piece("spin", torch.float64).view(-1, 3)
        self.workspace = piece("workspace", torch.uint8)
        field_dev = piece("fields", torch.float64)
        # the field arrays go through host memory: the caller's pinned staging buffer when it is
        # large enough (an asynchronous copy), else a pageable array (the copy waits for the stream)
        if staging is not None and staging.numel() >= field_doubles:
            host_t = staging[:field_doubles]
        else:
            host_t = torch.from_numpy(np.zeros(field_doubles))
        host = host_t.numpy()
        if get_field is None:
            from .fields import pack_fields_into
            fields_arr = pack_fields_into(field_list, host, field_dev.data_ptr())
        else:
            from .fields import FIELD_DTYPE
            for p, o in zip(params_host, offs):
                host[o:o + p.size] = p
            fields_arr = np.zeros(n, FIELD_DTYPE)
            fields_arr["params"] = field_dev.data_ptr() + 8 * offs
            fields_arr["n_params"] = [p.size for p in params_host]
        field_dev.copy_(host_t, non_blocking=host_t.is_pinned())
        self.h2d_bytes = 8 * field_doubles + ctypes.sizeof(insts) + fields_arr.nbytes
        self._insts, self._fields, self._keep = insts, fields_arr, keep
        handle = ctypes.c_void_p()
        stream = torch.cuda.current_stream(dev).cuda_stream
        _lib.check(lib.spinsim_batch_prepare(self._plan, insts, n, fields_arr.ctypes.data, n, self.workspace.data_ptr(),
                                             ws_bytes, stream, ctypes.byref(handle)))
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

    def layout_of(self, k):
        """(output offset, U offset, state offset (in doubles), N, d) of instance k."""
        r = self._inst_np[k]
        return int(r["out_offset"]), int(r["u_offset"]), int(r["state_offset"]), int(r["n_out"]), int(r["dim"])

    @property
    def layout(self):
        return [self.layout_of(k) for k in range(len(self.instances))]

    def result(self, k, keep=None):
        """Results of instance k (views of the batch's device arrays; ``keep`` is held by the
        Results for as long as it lives)."""
        out_off, u_off, st_off, n_out, d = self.layout_of(k)
        time = self.time[out_off:out_off + n_out]
        u = self.u[u_off // 2:u_off // 2 + n_out * d * d].view(n_out, d, d)
        st = self.state[st_off // 2:st_off // 2 + n_out * d].view(n_out, d)
        sp = self.spin[out_off:out_off + n_out]
        return Results(time, u, st, None, spin=sp, keep=keep)

    def final_states(self):
        """state[N-1] of every instance as a list of numpy arrays."""
        st = self.state.cpu().numpy()
        out = []
        for out_off, u_off, st_off, n_out, d in map(self.layout_of, range(len(self.instances))):
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
