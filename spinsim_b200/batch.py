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
from itertools import chain
from operator import attrgetter, itemgetter
from typing import Any, Optional, Sequence

import numpy as np

from . import _lib
from . import (BuiltinField, ExponentiationMethod, IntegrationMethod, Precision, Results, SpinQuantumNumber,
               _INTEGRATION_CODE, _cuda_device, bulk_error_estimate, magnus_method_bound)


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
    # (first, count): compute only output steps first .. first + count - 1 of this evaluate()
    # (one piece of a split evaluation; time indices stay those of the whole call)
    intervals: Optional[tuple] = None


INSTANCE_DTYPE = np.dtype(_lib.Instance)
# what a batch reads of every instance, gathered in one C-level pass
_INSTANCE_RECORD = attrgetter("spin", "time_start", "time_end", "time_step_integration", "time_step_output",
                              "state_init", "field")
_TIMES = itemgetter(1, 2, 3, 4)
_T0, _T1, _DT_OUT, _SPIN = (attrgetter(a) for a in ("time_start", "time_end", "time_step_output", "spin"))


def _column(records, k):
    return list(map(itemgetter(k), records))


def _dims_of(spins):
    """int32 array of the spins' dimensions; the per-item work is C-level lookups by object id."""
    ids = list(map(id, spins))
    dim_by_id = {k: v.dimension for k, v in dict(zip(ids, spins)).items()}  # few distinct spin objects
    return np.fromiter(map(dim_by_id.__getitem__, ids), np.int32, len(ids))


def _initial_states(states, dims):
    """(n, 6) float64 rows of interleaved (re, im) initial states, zero padded.  Instances usually
    share a few basis-state objects, so each distinct object is converted once."""
    ids = list(map(id, states))
    distinct = dict(zip(ids, states))
    slot = {k: j for j, k in enumerate(distinct)}
    table = np.zeros((len(distinct), 6), np.float64)
    sizes = np.zeros(len(distinct), np.int32)
    for j, st in enumerate(distinct.values()):
        p = np.asarray(st, np.complex128).reshape(-1)
        sizes[j] = p.size
        if p.size <= 3:
            table[j, 0:2 * p.size:2] = p.real
            table[j, 1:2 * p.size:2] = p.imag
    idx = np.fromiter(map(slot.__getitem__, ids), np.int64, len(ids))
    bad = np.flatnonzero(sizes[idx] != dims)
    if bad.size:
        k = int(bad[0])
        raise ValueError(f"instance {k}: state_init must have {int(dims[k])} entries")
    return table[idx]


class _InstanceColumns:
    """What a batch reads of each instance, in one C-level pass per attribute: the instances, their
    dimensions (int32), times (n, 4: t0, t1, dt_int, dt_out), initial-state rows (n, 6), fields and
    piece ranges."""

    __slots__ = ("instances", "dims", "times", "psi0", "fields", "intervals")

    def __init__(self, instances):
        self.instances = insts = list(instances)
        n = len(insts)
        recs = list(map(_INSTANCE_RECORD, insts))
        self.dims = _dims_of(_column(recs, 0))
        self.times = np.fromiter(chain.from_iterable(map(_TIMES, recs)), np.float64, 4 * n).reshape(n, 4)
        self.psi0 = _initial_states(_column(recs, 5), self.dims)
        self.fields = _column(recs, 6)
        try:
            self.intervals = list(map(attrgetter("intervals"), insts))
        except AttributeError:  # objects with only the other attributes
            self.intervals = [getattr(i, "intervals", None) for i in insts]

    def __len__(self):
        return len(self.instances)


class Batch:
    """A fixed list of instances (``Instance``, or any objects with its attributes) prepared for
    repeated launches.

    Parameters mirror Simulator: ``get_field`` (a user function shared by all instances, or None for
    per-instance built-in fields), ``integration_method``, ``exponentiation_half`` /
    ``exponentiation_one`` (defaults: analytic for spin half, Lie-Trotter for spin one, I:529-533),
    ``use_rotating_frame``, ``number_of_squares``, ``precision``, ``lanes``, ``threads_per_block``,
    ``max_registers``, ``variant`` (FP32-bulk tone fields: 0 the tensor-path kernel, 1 the warp
    synthesis; these four are picked by ``spinsim_b200.autotune.tune``), ``force_mixed``
    (use the mixed-spin kernel even for a single-spin batch), ``memory`` (a callable taking a byte
    count and returning a 256-byte aligned uint8 CUDA tensor of at least that size; default
    ``torch.empty``).  All device buffers of the batch (outputs, workspace, fields, sweep
    parameters) are carved from that one allocation, ``device_bytes`` long; the uploads run on the
    current stream.  ``staging`` (optional): a pinned uint8 host tensor (256-byte aligned), or a
    callable taking a byte count and returning one, that the descriptors and field arrays are
    written into for asynchronous uploads (when it is large enough); the caller must not reuse it
    before those uploads have completed on the current stream.
    """

    def __init__(self, instances, get_field=None, integration_method=IntegrationMethod.MAGNUS_CF4,
                 exponentiation_half=ExponentiationMethod.ANALYTIC, exponentiation_one=ExponentiationMethod.LIE_TROTTER,
                 use_rotating_frame=True, number_of_squares=24, precision=Precision.FP64, lanes=0,
                 threads_per_block=0, max_registers=0, plan_cache=None, force_mixed=False, memory=None,
                 staging=None, variant=0):
        import torch
        cols = _InstanceColumns(instances)
        self.instances = cols.instances
        if not self.instances:
            raise ValueError("empty batch")
        dev = _cuda_device()
        self.device = dev
        n = len(cols)
        dims = cols.dims
        dim_set = sorted(set(dims.tolist()))
        # force_mixed: always the mixed-spin kernel, so results do not depend on the batch's spin mix
        spin_dim = dim_set[0] if (len(dim_set) == 1 and not force_mixed) else 0
        if exponentiation_one == ExponentiationMethod.ANALYTIC:
            exponentiation_one = ExponentiationMethod.LIE_TROTTER
        if get_field is None:
            field_list = cols.fields
            types = set(map(type, field_list))
            kinds = {getattr(t, "kind", None) for t in types}
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
        desc.variant = int(variant)
        self.config = {"lanes": int(lanes), "threads_per_block": int(threads_per_block),
                       "max_registers": int(max_registers), "variant": int(variant)}
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
        insts = (_lib.Instance * n)()
        psi0 = np.ascontiguousarray(cols.psi0)
        dims = np.ascontiguousarray(dims)
        t0, t1, dti, dto = cols.times.T.copy()
        totals = (ctypes.c_int64 * 4)()
        _lib.check(lib.spinsim_batch_describe(n, t0.ctypes.data, t1.ctypes.data, dti.ctypes.data, dto.ctypes.data,
                                              dims.ctypes.data, psi0.ctypes.data, insts, totals))
        out_off, u_off, st_off, self.total_steps = (int(v) for v in totals)
        self._inst_np = np.frombuffer(insts, dtype=INSTANCE_DTYPE)
        if cols.intervals.count(None) != n:
            out_off, u_off, st_off = self._restrict_to_pieces()
        keep = []
        params_host = []
        if get_field is not None:
            params_host = [np.asarray(i.sweep_parameters, np.float64).reshape(-1) for i in self.instances]
        self.n_intervals = out_off
        ws_bytes = lib.spinsim_batch_workspace_size(self._plan, insts, n, n)
        if ws_bytes == 0:
            raise ValueError(_lib.last_error() or "batch layout rejected")
        if get_field is None:
            from .fields import field_plan
            plan_rows, packed = field_plan(field_list)
            field_doubles = max(4, packed)
        else:
            sizes = [max(1, p.size) for p in params_host]
            offs = np.cumsum([0] + sizes[:-1]).astype(np.int64)
            field_doubles = sum(sizes)
        # one device allocation, 256-byte aligned pieces
        # time, U, state and spin come first and back to back: one host copy takes all of them
        pieces = {"time": 8 * max(1, out_off), "u": 8 * max(2, u_off), "state": 8 * max(2, st_off),
                  "spin": 24 * max(1, out_off), "workspace": ws_bytes, "fields": 8 * field_doubles}
        self.precision = Precision(precision)
        if self.precision == Precision.FP32_BULK:  # per output step: sum of |g|^2 (the error statement)
            pieces["norms"] = 4 * max(1, out_off)
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

        # device addresses of the pieces; their tensor views are made on first use
        self._pieces, self._offsets = pieces, offsets
        base = buf.data_ptr()
        self._ptr = {name: base + o for name, o in offsets.items()}
        field_dev = self._piece("fields", torch.float64)
        # Field arrays and descriptors go through host memory: the caller's pinned staging buffer
        # when it is large enough (asynchronous copies: descriptors first, then fields), else
        # pageable memory (the copies wait for the stream).
        desc_bytes = 0
        if staging is not None:
            desc_bytes = (lib.spinsim_batch_staging_size(self._plan, insts, n, n) + 255) // 256 * 256
            if callable(staging):
                staging = staging(desc_bytes + 8 * field_doubles)
            if staging.dtype != torch.uint8 or not staging.is_pinned() or \
                    staging.numel() < desc_bytes + 8 * field_doubles or staging.data_ptr() % 256:
                staging = None
        if staging is not None:
            host_t = staging[desc_bytes:desc_bytes + 8 * field_doubles].view(torch.float64)
        else:
            host_t = torch.from_numpy(np.zeros(field_doubles))
        host = host_t.numpy()
        if get_field is None:
            from .fields import pack_plan_into
            fields_arr = pack_plan_into(plan_rows, n, host, field_dev.data_ptr())
        else:
            from .fields import FIELD_DTYPE
            for p, o in zip(params_host, offs):
                host[o:o + p.size] = p
            fields_arr = np.zeros(n, FIELD_DTYPE)
            fields_arr["params"] = field_dev.data_ptr() + 8 * offs
            fields_arr["n_params"] = [p.size for p in params_host]
        self.h2d_bytes = 8 * field_doubles + ctypes.sizeof(insts) + fields_arr.nbytes
        self._insts, self._fields, self._keep = insts, fields_arr, keep
        handle = ctypes.c_void_p()
        stream = torch.cuda.current_stream(dev).cuda_stream
        if staging is not None:
            _lib.check(lib.spinsim_batch_prepare_staged(self._plan, insts, n, fields_arr.ctypes.data, n,
                                                        self._ptr["workspace"], ws_bytes, staging.data_ptr(),
                                                        desc_bytes, stream, ctypes.byref(handle)))
        else:
            _lib.check(lib.spinsim_batch_prepare(self._plan, insts, n, fields_arr.ctypes.data, n,
                                                 self._ptr["workspace"], ws_bytes, stream, ctypes.byref(handle)))
        # after the descriptor upload, so that torch's record of this copy on the pinned staging
        # block (which keeps the block from reuse until the copy is done) covers both
        field_dev.copy_(host_t, non_blocking=host_t.is_pinned())
        self._staging = staging
        self._handle = handle
        self._graph = None
        self._variant = int(variant)
        self._get_field = get_field
        self._hypercubes = (int(number_of_squares) + 1) // 2
        self._lt_half = exponentiation_half == ExponentiationMethod.LIE_TROTTER
        if "norms" in self._ptr:
            _lib.check(lib.spinsim_batch_set_step_norms(handle, self._ptr["norms"]))

    def run(self, stream=None, with_state=True, with_spin=True):
        """Launch the batch (time evolution + state scan + spin) on ``stream`` (default: current)."""
        import torch
        if stream is None:
            stream = torch.cuda.current_stream(self.device).cuda_stream
        ptr = self._ptr
        _lib.check(self.lib.spinsim_batch_launch(self._handle, ptr["time"], ptr["u"], ptr["state"] if with_state else None,
                                                 ptr["spin"] if (with_state and with_spin) else None, stream))

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

    def launch_info(self):
        """The launch this batch makes: the plan's kernel (plan_info) and the batch's tile queue,
        tile size, lanes per output step and state-scan tiles."""
        info = _lib.BatchInfo()
        _lib.check(self.lib.spinsim_batch_get_info(self._handle, ctypes.byref(info)))
        return {**self.plan_info(), **{k: getattr(info, k) for k, _ in _lib.BatchInfo._fields_}}

    @property
    def lanes(self):
        return self.launch_info()["lanes"]

    def _restrict_to_pieces(self):
        """Apply the instances' ``intervals`` (first, count) to the descriptors and re-pack the
        output offsets; returns the new totals (output steps, U doubles, state doubles)."""
        rec = self._inst_np
        for k, inst in enumerate(self.instances):
            if inst.intervals is None:
                continue
            first, count = (int(v) for v in inst.intervals)
            if first < 0 or count < 0 or first + count > rec[k]["n_out"] or first >= 2 ** 31:
                raise ValueError(f"instance {k}: output steps {first}..{first + count} are outside 0..{rec[k]['n_out']}")
            rec[k]["n_out"] = count
            rec[k]["interval0"] = first
        n_out = rec["n_out"].astype(np.int64)
        d = rec["dim"].astype(np.int64)
        for name, per in (("out_offset", n_out), ("u_offset", 2 * d * d * n_out), ("state_offset", 2 * d * n_out)):
            rec[name][0] = 0
            rec[name][1:] = np.cumsum(per)[:-1]
        self.total_steps = int((n_out * rec["n_fine"]).sum())
        return int(n_out.sum()), int((2 * d * d * n_out).sum()), int((2 * d * n_out).sum())

    def _piece(self, name, dtype):
        o = self._offsets[name]
        return self.memory[o:o + self._pieces[name]].view(dtype)

    @property
    def time(self):
        """Output times of all instances, back to back (float64 device tensor)."""
        if "_time" not in self.__dict__:
            import torch
            self._time = self._piece("time", torch.float64)
        return self._time

    @property
    def u(self):
        """Time-evolution operators of all instances, back to back (flat complex128 device tensor)."""
        if "_u" not in self.__dict__:
            import torch
            self._u = self._piece("u", torch.complex128)
        return self._u

    @property
    def state(self):
        """States of all instances, back to back (flat complex128 device tensor)."""
        if "_state" not in self.__dict__:
            import torch
            self._state = self._piece("state", torch.complex128)
        return self._state

    @property
    def spin(self):
        """Spin expectations of all instances, back to back ((sum N, 3) float64 device tensor)."""
        if "_spin" not in self.__dict__:
            import torch
            self._spin = self._piece("spin", torch.float64).view(-1, 3)
        return self._spin

    @property
    def output_bytes(self):
        """Bytes from the start of the device block to the end of the spin piece: time, U, state and
        spin, back to back (256-byte aligned pieces)."""
        return self._offsets["workspace"]

    def host_views(self, host):
        """numpy (time, U, state, spin) views of a host copy of the first ``output_bytes`` of the
        device block (a uint8 tensor or array), shaped like the device tensors."""
        raw = host.numpy() if hasattr(host, "numpy") else np.asarray(host)
        out = []
        for name, dt in (("time", np.float64), ("u", np.complex128), ("state", np.complex128), ("spin", np.float64)):
            o = self._offsets[name]
            out.append(raw[o:o + self._pieces[name]].view(dt))
        out[3] = out[3].reshape(-1, 3)
        return out

    @property
    def workspace(self):
        if "_workspace" not in self.__dict__:
            import torch
            self._workspace = self._piece("workspace", torch.uint8)
        return self._workspace

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
        error = 0.0
        if self.precision == Precision.FP32_BULK:
            norms = self._piece("norms", __import__("torch").float32)
            terms = self._error_terms(k)

            def error():
                return bulk_error_estimate(norms[out_off:out_off + n_out].double().sum().item(), d, *terms)
        return Results(time, u, st, None, spin=sp, keep=keep, error=error)

    def _error_terms(self, k):
        """(Magnus bound, fine steps, Lie-Trotter hypercubes or None) of instance k's error statement."""
        rec = self._inst_np[k]
        steps = int(rec["n_out"]) * int(rec["n_fine"])
        lt = self._hypercubes if (int(rec["dim"]) == 3 or self._lt_half) else None
        return self._method_bound(k), steps, lt

    def _method_bound(self, k):
        inst = self.instances[k]
        if self._variant != 0 or self._get_field is not None:
            return 0.0
        rec = self._inst_np[k]
        return magnus_method_bound(inst.field, float(rec["dt_int"]), int(rec["n_out"]) * int(rec["n_fine"]))

    def error_estimates(self):
        """The stated error of every instance's state against the FP64 form (numpy, one per instance):
        0 for an FP64 batch; for FP32-bulk the error statement from the step norms the launch wrote
        (one device reduction and one copy for the whole batch)."""
        import torch
        n = len(self.instances)
        if self.precision != Precision.FP32_BULK:
            return np.zeros(n)
        rec = self._inst_np
        norms = self._piece("norms", torch.float32)[:max(1, self.n_intervals)].double()
        csum = torch.cat([torch.zeros(1, dtype=torch.float64, device=norms.device), torch.cumsum(norms, 0)])
        lo = torch.from_numpy(rec["out_offset"].astype(np.int64)).to(norms.device)
        hi = lo + torch.from_numpy(rec["n_out"].astype(np.int64)).to(norms.device)
        sums = (csum[hi] - csum[lo]).cpu().numpy()
        return np.array([bulk_error_estimate(sums[k], rec["dim"][k], *self._error_terms(k)) for k in range(n)])

    def final_states(self):
        """state[N-1] of every instance as a list of numpy arrays (gathered on the device, so only
        the final states are copied to the host)."""
        import torch
        rec = self._inst_np
        n_out = rec["n_out"].astype(np.int64)
        d = rec["dim"].astype(np.int64)
        start = rec["state_offset"].astype(np.int64) // 2 + (n_out - 1) * d
        full = np.flatnonzero(n_out > 0)  # an empty instance has no final state (and no entries to read)
        idx = np.concatenate([np.arange(start[k], start[k] + d[k]) for k in full]) if len(full) else None
        got = self.state[torch.from_numpy(idx).to(self.state.device)].cpu().numpy() if idx is not None else None
        out, at = [], 0
        for k in range(len(d)):
            if n_out[k]:
                out.append(got[at:at + d[k]].copy())
                at += d[k]
            else:
                out.append(np.zeros(d[k], complex))
        return out

    def spin_mean(self, first=0, count=None):
        """Mean spin over instances first .. first + count - 1, which must share N (the members of
        an ensemble); a (N, 3) float64 tensor on the device, reduced there (``spinsim_spin_mean``)."""
        import torch
        rec = self._inst_np
        count = len(self.instances) - first if count is None else count
        if count <= 0 or first < 0 or first + count > len(self.instances):
            raise ValueError("instance range out of bounds")
        n = int(rec["n_out"][first])
        if np.any(rec["n_out"][first:first + count] != n):
            raise ValueError("the members of a spin mean must share their number of output steps")
        offs = rec["out_offset"][first:first + count].astype(np.int64)
        if count > 1 and np.any(np.diff(offs) != n):
            raise ValueError("the members are not laid out one after another")
        mean = torch.empty((max(n, 1), 3), dtype=torch.float64, device=self.device)
        ws_bytes = self.lib.spinsim_spin_mean_workspace_size(count, n)
        ws = torch.empty(ws_bytes, dtype=torch.uint8, device=self.device)
        stream = torch.cuda.current_stream(self.device).cuda_stream
        _lib.check(self.lib.spinsim_spin_mean(self.spin.data_ptr(), int(offs[0]), n, count, n, mean.data_ptr(),
                                              ws.data_ptr(), ws_bytes, stream))
        return mean[:n]

    def __del__(self):
        try:
            if getattr(self, "_handle", None) is not None and self._handle.value:
                self.lib.spinsim_batch_destroy(self._handle)
            if getattr(self, "_owns_plan", False) and self._plan.value:
                self.lib.spinsim_plan_destroy(self._plan)
        except Exception:
            pass


class Evaluator:
    """Evaluate lists of instances into host memory with the stages overlapped.

    The list is split into ``chunks`` contiguous groups of about equal output bytes.  Group k's host set-up
    (descriptors, field packing into pinned staging), uploads and kernels run while group k-1's
    outputs are copied to pinned host memory, one copy per group; uploads, kernels and copies have
    a stream each.  The copies are usually the longest stage (every output crosses PCIe), so the
    end-to-end time approaches the time to set up and run the first group plus the time of all the
    copies.  ``evaluate`` returns one ``Results`` per instance whose arrays are numpy views of
    page-locked host buffers.  Remaining keyword arguments go to ``Batch``; with ``lanes``
    fixed and ``force_mixed=True`` the results are bit-identical to one ``Batch`` of the whole
    list, otherwise a group may pick other lanes or a single-spin kernel and the results agree to
    rounding.
    """

    def __init__(self, chunks=8, **batch_kwargs):
        import torch
        self.chunks = max(1, int(chunks))
        self.kw = batch_kwargs
        self.plans = batch_kwargs.pop("plan_cache", None)
        if self.plans is None:
            self.plans = {}
        self.upload = torch.cuda.Stream()
        self.compute = torch.cuda.Stream()
        self.copy = torch.cuda.Stream()
        self.h2d_bytes = self.d2h_bytes = 0

    @staticmethod
    def _pinned(nbytes):
        import torch
        return torch.empty(max(256, int(nbytes)), dtype=torch.uint8, pin_memory=True)

    def groups(self, instances):
        """Contiguous (first, end) groups of about equal output bytes, since the device-to-host copies
        are the longest stage: about (t1 - t0) / dt_out output steps, spin one weighted 224 / 128 (the
        bytes of time, U, state and spin per output step)."""
        n = len(instances)
        if not n:
            return []
        t0 = np.fromiter(map(_T0, instances), np.float64, n)
        t1 = np.fromiter(map(_T1, instances), np.float64, n)
        dt_out = np.fromiter(map(_DT_OUT, instances), np.float64, n)
        spins = list(map(_SPIN, instances))
        ids = list(map(id, spins))
        spin_one = {k for k, v in dict(zip(ids, spins)).items() if v.dimension == 3}  # few distinct objects
        one = np.fromiter(map(spin_one.__contains__, ids), np.bool_, n)
        work = np.maximum((t1 - t0) / dt_out, 1.0) * np.where(one, 224.0 / 128.0, 1.0)
        cum = np.cumsum(work)
        cuts = [0]
        for g in range(1, self.chunks):
            k = int(np.searchsorted(cum, cum[-1] * g / self.chunks))
            if k > cuts[-1]:
                cuts.append(k)
        cuts.append(n)
        return [(a, b) for a, b in zip(cuts, cuts[1:]) if b > a]

    def evaluate(self, instances):
        import torch
        instances = list(instances)
        if not instances:
            return []
        outs, self.h2d_bytes, self.d2h_bytes = [], 0, 0
        for a, b in self.groups(instances):
            with torch.cuda.nvtx.range(f"spinsim.evaluate.group[{a}:{b}]"):
                # Uploads on their own stream, so that they run during the previous group's kernels:
                # small host-to-device copies are several times slower while a large device-to-host
                # copy holds the link.
                with torch.cuda.stream(self.upload):
                    batch = Batch(instances[a:b], plan_cache=self.plans, staging=self._pinned, **self.kw)
                    ready = torch.cuda.Event()
                    ready.record(self.upload)
                self.compute.wait_event(ready)
                with torch.cuda.stream(self.compute):
                    batch.run()
                    done = torch.cuda.Event()
                    done.record(self.compute)
            self.copy.wait_event(done)
            # time, U, state and spin lie back to back at the start of the batch's device block: one copy
            nbytes = batch.output_bytes
            host = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
            with torch.cuda.stream(self.copy):
                host.copy_(batch.memory[:nbytes], non_blocking=True)
            outs.append((batch, host))
            self.h2d_bytes += batch.h2d_bytes
            self.d2h_bytes += nbytes
        self.copy.synchronize()
        return HostResults([(batch._inst_np.copy(), batch.host_views(host), host) for batch, host in outs])


class HostResults:
    """The ``Results`` of an ``Evaluator.evaluate`` call, in instance order: a sequence whose items
    are made on access from page-locked host arrays that already hold every output."""

    def __init__(self, groups):
        self._groups = groups
        self._index = []
        for g, (desc, _, _) in enumerate(groups):
            self._index += [(g, k) for k in range(len(desc))]

    def __len__(self):
        return len(self._index)

    def __getitem__(self, i):
        if isinstance(i, slice):
            return [self[j] for j in range(*i.indices(len(self)))]
        g, k = self._index[i]
        desc, (time, u, state, spin), host = self._groups[g]
        r = desc[k]
        out_off, u_off, st_off = int(r["out_offset"]), int(r["u_offset"]), int(r["state_offset"])
        n_out, d = int(r["n_out"]), int(r["dim"])
        return Results(time[out_off:out_off + n_out], u[u_off // 2:u_off // 2 + n_out * d * d].reshape(n_out, d, d),
                       state[st_off // 2:st_off // 2 + n_out * d].reshape(n_out, d), None,
                       spin=spin[out_off:out_off + n_out], keep=host)

    def __iter__(self):
        return (self[i] for i in range(len(self)))


def evaluate_many(instances, chunks=8, **batch_kwargs):
    """Evaluate a list of instances (see ``Instance``) into host ``Results`` with set-up, kernels
    and device-to-host copies overlapped across ``chunks`` groups (``Evaluator``)."""
    return Evaluator(chunks=chunks, **batch_kwargs).evaluate(instances)
