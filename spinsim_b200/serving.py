"""Continuous-batching server for evaluate() requests.

Requests (one ``evaluate`` each: spin, field, time span, steps, initial state) arrive over time.
The server keeps a queue and a set of in-flight launches on several CUDA streams:

* **admission** — a request is admitted when a stream slot is free and its device footprint
  (outputs + scan workspace, counted from the sizes the C ABI reports) fits the HBM budget;
* **continuous batching** — all requests admitted together form one persistent launch (the
  ``Batch`` path: one time-evolution launch over a longest-first tile queue, then the segmented
  state scan); requests that arrive while earlier launches run form the next launch on another
  stream, so their work overlaps on the device;
* **completion** — each launch records an event; when it has passed, the launch's requests are
  resolved with their ``Results`` (device tensors; numpy on access, or copied to the host when
  ``copy_to_host``), and their memory returns to the budget.

Every request runs in the same kernel (the mixed-spin plan, one lane per output step, fixed scan
tiles), so its result does not depend on what else is in the launch: alone and in the mix agree
bit for bit.  Latency is measured on the host clock from arrival to completion.
"""
import collections
import math
import time
from dataclasses import dataclass, field as dc_field
from typing import Any, Optional

import numpy as np

from . import ExponentiationMethod, Precision, SpinQuantumNumber, TabulatedField
from .batch import Batch, Instance

TAU = 2 * math.pi


@dataclass
class Request:
    spin: SpinQuantumNumber
    field: Any
    time_start: float
    time_end: float
    time_step_integration: float
    time_step_output: float
    state_init: Any
    arrival: float = 0.0
    id: int = 0
    meta: dict = dc_field(default_factory=dict)

    def instance(self):
        return Instance(self.spin, self.time_start, self.time_end, self.time_step_integration,
                        self.time_step_output, self.state_init, field=self.field)

    def steps(self):
        """Integration steps of the request (N output steps x K fine steps)."""
        n = max(0, int((float(self.time_end) - float(self.time_start)) / float(self.time_step_output)))
        k = int(math.floor(float(self.time_step_output) / float(self.time_step_integration) + 0.5))
        return n * max(k, 1)

    def footprint(self):
        """Device bytes of the request's outputs (time, U, state, spin) and scan scratch."""
        d = self.spin.dimension
        n = max(0, int((float(self.time_end) - float(self.time_start)) / float(self.time_step_output)))
        return n * (8 + 16 * d * d + 16 * d + 24) + n * 16 * d * d // 8 + 4096


@dataclass
class Completed:
    request: Request
    results: Any
    admitted: float
    completed: float

    @property
    def latency(self):
        return self.completed - self.request.arrival


class Server:
    """Continuous-batching evaluator.  ``hbm_budget`` bytes of outputs and scratch may be in flight
    on up to ``streams`` concurrent launches of at most ``max_batch`` requests and
    ``max_steps_per_launch`` integration steps each (a longer request runs alone), which bounds how
    long one launch holds the requests admitted with it."""

    def __init__(self, precision=Precision.FP32_BULK, hbm_budget=8 << 30, streams=4, max_batch=4096,
                 copy_to_host=False, number_of_squares=24, threads_per_block=128, max_registers=128,
                 max_steps_per_launch=400_000_000, warm_up=True):
        import torch
        self.precision = Precision(precision)
        self.hbm_budget = int(hbm_budget)
        self.streams = [torch.cuda.Stream() for _ in range(streams)]
        self.max_batch = max_batch
        self.copy_to_host = copy_to_host
        self.kw = dict(precision=self.precision, number_of_squares=number_of_squares, lanes=1,
                       threads_per_block=threads_per_block, max_registers=max_registers,
                       exponentiation_half=ExponentiationMethod.ANALYTIC, force_mixed=True)
        self.max_steps = int(max_steps_per_launch)
        self.plans = {}
        self.stats = collections.Counter()
        self.launch_log = []  # (requests, steps, admitted at, completed at)
        if warm_up:  # create the plan and load the kernels before the first request arrives
            probe = Request(SpinQuantumNumber.HALF, TabulatedField({0: ([0.0, 1e-6], [0.0, 0.0])}, order=0),
                            0.0, 2e-6, 1e-7, 1e-6, SpinQuantumNumber.HALF.plus_z)
            b, ev = self._launch([probe], self.streams[0])
            ev.synchronize()

    def _launch(self, reqs, stream):
        import torch
        with torch.cuda.stream(stream):
            b = Batch([r.instance() for r in reqs], plan_cache=self.plans, **self.kw)
            b.run()
            if self.copy_to_host:
                b.host = [t.to("cpu", non_blocking=True) for t in (b.time, b.u, b.state, b.spin)]
            ev = torch.cuda.Event()
            ev.record(stream)
        return b, ev

    def run(self, requests, clock=time.perf_counter, idle_sleep=20e-6):
        """Serve ``requests`` (arrival times in seconds from the start) in open loop; returns the
        list of ``Completed`` in completion order."""
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        for r in pending:
            if r.footprint() > self.hbm_budget:
                raise ValueError(f"request {r.id} needs {r.footprint()} bytes, above the HBM budget")
        queue = collections.deque()
        inflight = []  # (batch, event, requests, bytes, stream index, admitted time)
        free_streams = list(range(len(self.streams)))
        used = 0
        done = []
        t0 = clock()
        while pending or queue or inflight:
            now = clock() - t0
            while pending and pending[0].arrival <= now:
                queue.append(pending.popleft())
            # completions
            still = []
            for item in inflight:
                b, ev, reqs, nbytes, si, adm = item
                if ev.query():
                    tdone = clock() - t0
                    for k, r in enumerate(reqs):
                        done.append(Completed(r, b.result(k), adm, tdone))
                    used -= nbytes
                    free_streams.append(si)
                    self.stats["launches"] += 1
                    self.launch_log.append((len(reqs), b.total_steps, adm, tdone))
                else:
                    still.append(item)
            inflight = still
            # admission: one launch per free stream from the head of the queue
            while queue and free_streams:
                take, nbytes, steps = [], 0, 0
                while queue and len(take) < self.max_batch:
                    fp = queue[0].footprint()
                    st = queue[0].steps()
                    if used + nbytes + fp > self.hbm_budget:
                        break
                    if take and steps + st > self.max_steps:
                        break
                    take.append(queue.popleft())
                    nbytes += fp
                    steps += st
                if not take:
                    self.stats["budget_waits"] += 1
                    break
                si = free_streams.pop()
                b, ev = self._launch(take, self.streams[si])
                used += nbytes
                inflight.append((b, ev, take, nbytes, si, clock() - t0))
                self.stats["admitted"] += len(take)
            if not (queue and free_streams) and (inflight or pending):
                if pending and not queue and not inflight:
                    wait = pending[0].arrival - (clock() - t0)
                    if wait > 0:
                        time.sleep(min(wait, 1e-3))
                else:
                    time.sleep(idle_sleep)
        return done


# ---------------------------------------------------------------------------- synthetic workload
def pulse_sequence(rng, t_end, rabi=TAU * 25e3):
    """Piecewise-constant pulse train (zero-order-hold tables for channels x and y): random pi/2
    (10 us) and pi (20 us) pulses at Rabi frequency ``rabi`` along x with phase 0 or pi/2 (pi/2 puts
    the pulse on y), separated by gaps U[1, 50] us."""
    t, tx, ax, ay = 0.0, [0.0], [0.0], [0.0]
    while t < t_end:
        t += rng.uniform(1e-6, 50e-6)
        width = 10e-6 if rng.uniform() < 0.5 else 20e-6
        on_y = rng.uniform() < 0.5
        tx.append(t)
        ax.append(0.0 if on_y else rabi)
        ay.append(rabi if on_y else 0.0)
        t += width
        tx.append(t)
        ax.append(0.0)
        ay.append(0.0)
    tx = np.array(tx)
    return TabulatedField({0: (tx, np.array(ax)), 1: (tx, np.array(ay))}, order=0, zero_boundary=False)


def synthetic_requests(n, rate, seed=4, max_duration=100e-3):
    """n requests with Poisson arrivals at ``rate`` per second: 70% spin half / 30% spin one,
    durations log-uniform in [10 us, max_duration], dt_int from {10, 20, 50, 100} ns, dt_out 1 us,
    pulse-sequence fields."""
    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n))
    out = []
    for k in range(n):
        spin = SpinQuantumNumber.HALF if rng.uniform() < 0.7 else SpinQuantumNumber.ONE
        dur = float(np.exp(rng.uniform(np.log(10e-6), np.log(max_duration))))
        dti = float(rng.choice([10e-9, 20e-9, 50e-9, 100e-9]))
        fld = pulse_sequence(rng, dur)
        out.append(Request(spin, fld, 0.0, dur, dti, 1e-6, spin.plus_z, arrival=float(arrivals[k]), id=k))
    return out


def latency_summary(done):
    lat = np.array([c.latency for c in done])
    steps = sum(int(round((c.request.time_end - c.request.time_start) / c.request.time_step_output)) *
                int(round(c.request.time_step_output / c.request.time_step_integration)) for c in done)
    span = max(c.completed for c in done) - min(c.request.arrival for c in done)
    return {"requests": len(done), "p50_ms": 1e3 * float(np.percentile(lat, 50)),
            "p99_ms": 1e3 * float(np.percentile(lat, 99)), "mean_ms": 1e3 * float(lat.mean()),
            "steps_per_s": steps / span, "span_s": span}
