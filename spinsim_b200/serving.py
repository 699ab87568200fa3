"""Continuous-batching server for evaluate() requests.

Requests (one ``evaluate`` each: spin, field, time span, steps, initial state) arrive over time.
The server keeps a queue and a set of in-flight launches on several CUDA streams:

* **device memory** — the server takes ``hbm_budget`` bytes of HBM once, at start-up, as one
  arena; every launch carves its outputs, workspace and field tables from it (first fit, 256-byte
  aligned), so the serving loop never calls the CUDA allocator (whose cudaMalloc stalls the host
  for tens of milliseconds);
* **admission** — a request is admitted when a stream slot is free and its device footprint (an
  upper bound on the bytes of its outputs, scratch and field) fits the arena's largest free block;
* **continuous batching** — all requests admitted together form one persistent launch (the
  ``Batch`` path: one time-evolution launch over a longest-first tile queue, then the segmented
  state scan); requests that arrive while earlier launches run form the next launch on another
  stream, so their work overlaps on the device;
* **completion** — each launch records an event; when it has passed, the launch's requests are
  resolved with their ``Results`` (views of the arena; numpy on access, or copied to the host when
  ``copy_to_host``).  A launch's block returns to the arena when its last ``Results`` is released,
  so results the caller keeps hold budget, and results it drops free it.

Every request runs in the same kernel (the mixed-spin plan, one lane per output step, fixed scan
tiles), so its result does not depend on what else is in the launch: alone and in the mix agree
bit for bit.  Latency is measured on the host clock from arrival to completion.
"""
import bisect
import collections
import concurrent.futures
import gc
import math
import queue as queue_mod
import threading
import time
import weakref
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
    # a Request is also what a Batch reads as an instance (one evaluate() call, built-in field)
    sweep_parameters = (0.0,)
    intervals = None

    def instance(self):
        return Instance(self.spin, self.time_start, self.time_end, self.time_step_integration,
                        self.time_step_output, self.state_init, field=self.field)

    def steps(self):
        """Integration steps of the request (N output steps x K fine steps; computed once)."""
        got = self.meta.get("_steps")
        if got is None:
            n = max(0, int((float(self.time_end) - float(self.time_start)) / float(self.time_step_output)))
            k = int(math.floor(float(self.time_step_output) / float(self.time_step_integration) + 0.5))
            got = self.meta["_steps"] = n * max(k, 1)
        return got

    def footprint(self):
        got = self.meta.get("_footprint")
        if got is None:
            got = self.meta["_footprint"] = self._footprint()
        return got

    def _footprint(self):
        """Upper bound on the device bytes the request takes in a launch, even alone in it.

        Outputs (time 8, U 16 d^2, state 16 d, spin 24 bytes per output step); the launch workspace
        (a 120-byte instance and 224-byte field descriptor, time-evolution tiles of 16 bytes per 32
        steps at most, and per scan tile of 32 steps a 16-byte tile and two 144-byte operators: the
        tile's product and prefix, 9.5 bytes per step, counted as 3 d^2; on the tensor path the
        instance's 3,856-byte kernel constants and 32 bytes per step of SU(2) pairs); the field (tables or tones, 32-byte aligned chunks,
        and eight 32-byte table descriptors); 256-byte alignment of every piece."""
        d = self.spin.dimension
        n = max(0, int((float(self.time_end) - float(self.time_start)) / float(self.time_step_output)))
        fld = 256
        tables = getattr(self.field, "tables", None)
        if tables is not None:
            fld += sum(16 * t.size + 48 for t, _, _, _ in tables.values())
        elif self.field is not None and hasattr(self.field, "packed"):
            fld += 8 * self.field.packed()[0].size + 24
        return n * (65 + 16 * d + 19 * d * d) + 4160 * d * d + 6400 + 4112 + fld

class Completed:
    """A served request: its ``results`` (made on first access from the launch's arrays), the
    times it was admitted and completed, and its ``latency`` (completion - arrival)."""

    __slots__ = ("request", "admitted", "completed", "_batch", "_k", "_results")

    def __init__(self, request, batch, k, admitted, completed):
        self.request, self.admitted, self.completed = request, admitted, completed
        self._batch, self._k, self._results = batch, k, None

    @property
    def results(self):
        if self._results is None and self._batch is not None:
            self._results = self._batch.result(self._k, keep=self._batch.lease)
        return self._results

    @results.setter
    def results(self, value):
        self._results = value
        self._batch = None  # releases the launch's arrays (and its arena block) once nothing else holds them

    @property
    def latency(self):
        return self.completed - self.request.arrival


class Arena:
    """One device allocation handed out in 256-byte aligned blocks (first fit, coalescing frees).

    ``take`` and ``largest_free`` may be called from several threads; ``give`` may be called from
    any thread at any time, including from a finalizer that runs while another thread is inside
    ``take`` (a client dropping its ``Results`` while the serving thread admits a launch).  So
    ``give`` only queues the block on a lock-free ``SimpleQueue``, and the free list is changed
    only under the lock, where the queued blocks are merged back first."""

    ALIGN = 256

    def __init__(self, nbytes, device="cuda"):
        import torch
        self.size = (int(nbytes) + self.ALIGN - 1) // self.ALIGN * self.ALIGN
        self.buffer = torch.empty(self.size, dtype=torch.uint8, device=device)
        self._starts = [0]          # free blocks, sorted by offset
        self._sizes = {0: self.size}
        self._returned = queue_mod.SimpleQueue()  # blocks given back, not yet merged
        self._lock = threading.Lock()
        self._in_use = 0

    @property
    def in_use(self):
        """Bytes handed out and not yet given back."""
        with self._lock:
            self._merge_returned()
            return self._in_use

    def largest_free(self):
        with self._lock:
            self._merge_returned()
            return max(self._sizes.values(), default=0)

    def take(self, nbytes):
        """Offset of a free block of ``nbytes`` (rounded up to the alignment), or None."""
        n = (int(nbytes) + self.ALIGN - 1) // self.ALIGN * self.ALIGN
        with self._lock:
            self._merge_returned()
            for i, off in enumerate(self._starts):
                size = self._sizes[off]
                if size >= n:
                    del self._sizes[off]
                    if size == n:
                        del self._starts[i]
                    else:
                        self._starts[i] = off + n
                        self._sizes[off + n] = size - n
                    self._in_use += n
                    return off, n
        return None

    def give(self, off, n):
        """Return the block [off, off + n) (from ``take``); safe from any thread or finalizer."""
        self._returned.put((off, n))

    def _merge_returned(self):
        while True:
            try:
                off, n = self._returned.get_nowait()
            except queue_mod.Empty:
                return
            self._insert(off, n)

    def _insert(self, off, n):
        self._in_use -= n
        i = bisect.bisect_left(self._starts, off)
        if i < len(self._starts) and off + n == self._starts[i]:  # merge with the next block
            nxt = self._starts.pop(i)
            n += self._sizes.pop(nxt)
        if i > 0 and self._starts[i - 1] + self._sizes[self._starts[i - 1]] == off:  # with the previous
            self._sizes[self._starts[i - 1]] += n
        else:
            self._starts.insert(i, off)
            self._sizes[off] = n

    def free_blocks(self):
        """The free list as sorted (offset, size) pairs, after merging returned blocks."""
        with self._lock:
            self._merge_returned()
            return [(o, self._sizes[o]) for o in self._starts]


class _Lease:
    """Holds one launch's arena block; the block returns to the arena when the lease is released
    (when the launch's Batch and every Results made from it are gone)."""

    def __init__(self, arena, off, n):
        self.block = (off, n)
        weakref.finalize(self, arena.give, off, n)


class ArenaFull(Exception):
    pass


class BudgetHeld(RuntimeError):
    """Nothing is running and the next request does not fit: results still referenced hold the arena."""


class LaunchError(Exception):
    """A launch could not be made; ``requests`` were taken from the queue for it."""

    def __init__(self, requests, error):
        super().__init__(str(error))
        self.requests = requests
        self.error = error


class Server:
    """Continuous-batching evaluator.  ``hbm_budget`` bytes of HBM (one arena, taken at start-up)
    hold the outputs and scratch of launches in flight and of results the caller still holds; up to
    ``streams`` launches run concurrently, of at most ``max_batch`` requests and
    ``max_steps_per_launch`` integration steps each (a longer request runs alone), which bounds how
    long one launch holds the requests admitted with it.  Concurrent launches share the SMs, so more
    streams finish every launch later; the defaults (4 streams, 2e8 steps) gave the lowest p99 on
    one B200 for a mix of 10 us - 100 ms pulse-train requests near its capacity."""

    def __init__(self, precision=Precision.FP32_BULK, hbm_budget=8 << 30, streams=4, max_batch=4096,
                 copy_to_host=False, number_of_squares=24, threads_per_block=128, max_registers=128,
                 max_steps_per_launch=200_000_000, warm_up=True, staging_bytes=32 << 20):
        import torch
        self.precision = Precision(precision)
        self.hbm_budget = int(hbm_budget)
        self.arena = Arena(self.hbm_budget)
        self.streams = [torch.cuda.Stream() for _ in range(streams)]
        # pinned host staging for each stream's field upload (reused once the stream's launch is done)
        self.staging = [torch.empty(int(staging_bytes), dtype=torch.uint8, pin_memory=True) for _ in range(streams)]
        self.max_batch = max_batch
        self.copy_to_host = copy_to_host
        self.kw = dict(precision=self.precision, number_of_squares=number_of_squares, lanes=1,
                       threads_per_block=threads_per_block, max_registers=max_registers,
                       exponentiation_half=ExponentiationMethod.ANALYTIC, force_mixed=True)
        self.max_steps = int(max_steps_per_launch)
        self.plans = {}
        self.stats = collections.Counter()
        self.launch_log = []  # (requests, steps, admitted at, completed at)
        if warm_up:
            # create the plan and load the kernels before the first request arrives
            probe = Request(SpinQuantumNumber.HALF, TabulatedField({0: ([0.0, 1e-6], [0.0, 0.0])}, order=0),
                            0.0, 2e-6, 1e-7, 1e-6, SpinQuantumNumber.HALF.plus_z)
            with torch.cuda.stream(self.streams[0]):
                Batch([probe.instance()], plan_cache=self.plans, **self.kw).run()
            self.streams[0].synchronize()

    def _launch(self, reqs, si):
        """Place a launch in the arena, upload its descriptors and run it on ``stream`` (free, so the
        uploads' stream synchronisation does not wait on other work).  Raises ArenaFull when the
        launch does not fit."""
        import torch
        lease = []

        def memory(nbytes):
            blk = self.arena.take(nbytes)
            if blk is None:
                raise ArenaFull(nbytes)
            lease.append(_Lease(self.arena, *blk))
            return self.arena.buffer[blk[0]:blk[0] + blk[1]]

        stream = self.streams[si]
        try:
            with torch.cuda.stream(stream), torch.cuda.nvtx.range(f"spinsim.serve.launch[{len(reqs)}]"):
                b = Batch(reqs, plan_cache=self.plans, memory=memory, staging=self.staging[si], **self.kw)
                b.lease = lease[0]
                b.run()
                ev = torch.cuda.Event()
                if self.copy_to_host:
                    b.host = [t.to("cpu", non_blocking=True) for t in (b.time, b.u, b.state, b.spin)]
                ev.record(stream)
        except BaseException:
            # uploads or kernels already queued on the stream may still write into the block: let
            # them finish before the lease (and with it the block and the stream) can be reused
            stream.synchronize()
            raise
        return b, ev, lease[0]

    def run(self, requests, clock=time.perf_counter, idle_sleep=20e-6, on_complete=None, keep_results=True):
        """Serve ``requests`` (arrival times in seconds from the start) in open loop; returns the
        list of ``Completed`` in completion order.  ``on_complete(completed)`` is called as each
        request completes; with ``keep_results=False`` the returned ``Completed`` carry no results
        (their device memory goes back to the arena once ``on_complete`` returns)."""
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        for r in pending:
            if r.footprint() > self.arena.size:
                raise ValueError(f"request {r.id} needs {r.footprint()} bytes, above the HBM budget")
        gc_was_enabled = gc.isenabled()
        gc.disable()  # a full collection over the live results would stall the loop for tens of ms
        try:
            return self._run(pending, clock, idle_sleep, on_complete, keep_results)
        except LaunchError as e:
            raise e.error
        finally:
            if gc_was_enabled:
                gc.enable()

    def _run(self, pending, clock, idle_sleep, on_complete, keep_results):
        queue = collections.deque()
        inflight = []  # (batch, event, requests, stream index, admitted time)
        free_streams = list(range(len(self.streams)))
        done = []
        t0 = clock()
        while pending or queue or inflight:
            now = clock() - t0
            while pending and pending[0].arrival <= now:
                queue.append(pending.popleft())
            inflight = self._complete(inflight, free_streams, done, clock, t0, on_complete, keep_results)
            while queue and free_streams:
                if not self._admit(queue, inflight, free_streams, clock, t0):
                    break
            if not (queue and free_streams) and (inflight or pending):
                if pending and not queue and not inflight:
                    wait = pending[0].arrival - (clock() - t0)
                    if wait > 0:
                        time.sleep(min(wait, 1e-3))
                else:
                    time.sleep(idle_sleep)
        return done

    # ------------------------------------------------------------------ asynchronous serving
    def start(self):
        """Serve submitted requests on a background thread (``submit`` returns futures)."""
        import torch
        if getattr(self, "_thread", None) is not None:
            raise RuntimeError("the server is already running")
        self._inbox = queue_mod.SimpleQueue()
        self._stopping = threading.Event()
        self._t0 = time.perf_counter()
        self._error = None
        device = torch.cuda.current_device()
        self._thread = threading.Thread(target=self._serve_forever, args=(device,), name="spinsim-server", daemon=True)
        self._thread.start()
        return self

    def submit(self, request, timeout=None):
        """Queue ``request`` (a ``Request``; its arrival is now) and return a
        ``concurrent.futures.Future`` that resolves to its ``Results`` (views of the arena, which the
        request's block holds until they are released) or to the launch's exception.  With
        ``timeout`` (seconds), a request not yet admitted to a launch by then fails with
        ``TimeoutError`` (checked when it reaches the head of the queue); cancelling the future
        before admission withdraws the request."""
        if getattr(self, "_thread", None) is None or self._stopping.is_set():
            raise RuntimeError("the server is not running: call start()")
        if request.footprint() > self.arena.size:
            raise ValueError(f"request {request.id} needs {request.footprint()} bytes, above the HBM budget")
        future = concurrent.futures.Future()
        request.arrival = time.perf_counter() - self._t0
        if timeout is not None:
            request.meta["deadline"] = request.arrival + float(timeout)
        self._inbox.put((request, future))
        return future

    def close(self, wait=True):
        """Stop accepting requests, finish the queued and running ones, and stop the thread."""
        thread = getattr(self, "_thread", None)
        if thread is None:
            return
        self._stopping.set()
        if wait:
            thread.join()
        self._thread = None
        if self._error is not None:
            raise self._error

    def __enter__(self):
        return self.start()

    def __exit__(self, *exc):
        self.close()

    def _serve_forever(self, device, idle_sleep=20e-6):
        import torch
        torch.cuda.set_device(device)
        futures = {}
        queue = collections.deque()
        inflight = []
        free_streams = list(range(len(self.streams)))
        clock = time.perf_counter
        t0 = self._t0

        def resolve(c):
            futures.pop(id(c.request)).set_result(c.results)

        try:
            while True:
                while True:
                    try:
                        req, fut = self._inbox.get_nowait()
                    except queue_mod.Empty:
                        break
                    if fut.set_running_or_notify_cancel():
                        futures[id(req)] = fut
                        queue.append(req)
                inflight = self._complete(inflight, free_streams, [], clock, t0, resolve, False)
                now = clock() - t0
                while queue and queue[0].meta.get("deadline", math.inf) < now:
                    r = queue.popleft()
                    futures.pop(id(r)).set_exception(
                        TimeoutError(f"request {r.id} was not admitted within its timeout"))
                    self.stats["timeouts"] += 1
                while queue and free_streams:
                    try:
                        if not self._admit(queue, inflight, free_streams, clock, t0):
                            break
                    except LaunchError as e:  # a launch that cannot be made fails its requests
                        for r in e.requests:
                            futures.pop(id(r)).set_exception(e.error)
                    except BudgetHeld as e:  # the head request cannot run until results are released
                        futures.pop(id(queue.popleft())).set_exception(e)
                if self._stopping.is_set() and not queue and not inflight and self._inbox.empty():
                    break
                time.sleep(idle_sleep)
        except Exception as e:  # pragma: no cover - reported by close()
            self._error = e
            for fut in futures.values():
                fut.set_exception(e)

    def _complete(self, inflight, free_streams, done, clock, t0, on_complete, keep_results):
        """Resolve the launches whose event has passed; returns the launches still running (host time
        spent here accumulates in stats["host_complete_s"])."""
        h0 = time.perf_counter()
        still = []
        for item in inflight:
            b, ev, reqs, si, adm = item
            if not ev.query():
                still.append(item)
                continue
            tdone = clock() - t0
            for k, r in enumerate(reqs):
                c = Completed(r, b, k, adm, tdone)
                if on_complete is not None:
                    on_complete(c)
                if not keep_results:
                    c.results = None
                done.append(c)
            free_streams.append(si)
            self.stats["launches"] += 1
            self.launch_log.append((len(reqs), b.total_steps, adm, tdone))
        self.stats["host_complete_s"] += time.perf_counter() - h0
        return still

    def _admit(self, queue, inflight, free_streams, clock, t0):
        """Start one launch from the head of the queue on a free stream; False when nothing fits
        (wait for a completion or a released result).  Host time spent here (packing descriptors and
        issuing the launch) accumulates in stats["host_admit_s"]."""
        h0 = time.perf_counter()
        try:
            return self._admit_one(queue, inflight, free_streams, clock, t0)
        finally:
            self.stats["host_admit_s"] += time.perf_counter() - h0

    def _admit_one(self, queue, inflight, free_streams, clock, t0):
        avail = self.arena.largest_free()
        take, nbytes, steps = [], 0, 0
        while queue and len(take) < self.max_batch:
            fp = queue[0].footprint()
            st = queue[0].steps()
            if nbytes + fp > avail:
                break
            if take and steps + st > self.max_steps:
                break
            take.append(queue.popleft())
            nbytes += fp
            steps += st
        if not take:
            self.stats["budget_waits"] += 1
            if not inflight:
                gc.collect()  # results released only through a reference cycle
                if self.arena.largest_free() < queue[0].footprint():
                    raise BudgetHeld("the HBM budget is held by results still referenced: release Results "
                                     "(or serve with keep_results=False) or raise hbm_budget")
                return True
            return False
        si = free_streams.pop()
        while True:
            try:
                b, ev, _ = self._launch(take, si)
                break
            except ArenaFull:
                # footprints are upper bounds, so this follows only from fragmentation: launch fewer
                self.stats["arena_retries"] += 1
                if len(take) == 1:
                    free_streams.append(si)
                    queue.appendleft(take[0])
                    if not inflight:
                        raise RuntimeError("a request does not fit the arena's free blocks")
                    return False
                half = len(take) // 2
                queue.extendleft(reversed(take[half:]))
                take = take[:half]
            except Exception as e:
                free_streams.append(si)
                raise LaunchError(take, e) from e
        inflight.append((b, ev, take, si, clock() - t0))
        self.stats["admitted"] += len(take)
        return True


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
