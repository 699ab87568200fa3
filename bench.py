"""Benchmark: steps/s of the batched FP32-bulk form vs the plain FP64 form on B200.

Workload (one "step" = one pass of the hot path over the whole batch): 1024 instances, 70% spin half
(analytic exponential) / 30% spin one (Lie-Trotter, 24 squarings), durations log-uniform in
[10 us, 10 ms], dt_int 10 ns, dt_out 1 us, Magnus CF4, rotating frame, field = 8 tones per axis
(frequency U[0, 1 MHz], amplitude U[0, 2pi 10 kHz], phase U[0, 2pi)) from a per-instance seed,
q = 0; all instances in one persistent launch replayed from a CUDA graph, followed by the FP64
prefix scan (state) with the spin expectation fused.  Synthetic inputs (seeded).

The headline ``value`` is the FP32-bulk steps/s with inputs resident in HBM; ``plain_fp64`` is the
plain FP64 form on the same batch, ``state_err`` the final-state error of FP32-bulk against FP64.
``e2e`` repeats the measurement through the public API with host inputs and host outputs
(descriptors and tone tables copied in, time / time_evolution / state / spin copied out, every
step).  ``--impl reference`` times the reference's CPU algorithm (the oracle restatement, all host
threads) on a bounded sample of the same workload.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Multi-GPU: torchrun --nproc-per-node N bench.py --gpus N (weak scaling: every rank runs its own
batch of the same shape from its own seeds; no collective on the data path).
"""
import argparse
import json
import os
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))

METRIC = "steps/s batched FP32-bulk vs plain FP64 at state err<=1e-6; p50/p99 latency"
N_INSTANCES = 1024
TAU = 2 * np.pi


# ------------------------------------------------------------------------------------ workload
def workload(seed_base=0, n=N_INSTANCES):
    """Instance specs: (spin_dim, duration, tone parameter vector)."""
    rng = np.random.default_rng(3 + 7919 * seed_base)
    specs = []
    for k in range(n):
        dim = 2 if rng.uniform() < 0.7 else 3
        dur = float(np.exp(rng.uniform(np.log(10e-6), np.log(10e-3))))
        p = np.zeros(4 + 72)
        r = np.random.default_rng(10_000 + k + 1_000_003 * seed_base)
        for axis in range(3):
            for tone in range(8):
                b = 4 + 24 * axis + 3 * tone
                p[b] = TAU * r.uniform(0.0, 1e6)
                p[b + 1] = r.uniform(0.0, TAU * 10e3)
                p[b + 2] = r.uniform(0.0, TAU)
        specs.append((dim, dur, p))
    return specs


def tone_field(ss, p):
    tones = {a: np.array([(p[4 + 24 * a + 3 * j], p[5 + 24 * a + 3 * j], p[6 + 24 * a + 3 * j]) for j in range(8)])
             for a in range(3)}
    return ss.ToneField(tones, bias=list(p[:4]))


def instances(ss, specs):
    from spinsim_b200.batch import Instance
    out = []
    for dim, dur, p in specs:
        spin = ss.SpinQuantumNumber.HALF if dim == 2 else ss.SpinQuantumNumber.ONE
        psi0 = spin.plus_z if dim == 2 else spin.plus_x
        out.append(Instance(spin, 0.0, dur, 10e-9, 1e-6, psi0, sweep_parameters=p, field=tone_field(ss, p)))
    return out


# Algorithmic work per integration step, counted from the kernels' arithmetic (a fused multiply-add
# is 2 flops; sin, cos, sqrt and division count 1 each).  Plain FP64, spin half: field 192 + 48 sin,
# windings 8 + 4 sincos, frame 24, generators 24, two analytic exponentials 40 + 8, two 2x2 complex
# products 128, time 1.  Spin one (Lie-Trotter, 24 squarings): field 192 + 48, windings 8 + 4,
# frame 14, generators 32, two exponentials 10,920 + 14, two 3x3 products 432, time 1.  FP32-bulk
# (tensor-path tone kernel, Magnus step): field samples 192 as FP64 tensor-core products (two Gauss
# points x three channels x 16 multiply-adds) + the phasor table's recurrences 9, frame 24 (the xy
# rotations and the phasors' steps; z's frame shift is in the samples' starting value), sum and
# difference of the samples 6, the exponential's linear part and the SU(2) product into the
# interval's FP64 operator 39; in FP32 the commutator 15 and the exponential's O(|g|^2) remainder 21.
# Spin one runs as SU(2) (no quadratic shift here).
FLOPS_FP64_PLAIN = {2: 417 + 60, 3: 11600 + 66}
FLOPS_BULK = {2: {"fp64": 270, "fp32": 36}, 3: {"fp64": 270, "fp32": 36}}
# DRAM bytes (read + write) of one full-size FP32-bulk time-evolution launch of this workload (the
# tensor-path kernel at 96 registers, writing the scan's tile partials and each output step's SU(2)
# pair beside U: 46 MB of the writes are that scan scratch, not outputs), from one capture of
# `ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum --clock-control none -k regex:evolve_dmma -c 1`
# on `bench.py --workload profile --profile-size full --precision fp32_bulk --max-registers 96 --variant 0`.
TRAFFIC_BYTES_PER_LAUNCH = 7328000 + 137223936


def algorithmic_bytes(specs):
    """Bytes one time-evolution launch must write: time (8) and U (16 d^2) per output step."""
    return sum(int(dur / 1e-6) * (8 + 16 * dim * dim) for dim, dur, _ in specs)


def algorithmic_flops(specs, form):
    total64 = total32 = 0.0
    for dim, dur, _ in specs:
        n = int(dur / 1e-6)
        steps = n * 100
        if form == "fp64":
            total64 += steps * FLOPS_FP64_PLAIN[dim]
        else:
            total64 += steps * FLOPS_BULK[dim]["fp64"]
            total32 += steps * FLOPS_BULK[dim]["fp32"]
    return total64, total32


# ------------------------------------------------------------------------------------ helpers
class ClockSampler:
    """SM clock and throttle reasons sampled through NVML every 2 ms during the timed regions."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
               "sw_power_cap": 0x4}

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.reasons = set()
        self.max_mhz = None
        self._stop = threading.Event()

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))

            def run():
                while not self._stop.is_set():
                    try:
                        self.samples.append(float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)))
                        r = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                        for name, bit in self.REASONS.items():
                            if r & bit:
                                self.reasons.add(name)
                    except Exception:
                        pass
                    self._stop.wait(0.002)

            self.thread = threading.Thread(target=run, daemon=True)
            self.thread.start()
        except Exception:
            self.thread = None
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self.thread is not None:
            self.thread.join(timeout=2)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median(self.samples)), "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
                "samples": len(self.samples)}


def peaks_from_file():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return json.load(open(p))
    return None


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def barrier_max(value, world):
    """Max over ranks of a float (device timing); identity on one rank."""
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device="cuda" if torch.cuda.is_available() else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ------------------------------------------------------------------------------------ CPU baseline
def cpu_sample(specs, seconds_target=8.0, n_threads=0):
    """Time the oracle (the reference's algorithm restated in C, all host threads) on a bounded sample
    of the workload: the first intervals of every instance, grown until it takes ~seconds_target."""
    from oracle import oracle as O
    fields = []
    for dim, dur, p in specs:
        fields.append((dim, p, int(dur / 1e-6)))
    field = O.Field(8)

    def run(frac):
        steps = 0
        t0 = time.perf_counter()
        for dim, p, n in fields:
            cnt = max(1, int(n * frac)) if n else 0
            if cnt == 0:
                continue
            O.time_evolution(dim, field, p, 0.0, 10e-9, 1e-6, n, first=0, count=cnt, n_threads=n_threads)
            steps += cnt * 100
        return steps, time.perf_counter() - t0

    frac = 0.002
    steps, el = run(frac)
    while el < seconds_target / 4 and frac < 1.0:
        frac = min(1.0, frac * max(2.0, seconds_target / max(el, 1e-3) / 2))
        steps, el = run(frac)
    return steps, el, frac


# ------------------------------------------------------------------------------------ our arm
class PerSpinBatches:
    """The plain FP64 form run as one launch per spin (spin half and spin one, each with its own
    autotuned register budget and launch shape), on two streams: a mixed-spin FP64 launch carries the
    register budget and code of the spin-one Lie-Trotter path into the spin-half steps, so splitting by
    spin is the faster way to run this batch in FP64."""

    def __init__(self, ss, insts, plans, tune):
        import torch
        from spinsim_b200.batch import Batch
        self.index = {2: [k for k, i in enumerate(insts) if i.spin.dimension == 2],
                      3: [k for k, i in enumerate(insts) if i.spin.dimension == 3]}
        self.n = len(insts)
        self.parts, self.config, self.tuning = {}, {}, {}
        for d, idx in self.index.items():
            if not idx:
                continue
            sub = [insts[k] for k in idx]
            cfg, timing = tune(sub, use_cache=False, precision=ss.Precision.FP64)
            self.parts[d] = Batch(sub, precision=ss.Precision.FP64, plan_cache=plans, **cfg)
            self.config[d], self.tuning[d] = cfg, timing
        self.total_steps = sum(b.total_steps for b in self.parts.values())
        self.streams = {d: torch.cuda.Stream() for d in self.parts}
        self._graph = None

    def run(self, with_state=True):
        import torch
        cur = torch.cuda.current_stream()
        for d, b in self.parts.items():
            self.streams[d].wait_stream(cur)
            with torch.cuda.stream(self.streams[d]):
                b.run(with_state=with_state)
        for d in self.parts:
            cur.wait_stream(self.streams[d])

    def capture(self):
        import torch
        self.run()
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.run()
        self._graph = g

    def replay(self):
        if self._graph is None:
            self.capture()
        self._graph.replay()

    def final_states(self):
        out = [None] * self.n
        for d, b in self.parts.items():
            for k, st in zip(self.index[d], b.final_states()):
                out[k] = st
        return out

    def launch_info(self):
        return {str(d): b.launch_info() for d, b in self.parts.items()}


def bench_ours(args, world, rank):
    import torch
    import spinsim_b200 as ss
    from spinsim_b200.batch import Batch
    dev = torch.device("cuda", torch.cuda.current_device())
    specs = workload(seed_base=rank)
    insts = instances(ss, specs)
    total_steps = sum(int(d / 1e-6) * 100 for _, d, _ in specs)
    plans = {}
    from spinsim_b200.autotune import tune
    if args.bulk_config:  # a fixed configuration (profiling runs: the one the untuned run chose)
        cfg_bulk, tune_bulk = json.loads(args.bulk_config), {}
    else:
        cfg_bulk, tune_bulk = tune(insts, use_cache=False, precision=ss.Precision.FP32_BULK)
    bulk = Batch(insts, precision=ss.Precision.FP32_BULK, plan_cache=plans, **cfg_bulk)
    plain = PerSpinBatches(ss, insts, plans, tune)
    assert bulk.total_steps == total_steps
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)  # > L2 (126 MB)

    def timed(batch, k, evolve_only=False):
        for _ in range(args.warmup):
            batch.run(with_state=not evolve_only)
        torch.cuda.synchronize()
        times = []
        stream = torch.cuda.current_stream(dev)
        for _ in range(k):
            flush.zero_()
            s = torch.cuda.Event(enable_timing=True)
            e = torch.cuda.Event(enable_timing=True)
            s.record(stream)
            if evolve_only:
                batch.run(with_state=False)
            else:
                batch.replay()
            e.record(stream)
            times.append((s, e))
            e.synchronize()  # host waits here (GIL released), so the clock sampler runs during the step
        torch.cuda.synchronize()
        return [s.elapsed_time(e) / 1e3 for s, e in times]

    bulk.capture()
    plain.capture()
    barrier(world)
    torch.cuda.synchronize()
    # clocks sampled over both timed regions (the FP32-bulk steps, then the plain FP64 steps)
    with ClockSampler(torch.cuda.current_device()) as clocks:
        t_bulk = timed(bulk, args.steps)
        t_plain = timed(plain, max(1, args.steps // 3))
    t_bulk_total = barrier_max(sum(t_bulk), world)
    t_plain_total = barrier_max(sum(t_plain), world) * args.steps / len(t_plain)

    # dominant kernel alone (time evolution), same stream, CUDA events
    t_evolve = timed(bulk, max(2, args.steps // 2), evolve_only=True)
    t_evolve_plain = timed(plain, 1, evolve_only=True)

    # accuracy of FP32-bulk against FP64 on this batch
    bulk.replay()
    plain.replay()
    torch.cuda.synchronize()
    fb, fp = bulk.final_states(), plain.final_states()
    errs = np.array([np.abs(a - b).max() if a.size else 0.0 for a, b in zip(fb, fp)])

    # end to end through the public API with host buffers: host descriptors and fields in, every
    # output (time, U, state, spin) out to page-locked host memory, chunks overlapped (Evaluator)
    from spinsim_b200.batch import Evaluator
    ev = Evaluator(chunks=args.e2e_chunks, precision=ss.Precision.FP32_BULK, plan_cache=plans, **cfg_bulk)
    e2e_times, h2d, d2h = [], 0, 0
    for it in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = ev.evaluate(insts)
        el = time.perf_counter() - t0
        if it >= args.warmup:
            e2e_times.append(el)
        h2d, d2h = ev.h2d_bytes, ev.d2h_bytes
        del res
    e2e_total = barrier_max(sum(e2e_times), world)

    info = bulk.launch_info()
    peaks = peaks_from_file()
    fp64_flops, fp32_flops = algorithmic_flops(specs, "bulk")
    evolve_s = float(np.mean(t_evolve))
    fp64_peak = measured_fp64_peak()
    achieved = fp64_flops / evolve_s / 1e12
    fp64_plain_flops, _ = algorithmic_flops(specs, "fp64")
    # plain FP64 per spin (separate launches): time of each part alone, for the per-spin FP64 rates
    plain_parts = {}
    for d, b in plain.parts.items():
        tp = timed(b, 1, evolve_only=True)
        part_flops, _ = algorithmic_flops([sp for sp in specs if sp[0] == d], "fp64")
        plain_parts[f"spin_{'half' if d == 2 else 'one'}"] = {
            "evolve_kernel_ms": 1e3 * tp[0], "fp64_tflops": part_flops / tp[0] / 1e12,
            "fp64_frac": part_flops / tp[0] / 1e12 / measured_fp64_peak()["tflops"], "steps": b.total_steps,
            "config": plain.config[d]}
    value = world * total_steps * args.steps / t_bulk_total
    out = {
        "metric": METRIC,
        "value": value,
        "unit": "steps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * t_bulk_total / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "fp32+fp64",
        "data": "synthetic (seeded tone fields)",
        "config": {"workload": "uneven batch: 1024 instances, 70% spin-1/2 analytic / 30% spin-1 Lie-Trotter(24), "
                               "durations log-uniform 10us-10ms, dt_int 10ns, dt_out 1us, 8 tones per axis, "
                               "Magnus CF4, rotating frame, one persistent launch (CUDA graph)",
                   "instances_per_gpu": len(specs), "integration_steps_per_gpu": total_steps,
                   "l2": "256 MB buffer written between timed steps",
                   "autotuned": {"fp32_bulk": {"chosen": cfg_bulk, "launched": bulk.launch_info()},
                                 "fp64": {"chosen": {str(d): c for d, c in plain.config.items()},
                                          "launched": plain.launch_info()}},
                   "threads_per_block": info["threads_per_block"], "registers": info["registers_per_thread"],
                   "tuning_ms": {"fp32_bulk": {k: 1e3 * v["seconds"] for k, v in tune_bulk.items()},
                                 "fp64": {str(d): {k: 1e3 * v["seconds"] for k, v in t.items()}
                                          for d, t in plain.tuning.items()}}},
        "latency_ms": {"p50": 1e3 * float(np.percentile(t_bulk, 50)), "p99": 1e3 * float(np.percentile(t_bulk, 99))},
        "plain_fp64": {"value": world * total_steps * args.steps / t_plain_total, "unit": "steps/s",
                       "ms_per_step": 1e3 * t_plain_total / args.steps,
                       "launches": "one per spin (two streams), each autotuned",
                       "evolve_kernel_ms": 1e3 * float(np.mean(t_evolve_plain)),
                       "fp64_tflops": fp64_plain_flops / float(np.mean(t_evolve_plain)) / 1e12,
                       "fp64_frac": fp64_plain_flops / float(np.mean(t_evolve_plain)) / 1e12 / measured_fp64_peak()["tflops"],
                       "per_spin": plain_parts,
                       "flop_count": "sin, cos, sqrt and division count 1 flop each; a spin-half step's 60 "
                                     "transcendental calls (48 of them the tone field) keep the FP64 pipe busy far "
                                     "longer than their flop count"},
        "speedup_vs_fp64": t_plain_total / t_bulk_total,
        "state_err": {"max": float(errs.max()), "p50": float(np.median(errs)), "p99": float(np.percentile(errs, 99)),
                      "tolerance": 1e-6, "vs": "plain FP64 form, final state state[N-1] per instance"},
        "roofline": {"bound": "fp64", "achieved": achieved, "peak": fp64_peak["tflops"], "unit": "TFLOP/s",
                     "frac": achieved / fp64_peak["tflops"], "traffic": TRAFFIC_BYTES_PER_LAUNCH,
                     "algorithmic_bytes": algorithmic_bytes(specs),
                     "kernel": ("spinsim::evolve_dmma_kernel (FP32-bulk tensor path: field samples as FP64 "
                                "mma.m8n8k4 products, Magnus step, mixed spins)" if info["variant"] == 0 else
                                "spinsim::evolve_kernel (FP32-bulk warp tone synthesis, mixed spins)"),
                     "peak_source": fp64_peak["source"],
                     "fp32_achieved": fp32_flops / evolve_s / 1e12,
                     "kernel_ms": 1e3 * evolve_s},
        # per timed step (one graph replay): the tensor path's per-instance constants, the time
        # evolution, the scan's prefix, and one apply launch per spin present
        "gpu_launches": (int(info["variant"] == 0) + 2 + len({d for d, _, _ in specs})) * args.steps,
        "clocks": clocks.summary(),
        "e2e": {"value": world * total_steps * len(e2e_times) / e2e_total, "unit": "steps/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": 1e3 * e2e_total / len(e2e_times), "api": "spinsim_b200.batch.Evaluator.evaluate",
                "chunks": args.e2e_chunks, "outputs": "time, U, state, spin into page-locked host memory"},
    }
    if peaks:
        out["hbm_peak_gbs"] = peaks.get("hbm_gbs")
    return out, specs


_PEAK = {}


def measured_fp64_peak():
    """FP64 FMA throughput of this GPU measured in-run (dependent-chain-free DFMA loop)."""
    if "fp64" not in _PEAK:
        import torch
        import spinsim_b200 as ss
        lib = ss._lib.load()
        flops = ss._lib.c_dbl()
        dev = torch.cuda.current_device()
        best = 0.0
        stream = torch.cuda.current_stream().cuda_stream
        for _ in range(3):
            s = torch.cuda.Event(enable_timing=True)
            e = torch.cuda.Event(enable_timing=True)
            s.record()
            ss._lib.check(lib.spinsim_fma_peak(0, ss._lib.ctypes.byref(flops), stream))
            e.record()
            torch.cuda.synchronize()
            best = max(best, flops.value / (s.elapsed_time(e) / 1e3) / 1e12)
        _PEAK["fp64"] = {"tflops": best, "source": f"measured in-run on GPU {dev} (FP64 FMA loop)"}
    return _PEAK["fp64"]


# ------------------------------------------------------------------------------------ reference arm
def host_threads():
    """Host cores this process may run on (torchrun sets OMP_NUM_THREADS=1 for its workers, so the
    CPU arms pass this count to the oracle explicitly)."""
    try:
        return len(os.sched_getaffinity(0))
    except (AttributeError, OSError):
        return os.cpu_count() or 1


def bench_reference(args, world, rank):
    """The reference's CPU algorithm (the oracle: the reference's get_time_evolution and get_state,
    restated in C with OpenMP over output steps as the reference's CPU device parallelises them) on
    the whole benchmark batch every step: every instance's time evolution, then its state
    propagation (I:1081-1082), on all host threads."""
    from oracle import oracle as O
    specs = workload(seed_base=0)
    O.lib()
    threads = host_threads()
    field = O.Field(8)
    total = sum(int(dur / 1e-6) * 100 for _, dur, _ in specs)
    times = []
    for it in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        for dim, dur, p in specs:
            n = int(dur / 1e-6)
            if n:
                _, u = O.time_evolution(dim, field, p, 0.0, 10e-9, 1e-6, n, n_threads=threads)
                O.state(u, np.array([1, 0], complex) if dim == 2 else np.array([0.5, 0.5 ** 0.5, 0.5], complex))
        el = time.perf_counter() - t0
        if it >= args.warmup:
            times.append(el)
    value = total * len(times) / sum(times)
    sample = f"the whole batch every step: {len(specs)} instances, {total} integration steps, time evolution and state"
    return {
        "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(times)), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded tone fields)",
        "impl": "reference",
        "config": {"workload": "uneven batch: 1024 instances, 70% spin-1/2 analytic / 30% spin-1 Lie-Trotter(24), "
                               "durations log-uniform 10us-10ms, dt_int 10ns, dt_out 1us, 8 tones per axis, "
                               "Magnus CF4, rotating frame", "integration_steps": total, "threads": threads},
        "cpu_baseline": {"value": value, "unit": "steps/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def bench_serving(args):
    """Serving workload: Poisson arrivals of evaluate() requests (70% spin half / 30% spin one,
    durations log-uniform 10 us - 100 ms, dt_int from {10, 20, 50, 100} ns, dt_out 1 us, pulse-train
    tables), continuous batching under an HBM budget; p50/p99 latency and throughput per rate."""
    import torch
    import spinsim_b200 as ss
    from spinsim_b200.serving import Server, latency_summary, synthetic_requests
    rates = [float(r) for r in args.rates.split(",")]
    out = {"metric": "serving p50/p99 latency and steps/s", "workload": "serving", "requests_per_rate": args.requests,
           "precision": "fp32_bulk", "hbm_budget_gb": args.hbm_budget_gb, "rates": {}}
    kw = {"max_registers": args.max_registers} if args.max_registers > 0 else {}
    if args.max_steps_per_launch > 0:
        kw["max_steps_per_launch"] = args.max_steps_per_launch

    def serve(reqs):
        srv = Server(precision=ss.Precision.FP32_BULK, hbm_budget=int(args.hbm_budget_gb * (1 << 30)),
                     streams=args.streams, max_batch=args.max_batch, **kw)
        torch.cuda.synchronize()
        done = srv.run(reqs, keep_results=False)  # the client drops each result as it completes
        torch.cuda.synchronize()
        summ = latency_summary(done)
        dur = [c - a for _, _, a, c in srv.launch_log]
        summ.update({"launches": srv.stats["launches"], "budget_waits": srv.stats["budget_waits"],
                     "arena_retries": srv.stats["arena_retries"],
                     "launch_ms_p50": 1e3 * float(np.percentile(dur, 50)), "launch_ms_max": 1e3 * float(max(dur)),
                     "requests_per_launch_mean": float(np.mean([n for n, _, _, _ in srv.launch_log])),
                     # host time of the serving loop: packing and issuing launches, and completing them
                     "host_ms": {"admit": 1e3 * srv.stats["host_admit_s"], "complete": 1e3 * srv.stats["host_complete_s"],
                                 "admit_per_launch": 1e3 * srv.stats["host_admit_s"] / max(1, srv.stats["launches"]),
                                 "busy_fraction_of_span": (srv.stats["host_admit_s"] + srv.stats["host_complete_s"]) /
                                                          max(summ["span_s"], 1e-9)}})
        return summ, srv.kw

    # capacity: the same mix with every request present at the start (the server saturated), and the
    # device alone: all of these requests as one batched launch, timed with CUDA events
    cap_reqs = synthetic_requests(args.requests, 1e12, seed=4)
    capacity, server_kw = serve(cap_reqs)
    steps_per_request = float(np.mean([r.steps() for r in cap_reqs]))
    from spinsim_b200.batch import Batch
    one = Batch(cap_reqs, **server_kw)  # the server's kernel configuration
    device_s = _event_time(one.run)
    out["capacity"] = {"steps_per_s": capacity["steps_per_s"], "requests_per_s": capacity["steps_per_s"] / steps_per_request,
                       "mean_steps_per_request": steps_per_request, "launches": capacity["launches"],
                       "host_ms": capacity["host_ms"],
                       "device_steps_per_s": one.total_steps / device_s,
                       "how": "all requests arrive at t = 0; steps/s over the span to the last completion "
                              "(device_steps_per_s: the same requests as one launch with state and spin)"}
    del one
    for rate in rates:
        summ, _ = serve(synthetic_requests(args.requests, rate, seed=4))
        summ["offered_steps_per_s"] = rate * steps_per_request
        summ["load"] = rate * steps_per_request / capacity["steps_per_s"]  # above 1: latency grows with the backlog
        out["rates"][str(int(rate))] = summ
        print(json.dumps({"rate": rate, **summ}), file=sys.stderr, flush=True)
    return out


def _event_time(fn, reps=3):
    import torch
    fn()
    torch.cuda.synchronize()
    best = float("inf")
    for _ in range(reps):
        s = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        s.record()
        fn()
        e.record()
        torch.cuda.synchronize()
        best = min(best, s.elapsed_time(e) / 1e3)
    return best


def _err_summary(a, b):
    """Final-state error of each member (max |difference| of state[N-1]): p50 / p99 / max over members."""
    e = np.array([np.abs(x - y).max() if x.size else 0.0 for x, y in zip(a.final_states(), b.final_states())])
    return {"members": int(e.size), "p50": float(np.median(e)), "p99": float(np.percentile(e, 99)),
            "max": float(e.max()), "tolerance": 1e-6}


def bench_configs(args):
    """The drop-in on the other reference workloads, timed with CUDA events: Larmor precession (one
    evaluate(), spin half, 200,000 output steps), the spin-one detuned Rabi sweep (64 detunings,
    Lie-Trotter 28 squarings, 10 ms) and the spin-half Gaussian-pulse ensemble (4096 members, 1 ms),
    each as plain FP64 and, for the sweeps, FP32-bulk with its per-member final-state error."""
    import torch
    import spinsim_b200 as ss
    from spinsim_b200.batch import Batch, Instance
    import fields as F
    out = {"metric": "steps/s per reference workload", "workload": "configs", "configs": {}}
    # Simulator set-up (the reference JIT-compiles per Simulator): user field to LTO-IR with numba,
    # then nvJitLink into the kernel; a second Simulator of the same function reuses the LTO-IR
    t0 = time.perf_counter()
    ss.Simulator(F.detuned_rabi, ss.SpinQuantumNumber.ONE, ss.IntegrationMethod.MAGNUS_CF4,
                 ss.ExponentiationMethod.LIE_TROTTER, True, 28)
    t1 = time.perf_counter()
    ss.Simulator(F.detuned_rabi, ss.SpinQuantumNumber.ONE, ss.IntegrationMethod.MAGNUS_CF4,
                 ss.ExponentiationMethod.LIE_TROTTER, True, 28)
    t2 = time.perf_counter()
    out["simulator_setup_s"] = {"first": t1 - t0, "same_field_again": t2 - t1}
    # Larmor: one evaluate() through the drop-in API (FP64), outputs copied to the host
    sim = ss.Simulator(F.larmor, ss.SpinQuantumNumber.HALF)
    t = _event_time(lambda: sim.evaluate(0, 100e-3, 100e-9, 500e-9, ss.SpinQuantumNumber.HALF.plus_x).state)
    out["configs"]["larmor_fp64"] = {"steps": 1_000_000, "seconds": t, "steps_per_s": 1e6 / t,
                                     "api": "Simulator.evaluate (results read on the host)"}
    # detuned spin-one Rabi sweep: 64 instances of one user field
    deltas = np.random.default_rng(seed=1).uniform(-5e3, 5e3, 64)
    insts = [Instance(ss.SpinQuantumNumber.ONE, 0, 10e-3, 10e-9, 100e-9, ss.SpinQuantumNumber.ONE.plus_z, [d])
             for d in deltas]
    res = {}
    for prec in (ss.Precision.FP64, ss.Precision.FP32_BULK):
        b = Batch(insts, get_field=F.detuned_rabi, number_of_squares=28, precision=prec,
                  max_registers=128 if prec == ss.Precision.FP64 else 0)
        tt = _event_time(b.run, reps=2)
        res[prec.name] = b
        out["configs"][f"detuned_rabi_{prec.name.lower()}"] = {"steps": b.total_steps, "seconds": tt,
                                                              "steps_per_s": b.total_steps / tt}
    out["configs"]["detuned_rabi_fp32_bulk"]["state_err"] = _err_summary(res["FP32_BULK"], res["FP64"])
    # Gaussian-pulse ensemble: 4096 members
    members = np.random.default_rng(seed=2).normal(0.0, 500.0, 4096)
    insts = [Instance(ss.SpinQuantumNumber.HALF, 0, 1e-3, 20e-9, 1e-6, ss.SpinQuantumNumber.HALF.plus_z, [m])
             for m in members]
    res = {}
    for prec in (ss.Precision.FP64, ss.Precision.FP32_BULK):
        b = Batch(insts, get_field=F.gaussian_ensemble, precision=prec)
        tt = _event_time(b.run, reps=2)
        res[prec.name] = b
        out["configs"][f"gaussian_ensemble_{prec.name.lower()}"] = {"steps": b.total_steps, "seconds": tt,
                                                                   "steps_per_s": b.total_steps / tt}
    out["configs"]["gaussian_ensemble_fp32_bulk"]["state_err"] = _err_summary(res["FP32_BULK"], res["FP64"])
    torch.cuda.synchronize()
    return out


def profile_case(args):
    """One launch of the benchmark batch for profilers: the full batch, or a small case (the first 256
    instances with durations capped at 1 ms) that a full ncu capture can replay quickly.  With
    ``--profile-field pulses``: one serving launch instead, ``--requests`` pulse-train requests of the
    serving mix in the server's kernel configuration."""
    import torch
    import spinsim_b200 as ss
    from spinsim_b200.batch import Batch
    if args.profile_field == "pulses":
        from spinsim_b200.serving import Server, synthetic_requests
        reqs = synthetic_requests(args.requests, 1e12, seed=4)
        kw = Server(hbm_budget=1 << 20, warm_up=False).kw
        if args.max_registers > 0:
            kw["max_registers"] = args.max_registers
        b = Batch(reqs, **kw)
        b.run(with_state=not args.evolve_only)
        torch.cuda.synchronize()
        return {"workload": f"profile-pulses-{len(reqs)}", "precision": "fp32_bulk", "steps": b.total_steps,
                "intervals": b.n_intervals, "plan": b.plan_info()}
    specs = workload()
    if args.profile_size == "small":
        specs = [(d, min(t, 1e-3), p) for d, t, p in specs[:256]]
    if args.profile_spin != "mixed":  # one spin's instances (the plain FP64 form runs one launch per spin)
        specs = [sp for sp in specs if sp[0] == (2 if args.profile_spin == "half" else 3)]
    prec = ss.Precision.FP32_BULK if args.precision == "fp32_bulk" else ss.Precision.FP64
    b = Batch(instances(ss, specs), precision=prec, max_registers=args.max_registers, lanes=args.lanes,
              variant=args.variant)
    b.run(with_state=not args.evolve_only)
    torch.cuda.synchronize()
    return {"workload": f"profile-{args.profile_size}", "precision": args.precision, "steps": b.total_steps,
            "intervals": b.n_intervals, "plan": b.plan_info()}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extra-workloads", action="store_true",
                    help="skip the other reference workloads and the serving sweep in the main line")
    ap.add_argument("--line-rates", default="1000,10000,50000", help="serving rates in the main line")
    ap.add_argument("--line-requests", type=int, default=2000, help="serving requests per rate in the main line")
    ap.add_argument("--workload", default="batch", choices=["batch", "serving", "configs", "profile"])
    ap.add_argument("--profile-size", default="small", choices=["small", "full"])
    ap.add_argument("--profile-spin", default="mixed", choices=["mixed", "half", "one"])
    ap.add_argument("--profile-field", default="tones", choices=["tones", "pulses"],
                    help="profile workload: the benchmark's tone batch, or one launch of serving requests")
    ap.add_argument("--precision", default="fp32_bulk", choices=["fp32_bulk", "fp64"])
    ap.add_argument("--max-registers", type=int, default=168)
    ap.add_argument("--lanes", type=int, default=0)
    ap.add_argument("--variant", type=int, default=0, help="FP32-bulk tone kernel: 0 tensor path, 1 warp synthesis")
    ap.add_argument("--evolve-only", action="store_true")
    ap.add_argument("--bulk-config", default="",
                    help='FP32-bulk launch configuration as JSON (e.g. \'{"variant": 0, "max_registers": 96}\') '
                         "instead of autotuning it; for profiling runs, where serialised kernels distort the tuning")
    ap.add_argument("--e2e-chunks", type=int, default=8, help="groups overlapped in the end-to-end measurement")
    ap.add_argument("--rates", default="1000,2000,5000,10000,20000,50000")
    ap.add_argument("--requests", type=int, default=20000)
    ap.add_argument("--streams", type=int, default=4)
    ap.add_argument("--max-batch", type=int, default=2048)
    ap.add_argument("--max-steps-per-launch", type=float, default=0, help="serving: work cap of one launch")
    ap.add_argument("--hbm-budget-gb", type=float, default=16.0)
    args = ap.parse_args()
    world, rank, local = dist_setup()
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(bench_reference(args, world, rank)), flush=True)
        return
    import torch
    if not torch.cuda.is_available():
        if rank == 0:
            print(json.dumps({"metric": METRIC, "unavailable": "no CUDA device"}))
        return
    torch.cuda.set_device(local)
    if args.workload == "serving":
        if rank == 0:
            print(json.dumps(bench_serving(args)), flush=True)
        return
    if args.workload == "profile":
        print(json.dumps(profile_case(args)), flush=True)
        return
    if args.workload == "configs":
        if rank == 0:
            print(json.dumps(bench_configs(args)), flush=True)
        return
    out, specs = bench_ours(args, world, rank)
    if rank == 0 and world == 1 and not args.no_extra_workloads:
        # the other reference workloads and a short serving sweep, in the line the driver records
        cfg = bench_configs(args)
        out["reference_workloads"] = {"simulator_setup_s": cfg["simulator_setup_s"], **cfg["configs"]}
        sweep = argparse.Namespace(**{**vars(args), "rates": args.line_rates, "requests": args.line_requests,
                                      "hbm_budget_gb": 8.0, "max_registers": 0})
        out["serving"] = bench_serving(sweep)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O
        steps, el, frac = cpu_sample(specs, seconds_target=10.0, n_threads=host_threads())
        steps1, el1, frac1 = cpu_sample(specs, seconds_target=3.0, n_threads=1)
        out["cpu_baseline"] = {"value": steps / el, "unit": "steps/s", "cores": host_threads(), "kind": "port",
                               "sample": f"oracle (reference algorithm in C, OpenMP) on the first {frac:.4f} of "
                                         f"the output intervals of every instance: {steps} integration steps",
                               "single_core": {"value": steps1 / el1, "unit": "steps/s", "cores": 1,
                                               "sample": f"first {frac1:.4f} of the output intervals of every "
                                                         f"instance: {steps1} integration steps"}}
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
