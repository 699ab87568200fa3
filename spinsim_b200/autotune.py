"""Autotuner for batched launches: picks the time-evolution kernel's launch shape for a batch.

The candidates depend on the kernel the batch runs (``candidates_for``):

* FP32-bulk tone fields: the kernel variant (0: field samples as FP64 tensor-core products over CTA
  tiles of 32 output steps, 1: warp-synchronous phasor synthesis) and its register budget (which
  sets the resident CTAs per SM), plus the CTA size for the warp-synchronous kernel; lanes per output
  step do not apply (one lane per step, or a quad per step's time segments on the tensor path).
* every other plan: lanes per output step, CTA size and register budget.

Every candidate is a distinct launch.  For a given batch the tuner times each candidate after a
warm-up launch with CUDA events and keeps the fastest; it returns the configuration and, in the
timings, the launch that configuration produced (``plan_info``: registers, CTA size, CTAs per SM,
lanes, kernel variant, tile size).  Results are cached per workload signature (spin mix, fine steps
per output step, total output steps, precision, field kind) in a JSON file
(``$SPINSIM_AUTOTUNE_CACHE``, default ``~/.cache/spinsim_b200/autotune.json``).
"""
import hashlib
import json
import os
import threading

import numpy as np

_lock = threading.Lock()
DEFAULT_CANDIDATES = [
    {"lanes": lanes, "threads_per_block": tpb, "max_registers": regs}
    for regs in (0, 168, 128) for lanes in (1, 2) for tpb in (64, 128)
]
# FP32-bulk tone fields: tensor-path kernel at 80 and 96 (6 and 5 CTAs per SM), 128 and 168 registers; the warp
# synthesis at 168 and 128 registers with 64- or 128-thread CTAs.
BULK_TONE_CANDIDATES = (
    [{"variant": 0, "max_registers": regs} for regs in (80, 96, 128, 168)] +
    [{"variant": 1, "max_registers": regs, "threads_per_block": tpb} for regs in (168, 128) for tpb in (64, 128)]
)


def candidates_for(instances, precision=None, get_field=None, **_):
    """The distinct launch configurations worth timing for this batch."""
    from . import Precision, ToneField
    bulk = precision is not None and int(Precision(precision).value) == int(Precision.FP32_BULK.value)
    tones = get_field is None and all(isinstance(i.field, ToneField) for i in instances)
    return BULK_TONE_CANDIDATES if (bulk and tones) else DEFAULT_CANDIDATES


def cache_path():
    return os.environ.get("SPINSIM_AUTOTUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "spinsim_b200", "autotune.json"))


def signature(instances, **kw):
    dims = [i.spin.dimension for i in instances]
    durs = [float(i.time_end) - float(i.time_start) for i in instances]
    steps = [float(i.time_step_output) / float(i.time_step_integration) for i in instances]
    key = json.dumps({"n": len(instances), "d2": dims.count(2), "d3": dims.count(3),
                      "dur": round(float(np.sum(durs)), 9), "k": round(float(np.mean(steps)), 3),
                      "fields": sorted({type(i.field).__name__ for i in instances}),
                      **{k: str(v) for k, v in kw.items()}}, sort_keys=True)
    return hashlib.sha256(key.encode()).hexdigest()[:20]


def _load():
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(data):
    p = cache_path()
    try:
        os.makedirs(os.path.dirname(p), exist_ok=True)
        tmp = p + ".tmp"
        with open(tmp, "w") as f:
            json.dump(data, f, indent=1)
        os.replace(tmp, p)
    except OSError:
        pass


def tune(instances, candidates=None, use_cache=True, repeats=2, **batch_kwargs):
    """Return (best config dict, {config key: seconds}) for ``Batch(instances, **batch_kwargs, **cfg)``."""
    import torch
    from .batch import Batch
    sig = signature(instances, **batch_kwargs)
    if use_cache:
        with _lock:
            hit = _load().get(sig)
        if hit:
            return hit["best"], hit["timings"]
    candidates = candidates or candidates_for(instances, **batch_kwargs)
    timings = {}
    best, best_t = None, float("inf")
    seen = set()
    for cfg in candidates:
        try:
            b = Batch(instances, **batch_kwargs, **cfg)
        except (ValueError, NotImplementedError):
            continue
        info = b.launch_info()
        launch = (info["registers_per_thread"], info["threads_per_block"], info["blocks_per_sm"], info["lanes"],
                  info["variant"], info["tile_intervals"])
        if launch in seen:  # the same kernel and launch shape as a candidate already timed
            del b
            continue
        seen.add(launch)
        b.run(with_state=False)
        torch.cuda.synchronize()
        ts = []
        for _ in range(repeats):
            s = torch.cuda.Event(enable_timing=True)
            e = torch.cuda.Event(enable_timing=True)
            s.record()
            b.run(with_state=False)
            e.record()
            torch.cuda.synchronize()
            ts.append(s.elapsed_time(e) / 1e3)
        t = min(ts)
        timings[json.dumps(cfg, sort_keys=True)] = {"seconds": t, "launch": info}
        if t < best_t:
            best, best_t = cfg, t
        del b
    if best is None:
        raise RuntimeError("no candidate configuration could be launched")
    if use_cache:
        with _lock:
            data = _load()
            data[sig] = {"best": best, "timings": timings}
            _store(data)
    return best, timings
