"""Autotuner for batched launches: picks lanes per output step, CTA size and register budget.

For a given batch it times each candidate configuration once (after a warm-up launch) with CUDA
events and keeps the fastest.  Results are cached per workload signature (spin mix, fine steps per
output step, total output steps, precision, field kind) in a JSON file
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
    candidates = candidates or DEFAULT_CANDIDATES
    timings = {}
    best, best_t = None, float("inf")
    for cfg in candidates:
        try:
            b = Batch(instances, **batch_kwargs, **cfg)
        except (ValueError, NotImplementedError):
            continue
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
        timings[json.dumps(cfg, sort_keys=True)] = t
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
