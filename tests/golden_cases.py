"""Access to the committed golden fixtures (tests/golden/golden.npz, made by make_golden.py)."""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "golden.npz")
sys.path.insert(0, os.path.join(HERE, "golden"))
import fields as F  # noqa: E402

SPIN_DIM = {"half": 2, "one": 3}

_cache = {}


def load():
    if "npz" not in _cache:
        z = np.load(GOLDEN)
        _cache["npz"] = {k: z[k] for k in z.files}
        _cache["meta"] = json.loads(bytes(_cache["npz"]["meta"]).decode())
    return _cache["npz"], _cache["meta"]


def cases():
    return load()[1]


def case(name):
    for c in cases():
        if c["name"] == name:
            return c
    raise KeyError(name)


def expected(name):
    z = load()[0]
    return {k: z[f"{name}/{k}"] for k in ("time", "time_evolution", "state", "spin", "psi0")}


def tables():
    z = load()[0]
    return {k.split("/", 1)[1]: z[k] for k in z if k.startswith("table/")}


def table_channels(c):
    """(time, amplitude, order, zero_boundary) per channel x, y, z for a tabulated case."""
    t = tables()
    chans = [(t["tx"], t["ax"]), (t["ty"], t["ay"]), (t["tz"], t["az"])]
    return [(tt, aa, c["order"], c["zero_boundary"]) for tt, aa in chans]
