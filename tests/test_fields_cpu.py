"""Packing of built-in fields into one buffer (host side): table arrays, descriptors and tone rows
land where the spinsim_field structs point."""
import numpy as np
import pytest

BASE = 1 << 40  # a pretend device address of the packed buffer


def decode(host, addr):
    return (int(addr) - BASE) // 8


def test_tables_and_descriptors_round_trip():
    from spinsim_b200.fields import TABLE_DTYPE, TabulatedField, pack_fields_into, packed_doubles
    rng = np.random.default_rng(5)
    fields = []
    for k in range(7):
        chans = {}
        for c in rng.choice(8, size=rng.integers(1, 4), replace=False):
            m = int(rng.integers(2, 40))
            chans[int(c)] = (np.sort(rng.uniform(0, 1, m)), rng.normal(size=m), int(rng.choice([0, 1, 3])), bool(k % 2))
        fields.append(TabulatedField(chans, bias=rng.normal(size=8), gain=rng.normal(size=8)))
    total = packed_doubles(fields)
    host = np.full(total + 8, np.nan)
    out = pack_fields_into(fields, host, BASE)
    tabs = host[:32 * len(fields)].view(TABLE_DTYPE)  # the descriptors lead the buffer
    for f, st in zip(fields, out):
        slot0 = decode(host, st["tables"]) // 4
        assert np.array_equal(st["bias"], f.bias) and np.array_equal(st["gain"], f.gain)
        for c in range(8):
            row = tabs[slot0 + c]
            if c not in f.tables:
                assert row["size"] == 0 and row["time"] == 0
                continue
            t, a, o, zb = f.tables[c]
            assert (row["size"], row["order"], row["zero_boundary"]) == (t.size, o, int(zb))
            ti, ai = decode(host, row["time"]), decode(host, row["amplitude"])
            assert ti >= 8 * 4 * len(fields) and ai >= 8 * 4 * len(fields)  # after the descriptors
            assert np.array_equal(host[ti:ti + t.size], t) and np.array_equal(host[ai:ai + a.size], a)
    assert np.isnan(host[total:]).all()  # nothing written past the packed size


def test_tones_round_trip():
    from spinsim_b200.fields import ToneField, pack_fields_into, packed_doubles
    rng = np.random.default_rng(6)
    fields = [ToneField({c: rng.normal(size=(int(rng.integers(1, 5)), 3)) for c in range(3)}, bias=[0.1, 0, 2.0])
              for _ in range(5)]
    host = np.zeros(packed_doubles(fields))
    out = pack_fields_into(fields, host, BASE)
    for f, st in zip(fields, out):
        flat, start, count = f.packed()
        i = decode(host, st["tones"])
        assert np.array_equal(host[i:i + flat.size], flat)
        assert np.array_equal(st["tone_start"], start) and np.array_equal(st["tone_count"], count)
        assert np.array_equal(st["bias"], f.bias) and np.all(st["gain"] == 1.0)


def test_mixed_kinds_rejected_and_tables_snapshotted():
    from spinsim_b200.fields import TabulatedField, ToneField, packed_doubles
    t = np.array([0.0, 1.0])
    a = np.array([1.0, 2.0])
    f = TabulatedField({0: (t, a)})
    a[0] = 99.0  # the field keeps its own copy
    assert f.tables[0][1][0] == 1.0
    with pytest.raises(TypeError):
        packed_doubles([f, ToneField({0: [[1.0, 1.0, 0.0]]})])


def test_shared_time_array_is_packed_once():
    from spinsim_b200.fields import TabulatedField, pack_fields_into, packed_doubles
    t = np.linspace(0.0, 1.0, 10)
    f = TabulatedField({0: (t, np.arange(10.0)), 1: (t, -np.arange(10.0))}, order=0)
    assert packed_doubles([f]) == 32 + 10 + 20  # descriptors, one time array, two amplitude arrays
    host = np.zeros(packed_doubles([f]))
    out = pack_fields_into([f], host, BASE)
    tabs = host[:32].view(__import__("spinsim_b200.fields", fromlist=["TABLE_DTYPE"]).TABLE_DTYPE)
    assert tabs[0]["time"] == tabs[1]["time"] and tabs[0]["amplitude"] != tabs[1]["amplitude"]
    assert int(out[0]["tables"]) == BASE


def test_packing_rejects_a_short_buffer():
    from spinsim_b200.fields import TabulatedField, pack_fields_into, packed_doubles
    f = TabulatedField({0: (np.linspace(0, 1, 50), np.ones(50))})
    need = packed_doubles([f])
    with pytest.raises(ValueError):
        pack_fields_into([f], np.zeros(need - 1), BASE)
    out = pack_fields_into([f], np.zeros(need), BASE)
    assert int(out[0]["tables"]) == BASE
