"""Host logic of the continuous-batching server: the HBM arena (first fit, coalescing), leases,
request footprints and the synthetic pulse-train workload."""
import gc

import numpy as np
import pytest


def arena(nbytes):
    from spinsim_b200.serving import Arena
    return Arena(nbytes, device="cpu")


def test_arena_first_fit_and_alignment():
    a = arena(10_000)
    assert a.size == 10_240 and a.largest_free() == 10_240
    b1 = a.take(1)
    b2 = a.take(300)
    b3 = a.take(256)
    assert b1 == (0, 256) and b2 == (256, 512) and b3 == (768, 256)
    assert a.in_use == 1024 and a.largest_free() == 10_240 - 1024
    assert a.take(20_000) is None


def test_arena_coalesces_in_any_order():
    rng = np.random.default_rng(0)
    a = arena(1 << 16)
    for trial in range(20):
        blocks = []
        while True:
            b = a.take(int(rng.integers(1, 4000)))
            if b is None:
                break
            blocks.append(b)
        assert len(blocks) > 5
        # blocks never overlap
        spans = sorted(blocks)
        for (o1, n1), (o2, _) in zip(spans, spans[1:]):
            assert o1 + n1 <= o2
        for k in rng.permutation(len(blocks)):
            a.give(*blocks[k])
        assert a.in_use == 0
        assert a.largest_free() == a.size
        assert a.free_blocks() == [(0, a.size)]


def test_arena_reuses_freed_hole():
    a = arena(4096)
    x = a.take(1024)
    y = a.take(1024)
    a.take(1024)
    a.give(*x)
    assert a.take(512) == (0, 512)
    a.give(*y)
    assert a.take(1536) == (512, 1536)


def test_lease_returns_block_when_released():
    from spinsim_b200.serving import _Lease
    a = arena(4096)
    blk = a.take(2048)
    lease = _Lease(a, *blk)
    holder = [lease]
    del lease
    assert a.in_use == 2048
    holder.clear()
    gc.collect()
    assert a.in_use == 0 and a.largest_free() == 4096


def test_footprint_counts_outputs_and_field():
    import spinsim_b200 as ss
    from spinsim_b200.serving import Request, synthetic_requests
    reqs = synthetic_requests(50, 1e4, seed=3)
    for r in reqs:
        d = r.spin.dimension
        n = int((r.time_end - r.time_start) / r.time_step_output)
        outputs = n * (8 + 16 * d * d + 16 * d + 24)
        table_bytes = sum(16 * t.size for t, _, _, _ in r.field.tables.values())
        assert r.footprint() >= outputs + table_bytes
        assert r.steps() == n * int(round(r.time_step_output / r.time_step_integration))
    small = Request(ss.SpinQuantumNumber.HALF, None, 0.0, 1e-6, 1e-7, 1e-6, ss.SpinQuantumNumber.HALF.plus_z)
    assert small.footprint() > 0


def test_pulse_sequence_is_zero_order_hold_on_x_or_y():
    from spinsim_b200.serving import pulse_sequence
    f = pulse_sequence(np.random.default_rng(1), 500e-6)
    (tx, ax, ox, zx), (ty, ay, oy, zy) = f.tables[0], f.tables[1]
    assert ox == 0 and oy == 0 and np.array_equal(tx, ty)
    assert np.all(np.diff(tx) > 0)
    on = (ax != 0) | (ay != 0)
    assert not np.any((ax != 0) & (ay != 0))  # one axis at a time
    widths = np.diff(tx)[on[:-1]]
    assert np.all(np.isclose(widths, 10e-6) | np.isclose(widths, 20e-6))


def test_arena_gives_from_other_threads_while_taking():
    """Blocks given back from other threads (a client dropping Results: the lease's finalizer runs
    on the client thread) while one thread takes blocks: no block is handed out twice and the free
    list coalesces back to one block."""
    import threading
    import queue
    from spinsim_b200.serving import _Lease
    a = arena(1 << 20)
    handoff = queue.Queue()
    stop = threading.Event()
    errors = []

    def client():
        while not stop.is_set() or not handoff.empty():
            try:
                lease = handoff.get(timeout=0.01)
            except queue.Empty:
                continue
            del lease  # the finalizer gives the block back on this thread

    clients = [threading.Thread(target=client) for _ in range(3)]
    for t in clients:
        t.start()
    rng = np.random.default_rng(5)
    live = {}
    try:
        for it in range(4000):
            blk = a.take(int(rng.integers(1, 20_000)))
            if blk is None:
                continue
            off, n = blk
            for o, m in live.items():  # no overlap with blocks still held here
                if off < o + m and o < off + n:
                    errors.append((blk, (o, m)))
            if rng.uniform() < 0.5:
                live[off] = n
            else:
                handoff.put(_Lease(a, off, n))
            if len(live) > 20:
                o = next(iter(live))
                handoff.put(_Lease(a, o, live.pop(o)))
    finally:
        stop.set()
        for t in clients:
            t.join()
    for o, m in live.items():
        a.give(o, m)
    gc.collect()
    assert not errors
    assert a.in_use == 0
    assert a.free_blocks() == [(0, a.size)]
