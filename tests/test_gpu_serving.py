"""Continuous-batching server: correctness against the oracle, identity of a result alone and in
the mix, and HBM-budget admission."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def oracle_of(req):
    f = req.field
    tabs = [(f.tables[0][0], f.tables[0][1], 0, False), (f.tables[1][0], f.tables[1][1], 0, False),
            (f.tables[0][0], f.tables[0][1], 0, False)]
    return O.evaluate(req.spin.dimension, O.Field(9, tabs), [1.0, 1.0, 0.0, 0.0], req.time_start, req.time_end,
                      req.time_step_integration, req.time_step_output, req.state_init)


def requests(n=24, rate=2e5, seed=7, max_duration=400e-6):
    from spinsim_b200.serving import synthetic_requests
    return synthetic_requests(n, rate, seed=seed, max_duration=max_duration)


def test_serving_fp64_matches_oracle_and_is_mix_independent(cuda):
    import spinsim_b200 as ss
    from spinsim_b200.serving import Server
    reqs = requests()
    srv = Server(precision=ss.Precision.FP64, streams=3, max_batch=6)
    done = srv.run(reqs)
    assert len(done) == len(reqs)
    assert srv.stats["launches"] >= 4
    by_id = {c.request.id: c for c in done}
    for r in reqs[:10]:
        t, u, s, sp = oracle_of(r)
        got = by_id[r.id].results
        assert np.array_equal(got.time, t)
        assert np.abs(got.time_evolution - u).max() < 1e-10
        assert np.abs(got.state - s).max() < 1e-10
    for r in reqs[::5]:
        alone = Server(precision=ss.Precision.FP64, streams=1).run([r])[0].results
        assert np.array_equal(alone.state, by_id[r.id].results.state)
        assert np.array_equal(alone.time_evolution, by_id[r.id].results.time_evolution)


def test_serving_fp32_bulk_alone_equals_mix_and_error_bound(cuda):
    import spinsim_b200 as ss
    from spinsim_b200.serving import Server
    reqs = requests(seed=8)
    done = Server(precision=ss.Precision.FP32_BULK, streams=2, max_batch=5).run(reqs)
    by_id = {c.request.id: c for c in done}
    for r in reqs[::4]:
        alone = Server(precision=ss.Precision.FP32_BULK, streams=1).run([r])[0].results
        assert np.array_equal(alone.state, by_id[r.id].results.state)
        t, u, s, sp = oracle_of(r)
        assert np.abs(by_id[r.id].results.state - s).max() < 1e-6


def test_hbm_budget_admission(cuda):
    import spinsim_b200 as ss
    from spinsim_b200.serving import Server
    reqs = requests(n=12, rate=1e6, seed=9)
    budget = max(r.footprint() for r in reqs) + 1
    srv = Server(precision=ss.Precision.FP64, hbm_budget=budget, streams=4)
    seen = []
    done = srv.run(reqs, on_complete=lambda c: seen.append(float(c.results.state[-1, 0].real)), keep_results=False)
    assert len(done) == len(reqs) == len(seen)
    assert all(c.results is None for c in done)
    assert srv.stats["budget_waits"] > 0
    assert srv.arena.in_use == 0
    with pytest.raises(ValueError):
        Server(precision=ss.Precision.FP64, hbm_budget=1000).run(reqs[:1])


def test_held_results_hold_the_budget(cuda):
    import gc
    import spinsim_b200 as ss
    from spinsim_b200.serving import Server
    reqs = requests(n=12, rate=1e6, seed=9)
    srv = Server(precision=ss.Precision.FP64, hbm_budget=max(r.footprint() for r in reqs) + 1, streams=2)
    with pytest.raises(RuntimeError, match="held by results"):
        srv.run(reqs)  # keeps every result: the arena fills up
    gc.collect()
    assert srv.arena.in_use == 0
    big = Server(precision=ss.Precision.FP64, hbm_budget=256 << 20, streams=2)
    done = big.run(reqs)
    held = big.arena.in_use
    assert 0 < held <= sum(r.footprint() for r in reqs)
    del done
    gc.collect()
    assert big.arena.in_use == 0


def test_footprint_bounds_the_launch(cuda):
    import spinsim_b200 as ss
    from spinsim_b200.batch import Batch
    from spinsim_b200.serving import Server
    reqs = requests(n=16, rate=1e6, seed=11, max_duration=2e-3)
    srv = Server(precision=ss.Precision.FP32_BULK, warm_up=False)
    for group in (reqs[:1], reqs[1:2], reqs[:8], reqs):
        b = Batch([r.instance() for r in group], **srv.kw)
        assert b.device_bytes <= sum(r.footprint() for r in group)


def test_async_submit_futures(cuda):
    """start/submit/close: futures resolve to the same results as a synchronous run, and a request
    whose launch cannot be made fails its own future."""
    import spinsim_b200 as ss
    from spinsim_b200.serving import Request, Server
    reqs = requests(n=16, rate=1e5, seed=21)
    sync = {c.request.id: c.results for c in Server(precision=ss.Precision.FP64, streams=2).run(reqs)}
    with Server(precision=ss.Precision.FP64, streams=3, max_batch=4) as srv:
        bad = Request(ss.SpinQuantumNumber.HALF, reqs[0].field, 0.0, 20e-6, 1e-7, 1e-6, [1.0, 0.0, 0.0], id=-1)
        bad_future = srv.submit(bad)
        with pytest.raises(ValueError):
            bad_future.result(timeout=60)
        futures = [srv.submit(r) for r in reqs]
        got = [f.result(timeout=120) for f in futures]
    for r, res in zip(reqs, got):
        assert np.array_equal(res.state, sync[r.id].state)
        assert np.array_equal(res.time_evolution, sync[r.id].time_evolution)
    with pytest.raises(RuntimeError):
        srv.submit(reqs[0])  # closed


def test_async_timeout_and_cancel(cuda):
    """A request whose timeout passes before admission fails with TimeoutError; others still run."""
    import spinsim_b200 as ss
    from spinsim_b200.serving import Server
    reqs = requests(n=6, rate=1e5, seed=23)
    with Server(precision=ss.Precision.FP64, streams=2) as srv:
        late = srv.submit(reqs[0], timeout=-1.0)  # already past its deadline
        ok = [srv.submit(r) for r in reqs[1:]]
        with pytest.raises(TimeoutError):
            late.result(timeout=60)
        assert all(f.result(timeout=120) is not None for f in ok)
        assert srv.stats["timeouts"] == 1


def test_async_results_dropped_on_client_thread_while_admitting(cuda):
    """Clients drop their Results (the arena block's finalizer runs on the client thread) while the
    serving thread admits further launches into the same arena: every result still matches the
    synchronous run and the arena is whole again at the end."""
    import gc
    import queue
    import threading
    import spinsim_b200 as ss
    from spinsim_b200.serving import Server
    reqs = requests(n=40, rate=1e5, seed=31)
    sync = {c.request.id: c.results.state.copy() for c in Server(precision=ss.Precision.FP64, streams=2).run(reqs)}
    mismatches = []
    srv = Server(precision=ss.Precision.FP64, streams=4, max_batch=3,
                 hbm_budget=2 * sum(r.footprint() for r in reqs) + (1 << 20))
    work = queue.Queue()
    with srv:
        for r in reqs:
            work.put((r, srv.submit(r)))

        def client():
            while True:
                try:
                    r, f = work.get_nowait()
                except queue.Empty:
                    return
                res = f.result(timeout=120)
                if not np.array_equal(res.state, sync[r.id]):
                    mismatches.append(r.id)
                del res, f  # the launch's block returns to the arena from this thread

        threads = [threading.Thread(target=client) for _ in range(3)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
    gc.collect()
    assert not mismatches
    assert srv.arena.in_use == 0
    assert srv.arena.free_blocks() == [(0, srv.arena.size)]
