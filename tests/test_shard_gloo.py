"""Multi-process sharding logic on CPU with gloo ranks (world size 2): partition balance and the
gather of per-instance results."""
import os
import socket

import numpy as np
import pytest


def _instances(n=40, seed=0):
    import spinsim_b200 as ss
    from spinsim_b200.batch import Instance
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        spin = ss.SpinQuantumNumber.HALF if rng.uniform() < 0.7 else ss.SpinQuantumNumber.ONE
        dur = float(np.exp(rng.uniform(np.log(10e-6), np.log(10e-3))))
        out.append(Instance(spin, 0.0, dur, 10e-9, 1e-6, spin.plus_z))
    return out


def test_partition_covers_and_balances():
    from spinsim_b200.shard import partition, work
    insts = _instances()
    for world in (1, 2, 3, 8):
        parts = partition(insts, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(insts)))
        loads = [sum(work(insts[i]) for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(work(i) for i in insts)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from spinsim_b200.shard import gather_final_states, partition
        insts = _instances()
        mine = partition(insts, world)[rank]
        # stand-in per-instance result computed on the host: the instance index as a state
        finals = [np.array([i, -i], dtype=complex) for i in mine]
        out = gather_final_states(mine, finals, len(insts))
        q.put((rank, [complex(o[0]).real for o in out]))
    finally:
        dist.destroy_process_group()


def test_gather_over_two_gloo_ranks():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    n = len(_instances())
    for r in (0, 1):
        assert res[r] == [float(i) for i in range(n)]


def test_piece_ranges_cover():
    from spinsim_b200.shard import piece_ranges
    for n in (0, 1, 7, 1000, 1001):
        for world in (1, 2, 3, 8):
            r = piece_ranges(n, world)
            assert len(r) == world and r[0][0] == 0
            assert sum(c for _, c in r) == n
            assert all(r[k][0] + r[k][1] == r[k + 1][0] for k in range(world - 1))
            assert max(c for _, c in r) - min(c for _, c in r) <= 1


def _split_worker(rank, world, port, q):
    """One rank of a split evaluate(), with the oracle standing in for the device: the rank's piece
    of operators (time indices of the whole call), its product, the all-gather of products over
    gloo, the state entering its piece, and its states."""
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import oracle as O
        from spinsim_b200.shard import exchange_products, incoming_states, piece_ranges
        import fields as F
        sweep = [F.TAU * 1e3, F.TAU * 4e3]
        dt_int, n, _, _ = O.normalise_steps(0.0, 2e-3, 100e-9, 1e-6)
        first, count = piece_ranges(n, world)[rank]
        time, u = O.time_evolution(3, O.Field(3), sweep, 0.0, dt_int, 1e-6, n, first=first, count=count)
        u = u[first:first + count]
        prod = np.eye(3, dtype=complex)
        for m in u:
            prod = m @ prod
        products = exchange_products(torch.from_numpy(prod))
        psi0 = np.array([0.0, 1.0, 0.0], complex)
        psi_in = incoming_states(products, psi0)[rank]
        q.put((rank, first, time[first:first + count], O.state(u, psi_in)))
    finally:
        dist.destroy_process_group()


def test_split_evaluate_over_two_gloo_ranks():
    import multiprocessing as mp
    from oracle import oracle as O
    import fields as F
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_split_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    parts = sorted((q.get(timeout=180) for _ in procs), key=lambda x: x[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    t, u, s, _ = O.evaluate(3, O.Field(3), [F.TAU * 1e3, F.TAU * 4e3], 0.0, 2e-3, 100e-9, 1e-6,
                            np.array([0.0, 1.0, 0.0], complex))
    time = np.concatenate([p[2] for p in parts])
    state = np.concatenate([p[3] for p in parts])
    assert parts[1][1] == len(parts[0][2])
    assert np.array_equal(time, t)  # time indices of the whole call
    assert np.abs(state - s).max() < 1e-12
