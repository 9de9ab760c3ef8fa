"""The N > 1 path of the bench on CPU: two ranks (gloo, 127.0.0.1) each take
their share of the ensemble from the static partition (cdns.ensemble, replicas
only) with no communication, the shares are disjoint and complete and balanced,
and the per-rank times reduce to their maximum (the bench's timing rule)."""
import datetime
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    from cdns.ensemble import rank_members, step_bytes
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mine = rank_members(64, world, rank)
        shares = [None] * world
        dist.all_gather_object(shares, [i for i, _, _ in mine])
        t = torch.tensor([1.5 + rank], dtype=torch.float64)      # a per-rank elapsed time
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        load = torch.tensor([sum(step_bytes(n) for _, n, _ in mine)], dtype=torch.float64)
        loads = [torch.zeros(1, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(loads, load)
        if rank == 0:
            q.put((shares, float(t.item()), [float(x.item()) for x in loads]))
    finally:
        dist.destroy_process_group()


def test_two_rank_ensemble_partition_and_timing():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        shares, tmax, loads = q.get(timeout=120)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    a, b = set(shares[0]), set(shares[1])
    assert not (a & b) and a | b == set(range(64))
    assert tmax == 2.5
    assert max(loads) / (sum(loads) / 2) <= 1.01


def test_partition_properties():
    from cdns.ensemble import members, partition, step_bytes
    costs = [step_bytes(n) for n, _ in members(64)]
    for world in (1, 2, 3, 8):
        part = partition(costs, world)
        flat = sorted(i for p in part for i in p)
        assert flat == list(range(64))
        assert part == partition(costs, world)       # every rank derives the same assignment
    with pytest.raises(ValueError):
        partition(costs, 0)
