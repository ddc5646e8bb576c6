"""The multi-GPU control plane on CPU: two gloo ranks (world size 2), the
same calls bench.py makes under torchrun with nccl -- the max-over-ranks
timing, the replica seeds, the job throughput -- and the cost-balanced
assignment of ensemble members to ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from fvmpor_b200.replicas import job_throughput, partition_members, replica_seed


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, q):
    import datetime

    import torch.distributed as dist

    from fvmpor_b200.replicas import max_over_ranks

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        t = max_over_ranks(1.0 + rank * 0.5)
        parts = partition_members([5, 9, 2, 7, 7, 1, 3], ws)
        out = [None] * ws
        dist.all_gather_object(out, parts)
        q.put((rank, t, replica_seed(1, rank), out))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_gloo_ranks():
    ws = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(ws)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res.sort()
    # every rank sees the slowest rank's time
    assert [r[1] for r in res] == [1.5, 1.5]
    # replicas run different Ks realisations
    assert res[0][2] != res[1][2]
    # all ranks agree on the member assignment
    assert res[0][3] == res[1][3]


def test_partition_members_balances_cost():
    costs = [40000, 2000, 39000, 3000, 20000, 21000, 10000, 30000]
    parts = partition_members(costs, 3)
    assert sorted(m for p in parts for m in p) == list(range(len(costs)))
    loads = [sum(costs[m] for m in p) for p in parts]
    assert max(loads) - min(loads) <= max(costs)
    assert partition_members(costs, 3) == parts   # deterministic
    with pytest.raises(ValueError):
        partition_members(costs, 0)


def test_job_throughput():
    # two ranks each simulate 30 days; the job takes the slowest rank's time
    assert job_throughput(30 * 86400.0, 2, 10.0) == pytest.approx(2 * 30 * 86400.0 / 10.0)
