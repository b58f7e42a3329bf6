"""Job sharding across ranks (opticrcwafdtd_b200/replicas.py), exercised with
two gloo ranks on the CPU: every job runs exactly once, the load is balanced
by cells x steps, and every rank ends with all results in submission order."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from opticrcwafdtd_b200.replicas import partition_by_cost, sharded_map


def test_partition_covers_each_job_once_and_balances():
    costs = [5, 1, 9, 3, 3, 7, 2, 8, 4, 6]
    for world in (1, 2, 3, 4):
        shares = partition_by_cost(costs, world)
        flat = sorted(i for s in shares for i in s)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in s) for s in shares]
        assert max(loads) - min(loads) <= max(costs)
    assert partition_by_cost([], 2) == [[], []]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    seen = []

    def run_batch(items):
        seen.extend(items)
        return [x * x for x in items]

    items = list(range(11))
    costs = [(7 * x) % 5 + 1 for x in items]
    out = sharded_map(run_batch, items, costs)
    q.put((rank, out, seen))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_sharded_map_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=100) for _ in procs]
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    seen = sorted(x for _, _, s in res for x in s)
    assert seen == list(range(11))                     # each job ran once
    for _, out, _ in res:
        assert out == [x * x for x in range(11)]       # all results, in order, on every rank


def test_sharded_map_without_process_group():
    assert sharded_map(lambda xs: [x + 1 for x in xs], [1, 2, 3], [1, 1, 1]) == [2, 3, 4]
