"""Box sharding of an ensemble across ranks (no data-path collective) and the
max-over-ranks timing reduction, on two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from afid_b200.ensemble import cells, ensemble_configs, shard


def test_shard_partitions_and_balances():
    cfgs = ensemble_configs(64, seed=1000)
    for world in (1, 2, 3, 4, 8):
        parts = [shard(cfgs, r, world) for r in range(world)]
        flat = sorted(q for p in parts for q in p)
        assert flat == list(range(64))
        loads = [sum(cells(cfgs[q]) for q in p) for p in parts]
        assert max(loads) - min(loads) <= max(cells(c) for c in cfgs)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    cfgs = ensemble_configs(16, seed=7)
    mine = shard(cfgs, rank, world)
    # every rank computes the same assignment without communication
    owners = torch.zeros(16, dtype=torch.int64)
    owners[mine] = 1
    total = owners.clone()
    dist.all_reduce(total)            # checking only: each box owned exactly once
    t = torch.tensor([0.5 + rank], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    q.put((rank, total.tolist(), float(t.item()), len(mine)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_sharding_and_max_timing():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, total, tmax, n in res:
        assert total == [1] * 16
        assert tmax == 1.5
    assert sum(n for *_, n in res) == 16
