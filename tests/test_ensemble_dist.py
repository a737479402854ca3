"""Multi-rank dispatch on two gloo ranks on the CPU: the box shards of an
ensemble (ensemble.rank_share) and the routing of a served stream
(serve.shard_requests) that bench.py uses with one rank per GPU, run with a
host stand-in for the device (each rank "advances" the boxes it owns and
reports per-box results), plus the max-over-ranks timing reduction."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from afid_b200.ensemble import cells, ensemble_configs, rank_share, shard


def test_shard_partitions_and_balances():
    cfgs = ensemble_configs(64, seed=1000)
    for world in (1, 2, 3, 4, 8):
        parts = [shard(cfgs, r, world) for r in range(world)]
        flat = sorted(q for p in parts for q in p)
        assert flat == list(range(64))
        loads = [sum(cells(cfgs[q]) for q in p) for p in parts]
        assert max(loads) - min(loads) <= max(cells(c) for c in cfgs)


def test_request_routing_partitions_and_balances():
    from afid_b200.serve import request_stream, serve_mix, shard_requests
    reqs = request_stream(96, 50.0, seed=2000, steps=200, mix=serve_mix)
    for world in (1, 2, 4, 8):
        parts = [shard_requests(reqs, r, world) for r in range(world)]
        assert sorted(r.rid for p in parts for r in p) == list(range(96))
        loads = [sum(r.cells * r.nsteps for r in p) for p in parts]
        assert max(loads) - min(loads) <= max(r.cells * r.nsteps for r in reqs)
        for p in parts:                      # each rank keeps arrival order
            assert [r.arrival for r in p] == sorted(r.arrival for r in p)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _stub_advance(cfg, seed, nsteps):
    """Host stand-in for advancing one box: a value that depends only on the
    box (its configuration and seed) and the step count."""
    return float(cells(cfg) * nsteps + seed) + cfg.ray * 1e-9


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from afid_b200.serve import request_stream, serve_mix, shard_requests
    # the ensemble of bench.py's batch workload: 64 boxes per rank, one seed
    cfgs, mine = rank_share(64, 1000, rank, world)
    res = {q: _stub_advance(c, q, 20) for c, q in zip(cfgs, mine)}
    gathered = [None] * world
    dist.all_gather_object(gathered, res)
    # the served stream of bench.py: each rank serves its routed share
    reqs = shard_requests(request_stream(32 * world, 50.0 * world, seed=2000, steps=200, mix=serve_mix),
                          rank, world)
    served = [None] * world
    dist.all_gather_object(served, sorted(r.rid for r in reqs))
    # the timing reduction: the maximum over ranks
    t = torch.tensor([0.5 + rank], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    work = torch.tensor([float(sum(cells(c) for c in cfgs))], dtype=torch.float64)
    dist.all_reduce(work)
    q.put((rank, gathered, served, float(t.item()), float(work.item())))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_dispatch_and_max_timing():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=180) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    allc = ensemble_configs(64 * world, seed=1000)
    want = {q: _stub_advance(c, q, 20) for q, c in enumerate(allc)}
    for rank, gathered, served, tmax, work in res:
        merged = {}
        for part in gathered:
            assert not set(part) & set(merged)          # each box advanced by one rank
            merged.update(part)
        assert merged == want                           # ... and every box advanced
        flat = sorted(x for part in served for x in part)
        assert flat == list(range(32 * world))
        assert tmax == 0.5 + (world - 1)
        assert work == sum(cells(c) for c in allc)
