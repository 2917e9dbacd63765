"""The multi-GPU path of bench.py is replicas only (independent Monte Carlo
paths need no exchange): two gloo ranks on CPU take the max of their timings
and aggregate weak-scaled throughput; replicas of the same request agree."""

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    from montepath_b200.requests import make_request
    from oracle import oracle as O

    req = make_request("european_call", dict(bench.HESTON, n_paths=512, n_steps=16))
    res = O.price(req)
    bench.barrier(dist)
    worst = bench.reduce_max(dist, 10.0 + rank, "cpu")
    value = bench.aggregate(world, req.n_paths * req.n_steps, 3, worst)
    out.put((rank, res.price, res.stderr, worst, value))
    dist.destroy_process_group()


def test_two_rank_replicas():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, p0, s0, w0, v0), (_, p1, s1, w1, v1) = results
    assert p0 == p1 and s0 == s1  # replicas are deterministic
    assert w0 == w1 == 11.0  # max over ranks
    assert v0 == v1 == pytest.approx(2 * 512 * 16 * 3 / 11.0e-3)
