"""Multi-GPU plumbing on CPU: two gloo ranks route the serving stream by
tensor key and reduce timings exactly as bench.py does under torchrun (one
replica per GPU, no collective on the data path)."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    import sys

    sys.path[:0] = [os.path.join(os.path.dirname(__file__), "..", "topo-dda_b200")]
    import torch.distributed as dist

    from dda_model.replicas import max_over_ranks, route, shard, sum_over_ranks, tensor_key
    from dda_model.serving import synthetic_stream

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        reqs = synthetic_stream(n=96, rate=200.0, seed=11)
        # a few requests that share a tensor with an earlier one
        for k in range(0, 12, 3):
            r = reqs[k + 40]
            r.shape, r.lam = reqs[k].shape, reqs[k].lam
        mine = shard(reqs, rank, world)
        gathered = [None] * world
        dist.all_gather_object(gathered, [r.tag for r in mine])
        owners = {}
        for rk, tags in enumerate(gathered):
            for t in tags:
                owners.setdefault(t, []).append(rk)
        key_owner = {}
        ok_keys = True
        for r in reqs:
            k = tensor_key(r)
            ok_keys &= key_owner.setdefault(k, route(r, world)) == route(r, world)
        # timings: rank r took r + 1.5 s for len(mine) requests
        wall = max_over_ranks(rank + 1.5)
        total = sum_over_ranks(len(mine))
        out.put((rank, sorted(owners.items()), ok_keys, wall, total, len(mine)))
    finally:
        dist.destroy_process_group()


def test_two_replicas_route_and_reduce():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    owners = dict(res[0][1])
    assert sorted(owners) == list(range(96))                  # every request served once...
    assert all(len(v) == 1 for v in owners.values())          # ...by exactly one rank
    assert res[0][2] and res[1][2]                             # same tensor key -> same rank
    assert res[0][3] == res[1][3] == pytest.approx(2.5)        # slowest rank's time
    assert res[0][4] == res[1][4] == 96                        # all ranks' requests
    assert 0 < res[0][5] < 96 and res[0][5] + res[1][5] == 96  # both ranks got work
