"""The N > 1 paths on CPU: two gloo ranks run the aggregation the bench uses
(max over ranks of the timed region, barrier) and the sharding of the
batched sweep (instances split by cell count, no exchange between ranks)."""
import datetime
import multiprocessing as mp
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, q):
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    import bench
    from gpk_b200.sweep import lamellar_side, shard
    out = {"max": bench._allmax(float(rank + 1) * 1.5, ws)}
    bench._barrier(ws)
    sizes = [lamellar_side(5000 + i) ** 2 for i in range(96)]
    out["part"] = shard(sizes, ws)[rank]
    out["sizes"] = sizes
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, out))


def test_two_gloo_ranks_aggregate_and_shard():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0]["max"] == res[1]["max"] == 3.0
    a, b = set(res[0]["part"]), set(res[1]["part"])
    sizes = res[0]["sizes"]
    assert not (a & b) and a | b == set(range(len(sizes)))
    load = [sum(sizes[i] for i in a), sum(sizes[i] for i in b)]
    assert abs(load[0] - load[1]) <= max(sizes)


def test_shard_is_deterministic_and_balanced():
    from gpk_b200.sweep import lamellar_side, shard
    sizes = [lamellar_side(5000 + i) ** 2 for i in range(512)]
    for n in (1, 2, 3, 8):
        parts = shard(sizes, n)
        assert parts == shard(sizes, n)
        assert sorted(i for p in parts for i in p) == list(range(512))
        loads = [sum(sizes[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(sizes)
