"""Multi-rank host logic of bench.py on CPU: two gloo ranks, each with its
own shard of batched scenes (weak scaling: no data-path collective), and the
cross-rank max-of-times / sum-of-work reductions the headline number uses."""
import importlib
import os
import socket
import sys
from datetime import timedelta

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        bench = importlib.import_module("bench")
        red = bench.RankReducer(dist, "cpu")
        red.barrier()
        ms = red.max(10.0 + rank)                      # slowest rank sets the time
        units = red.sum(1000.0 * (rank + 1))           # all ranks' work counts
        specs = bench.batched_specs(6, rank)
        out.put((rank, ms, units, [float(s.bodies[:, :3].sum()) for s in specs],
                 sum(s.n_bodies for s in specs)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_reduce():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, ms0, u0, sig0, n0), (r1, ms1, u1, sig1, n1) = res
    assert ms0 == ms1 == 11.0
    assert u0 == u1 == 3000.0
    assert not set(sig0) & set(sig1), "each rank steps its own scenes"
    assert n0 > 0 and n1 > 0


def test_single_process_reducer_is_identity():
    sys.path.insert(0, ROOT)
    bench = importlib.import_module("bench")
    red = bench.RankReducer(None)
    assert red.max(3.5) == 3.5 and red.sum(2.0) == 2.0
    red.barrier()
