"""CPU: the multi-rank logic of bench.py's weak-scaling run, on two gloo ranks.

Seeds are independent, so ranks exchange nothing on the data path: each rank scans its own
contiguous seed range (shard()), and the only collective steps are the max-reduce of timings
and the sum of survivor counts.  The per-rank work here is the C oracle (no GPU), standing in
for the engine, to check that the shards are disjoint, cover the stream, and that the reduced
survivor list equals a single-process scan.
"""
from __future__ import annotations

import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, n_total, queue):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "tests"))
    sys.path.insert(0, os.path.join(root, "oracle"))
    import torch
    from conftest import load_package
    import bind
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    wg = load_package()
    lo, hi = wg.shard(n_total, rank, world)
    port_ = bind.Port()
    surv, hist = port_.scan_seeds(bind.rules("1.19.x~26.1"), 0, (-4, 5, -4, 5), gen=(2 + lo, hi - lo), threads=1)
    t = torch.tensor([float(rank + 1)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    counts = torch.tensor(hist, dtype=torch.int64)
    dist.all_reduce(counts)
    gathered = [None] * world
    dist.all_gather_object(gathered, [(int(c["seed_index"]) + lo, int(c["rx"]), int(c["rz"])) for c in surv])
    if rank == 0:
        queue.put((float(t.item()), counts.tolist(), sorted(sum(gathered, []))))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_seed_shards(port):
    n_total = 6000
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    p = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, p, n_total, queue)) for r in range(2)]
    for pr in procs:
        pr.start()
    tmax, counts, survivors = queue.get(timeout=120)
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    assert tmax == 2.0
    import bind
    whole, hist = port.scan_seeds(bind.rules("1.19.x~26.1"), 0, (-4, 5, -4, 5), gen=(2, n_total))
    assert counts == hist.tolist()
    assert sum(counts) == n_total * 81
    assert survivors == sorted((int(c["seed_index"]), int(c["rx"]), int(c["rz"])) for c in whole)
