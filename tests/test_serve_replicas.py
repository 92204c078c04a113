"""The served stream on several GPUs as independent replicas (no data-path
collective): each rank serves its shard of the stream with its own batch, and
the ranks' statistics are gathered once at the end.  Runs as two gloo ranks on
the CPU with a fake batch (the device work of one replica is the single-GPU
server, tested on the GPU elsewhere)."""
from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def _rank_main(rank, world, port, outdir):
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "smaug-all_b200" / "python"))
    sys.path.insert(0, str(ROOT / "tests"))
    import datetime

    import torch.distributed as dist

    from smaug_b200.serve import Request, Server, merge_stats, shard
    from test_serve_logic import Clock, FakeBatch, prob
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    reqs = [Request(i, prob(i, 2 + i % 3), 4 + i % 5, 0.002 * i) for i in range(25)]  # the same stream on every rank
    mine = shard(reqs, rank, world)
    ck = Clock()
    srv = Server(FakeBatch(capacity=6), chunk=2, depth=2)
    st = srv.run(mine, clock=ck, sleep=ck.sleep)
    gathered = [None] * world
    dist.all_gather_object(gathered, (st, srv.latencies, [r.rid for r in mine if r.done is not None]))
    if rank == 0:
        merged = merge_stats([(g[0], g[1]) for g in gathered])
        served = sorted(rid for g in gathered for rid in g[2])
        np.save(Path(outdir) / "served.npy", np.array(served))
        np.save(Path(outdir) / "merged.npy", np.array([merged["requests"], merged["completed"],
                                                       merged["cell_updates"]]))
    dist.destroy_process_group()


def test_two_replicas_serve_every_request_once(tmp_path):
    import socket

    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn", join=True)
    served = np.load(tmp_path / "served.npy")
    assert list(served) == list(range(25))
    requests, completed, cu = np.load(tmp_path / "merged.npy")
    assert requests == 25 and completed == 25
    assert cu == sum((2 + i % 3) * (4 + i % 5) for i in range(25))


def test_shards_partition_the_stream():
    from smaug_b200.serve import Request, shard
    reqs = [Request(i, None, 1, float(i)) for i in range(10)]
    parts = [shard(reqs, r, 3) for r in range(3)]
    assert sorted(x.rid for p in parts for x in p) == list(range(10))
    assert [x.rid for x in parts[1]] == [1, 4, 7]
