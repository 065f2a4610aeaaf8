"""The N > 1 path of bench.py on CPU: two gloo ranks run the same rank
plumbing the GPU replicas use (barrier, max of the per-rank times, sum of the
per-rank work, round-robin sharding of ensemble instances)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from cases import ROOT

sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    r = bench.Ranks("gloo", timeout_s=60)
    try:
        assert (r.rank, r.world) == (rank, world)
        r.barrier()
        # per-rank "device times" and "work": the slowest rank sets the time
        t = r.max(1.0 + rank)
        w = r.sum(10.0 * (rank + 1))
        mine = bench.shard(96, rank, world)
        n_all = int(r.sum(float(len(mine))))
        q.put((rank, t, w, mine[:3], n_all, bench.aggregate_rate(w, t)))
    finally:
        r.close()


def test_two_gloo_ranks_reduce_and_shard():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = sorted(q.get(timeout=10) for _ in range(world))
    for rank, t, w, head, n_all, rate in res:
        assert t == 2.0 and w == 30.0 and n_all == 96
        assert head == [rank, rank + 2, rank + 4]
        assert rate == 15.0


def test_single_process_ranks_are_identity():
    r = bench.Ranks("gloo")
    assert r.world == 1 and r.max(3.5) == 3.5 and r.sum(2.0) == 2.0
    r.barrier()
    r.close()
    parts = [bench.shard(10, k, 3) for k in range(3)]
    assert sorted(i for p in parts for i in p) == list(range(10))
