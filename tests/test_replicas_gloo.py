"""The replica path's host logic with two gloo ranks on CPU: per-rank streams
differ and are seeded, reductions take the slowest rank and the total rays,
latencies are gathered in rank order."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from xtracer_b200 import replicas


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    g = replicas.Group(world, backend="gloo", timeout_s=60)
    jobs = replicas.rank_stream(rank, n_jobs=16)
    t = 1.0 + rank            # rank 1 is slower
    rays = 1000 * (rank + 1)
    out = dict(rank=rank, first=(jobs[0].scene, jobs[0].width, jobs[0].spp), tmax=g.max(t), rays=g.sum(rays),
               lat=g.gather([float(rank)] * (rank + 2)))
    g.barrier()
    g.close()
    q.put(out)


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=120) for _ in procs], key=lambda d: d["rank"])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0]["tmax"] == res[1]["tmax"] == 2.0
    assert res[0]["rays"] == res[1]["rays"] == 3000
    assert res[0]["lat"] == res[1]["lat"] == [0.0, 0.0, 1.0, 1.0, 1.0]
    assert res[0]["first"] != res[1]["first"] or replicas.rank_stream(0, 16)[1:] != replicas.rank_stream(1, 16)[1:]
    assert replicas.rank_stream(1, 16)[0].seed == replicas.rank_stream(1, 16)[0].seed


def test_single_rank_is_identity():
    g = replicas.Group(1)
    assert g.max(3.0) == 3.0 and g.sum(4.0) == 4.0 and g.gather([1.0, 2.0]) == [1.0, 2.0]
