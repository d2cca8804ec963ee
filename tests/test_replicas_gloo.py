"""The replica path's host logic with two gloo ranks on CPU: per-rank streams
differ and are seeded, reductions take the slowest rank and the total rays,
latencies are gathered in rank order."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from xtracer_b200 import replicas, scenes


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
    out = dict(rank=rank, seeds=[j.seed for j in jobs], shapes=[(j.scene, j.width, j.spp) for j in jobs],
               tmax=g.max(t), rays=g.sum(rays), lat=g.gather([float(rank)] * (rank + 2)))
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
    # each rank serves the seeded stream of its own rank (seed 4 + rank), made
    # inside the rank's process: its jobs' seeds and shapes are that stream's,
    # and no sample seed is shared between the ranks
    for r in (0, 1):
        want = scenes.job_stream(16, seed=4 + r)
        assert res[r]["seeds"] == [j.seed for j in want]
        assert res[r]["shapes"] == [(j.scene, j.width, j.spp) for j in want]
    assert not set(res[0]["seeds"]) & set(res[1]["seeds"])
    assert res[0]["shapes"] != res[1]["shapes"]


def test_single_rank_is_identity():
    g = replicas.Group(1)
    assert g.max(3.0) == 3.0 and g.sum(4.0) == 4.0 and g.gather([1.0, 2.0]) == [1.0, 2.0]
