"""Replica plumbing on two host processes (gloo): the timing collectives and the sharing of independent work.

On the GPUs one rank runs per GPU under torchrun with NCCL; the collectives are the same two (a barrier and a
maximum of durations), so their host-side logic is covered here without a GPU.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp

from cerebrosim_b200.replicas import Replicas


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def worker(rank, world, port, q):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    rep = Replicas("gloo", timeout_s=30)
    try:
        rep.barrier()
        seconds = [2.0, 3.5][rank]
        units = [100.0, 300.0][rank]
        # a sweep shared out: each rank runs its specs, the per-rank results are assembled on every rank
        from cerebrosim_b200 import workloads
        mine = rep.share(workloads.sweep())
        done = [{"seed": sp["seed"], "nodes": sp["nodes"], "rank": rep.rank} for sp in mine]
        out = {"rank": rep.rank, "world": rep.world, "max": rep.max(seconds), "sum": rep.sum(units),
               "rate": rep.rate(units, seconds), "share": rep.share(range(7)), "gathered": rep.gather(done)}
        rep.barrier()
        q.put(out)
    finally:
        rep.close()


def test_two_replicas_over_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=120) for _ in procs), key=lambda r: r["rank"])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in res:
        assert r["world"] == 2
        assert r["max"] == 3.5 and r["sum"] == 400.0
        assert r["rate"] == pytest.approx(400.0 / 3.5)
    assert res[0]["share"] == [0, 2, 4, 6] and res[1]["share"] == [1, 3, 5]
    # every spec of the sweep ran on exactly one rank, and both ranks hold the same assembled list
    from cerebrosim_b200 import workloads
    assert res[0]["gathered"] == res[1]["gathered"]
    ran = sorted(d["seed"] for part in res[0]["gathered"] for d in part)
    assert ran == sorted(sp["seed"] for sp in workloads.sweep())
    assert [d["rank"] for d in res[0]["gathered"][1]] == [1] * len(res[0]["gathered"][1])


def test_single_process_is_a_plain_run(monkeypatch):
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    rep = Replicas("gloo")
    assert (rep.rank, rep.world) == (0, 1)
    assert rep.max(2.5) == 2.5 and rep.rate(10.0, 2.0) == 5.0 and rep.share([1, 2, 3]) == [1, 2, 3]
    rep.barrier()
    rep.close()
