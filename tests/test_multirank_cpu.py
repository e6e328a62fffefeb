"""Replica (multi-GPU) host logic on CPU: two gloo ranks as child processes.
The data path has no collective; the group carries the max-over-ranks
timing and the summaries, and a rank that dies is found by its missing
heartbeat and result instead of being waited for."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, mode, out):
    sys.path.insert(0, os.path.join(HERE, "..", "gpu-comcot_b200"))
    import datetime

    import torch.distributed as dist
    from torch.distributed import TCPStore

    from comcot_b200 import replicas

    store = TCPStore("127.0.0.1", port + 1, world, rank == 0, timeout=datetime.timedelta(seconds=20))
    hb = replicas.Heartbeat(store, rank, world)
    hb.beat()
    if mode == "dies" and rank == 1:
        os._exit(0)                                   # leaves between steps, before any collective
    if mode == "ok":
        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                                timeout=datetime.timedelta(seconds=20))
        mine = replicas.shard(range(10), rank, world)
        t_max = replicas.reduce_max(1.0 + rank, dist)
        total = replicas.reduce_sum(len(mine), dist)
        replicas.publish(store, rank, {"items": mine})
        if rank == 0:
            got, missing = replicas.gather(store, world, timeout_s=10)
            out.put({"t_max": t_max, "total": total, "items": sorted(sum((g["items"] for g in got.values()), [])),
                     "missing": missing})
        dist.barrier()
        dist.destroy_process_group()
    else:
        replicas.publish(store, rank, {"items": replicas.shard(range(10), rank, world)})
        if rank == 0:
            got, missing = replicas.gather(store, world, timeout_s=1.0)
            out.put({"missing": missing, "dead": hb.dead(stale_s=30.0), "got": sorted(got)})


def _run(mode):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, mode, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = q.get(timeout=60)
    for p in ps:
        p.join(timeout=60)
    assert all(p.exitcode == 0 for p in ps)
    return res


def test_replicas_shard_and_reduce_over_two_gloo_ranks():
    r = _run("ok")
    assert r["t_max"] == 2.0 and r["total"] == 10.0
    assert r["items"] == list(range(10)) and r["missing"] == []


def test_dead_rank_is_reported_not_waited_for():
    r = _run("dies")
    assert r["missing"] == [1] and r["got"] == [0]
    assert r["dead"] == []          # it beat once before dying; only the missing result shows it


def test_shard_rejects_bad_rank():
    sys.path.insert(0, os.path.join(HERE, "..", "gpu-comcot_b200"))
    from comcot_b200 import replicas

    with pytest.raises(ValueError):
        replicas.shard([1, 2], 2, 2)
    assert replicas.shard(range(5), 1, 2) == [1, 3]


def _serve_worker(rank, world, port, dies, out):
    """each rank serves its round-robin share of a trace (forecast server
    over the fake engine of the serving tests); rank 0 gathers the ranks'
    latencies through the store with a bounded wait"""
    sys.path.insert(0, os.path.join(HERE, "..", "gpu-comcot_b200"))
    sys.path.insert(0, HERE)
    import datetime

    from torch.distributed import TCPStore

    from comcot_b200 import replicas
    from comcot_b200.serving import ForecastServer, Request, percentiles
    from test_serving_cpu import FakeCase, FakeEngine

    store = TCPStore("127.0.0.1", port + 1, world, rank == 0, timeout=datetime.timedelta(seconds=20))
    hb = replicas.Heartbeat(store, rank, world)
    hb.beat()
    trace = [(0.001 * k, 10 + 3 * k, 10) for k in range(12)]
    mine = replicas.shard(trace, rank, world)
    reqs = [Request(k, t, FakeCase(nsteps=n, nbytes=b)) for k, (t, n, b) in enumerate(mine)]
    srv = ForecastServer(100, chunk=4, engine=FakeEngine(budget=100))
    srv.serve(reqs, speed=float("inf"))
    if dies and rank == 1:
        os._exit(0)                       # leaves after its work, before reporting it
    lat = [r.latency for r in reqs]
    got, missing, stale = replicas.collect(store, rank, world, {"lat": lat, "done": [r.status for r in reqs]},
                                           timeout_s=2.0, hb=hb)
    if rank == 0:
        merged = sum((g["lat"] for g in got.values()), [])
        out.put({"n": len(merged), "missing": missing, "p99": percentiles(merged)["p99"],
                 "done": sum((g["done"] for g in got.values()), [])})


def _run_serve(dies):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    ps = [ctx.Process(target=_serve_worker, args=(r, 2, port, dies, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = q.get(timeout=60)
    for p in ps:
        p.join(timeout=60)
    assert all(p.exitcode == 0 for p in ps)
    return res


def test_served_shares_are_gathered_over_two_ranks():
    r = _run_serve(dies=False)
    assert r["n"] == 12 and r["missing"] == [] and set(r["done"]) == {"done"}
    assert r["p99"] >= 0.0


def test_serving_rank_that_dies_is_reported_not_waited_for():
    r = _run_serve(dies=True)
    assert r["missing"] == [1] and r["n"] == 6
