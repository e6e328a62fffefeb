"""Multi-GPU as replicas: one process per GPU, independent forecasts
(ensemble scenarios, served requests, replicas of one configuration) split
over the ranks with no exchange on the data path.  The process group carries
only the timing reduction (max over ranks) and the final summaries; a
TCPStore heartbeat lets rank 0 find ranks that died and report their share of
the work as unserved instead of waiting for them.
"""
from __future__ import annotations

import json
import time


def shard(items, rank: int, world: int):
    """round-robin share of `items` for `rank` (balances mixed request sizes)"""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world {world}")
    return list(items)[rank::world]


def reduce_max(value: float, dist=None, device=None) -> float:
    """max of a per-rank scalar (device timings are reported as the max)"""
    if dist is None:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(value: float, dist=None, device=None) -> float:
    if dist is None:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


class Heartbeat:
    """liveness through a key-value store: each rank stamps hb/<rank>"""

    def __init__(self, store, rank: int, world: int):
        self.store, self.rank, self.world = store, rank, world

    def beat(self):
        self.store.set(f"hb/{self.rank}", repr(time.time()))

    def last_seen(self, rank: int):
        if not self._has(f"hb/{rank}"):
            return None
        return float(self.store.get(f"hb/{rank}").decode())

    def dead(self, stale_s: float):
        """ranks with no beat in the last stale_s seconds (or none at all)"""
        now = time.time()
        out = []
        for r in range(self.world):
            t = self.last_seen(r)
            if t is None or now - t > stale_s:
                out.append(r)
        return out

    def _has(self, key):
        return self.store.check([key])


def publish(store, rank: int, summary: dict):
    store.set(f"result/{rank}", json.dumps(summary))


def gather(store, world: int, timeout_s: float, poll_s: float = 0.02):
    """rank 0's collection of every rank's summary, waiting at most
    timeout_s; returns ({rank: summary}, [ranks that never published])"""
    deadline = time.time() + timeout_s
    got = {}
    while True:
        for r in range(world):
            if r not in got and store.check([f"result/{r}"]):
                got[r] = json.loads(store.get(f"result/{r}").decode())
        if len(got) == world or time.time() >= deadline:
            break
        time.sleep(poll_s)
    return got, [r for r in range(world) if r not in got]


def default_store(dist):
    """the key-value store of the default process group (None where the
    build does not expose it)"""
    try:
        from torch.distributed import distributed_c10d as c10d

        return c10d._get_default_store()
    except Exception:
        return None


def collect(store, rank: int, world: int, summary: dict, timeout_s: float, hb: Heartbeat | None = None):
    """every rank publishes its summary; rank 0 waits at most timeout_s for
    the others and returns ({rank: summary}, missing ranks, ranks whose
    heartbeat is older than timeout_s); other ranks return (None, None, None).
    A rank that died is reported, not waited for."""
    if hb is not None:
        hb.beat()
    publish(store, rank, summary)
    if rank != 0:
        return None, None, None
    got, missing = gather(store, world, timeout_s)
    stale = hb.dead(stale_s=timeout_s) if hb is not None else []
    return got, missing, stale
