"""Forecast serving for a tsunami warning system: continuous batching over
the engine (gc_engine_* in include/gcomcot.h).

Requests (a source, a grid class, a duration and gauges) arrive while
others are on the GPU.  A request is admitted, in arrival order, as soon as
the engine's HBM budget has room for its state; it then joins the running
batch at the next step and its grids stay resident until it completes.
Every few steps the loop harvests finished requests (gauge series, max-eta
and arrival steps), frees their memory and admits waiting ones.  A result
does not depend on what else was in the batch: every member's kernels read
and write only that member's state.

Time-to-forecast is measured per request from its arrival to the moment its
products are in host memory.
"""
from __future__ import annotations

import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from .engine import Engine


@dataclass
class Request:
    rid: int
    t_arrival: float          # seconds after the start of the trace
    case: object              # synth.Case: layers (shared per class), Z0, gauges, nsteps
    t_admit: float = -1.0
    t_done: float = -1.0
    result: dict = field(default_factory=dict)

    t_arrival_wall: float = 0.0

    @property
    def latency(self) -> float:
        return self.t_done - self.t_arrival_wall


class ForecastServer:
    """Continuous-batching request loop on one GPU."""

    def __init__(self, budget_bytes: int, chunk: int = 32, variant: int = -1, keep_fields=("zmax", "arrival", "ts"),
                 engine=None):
        """engine: an object with Engine's add/step/sync/done/read/release
        (default: a new Engine with this budget)"""
        self.eng = engine if engine is not None else Engine(budget=budget_bytes)
        self.eng.config(variant=variant, use_graphs=1, chunk=chunk)
        self.chunk = chunk
        self.budget = budget_bytes
        self.keep = keep_fields
        self.max_active = 0
        self.refused = 0      # admission attempts that found no room

    def close(self):
        self.eng.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _try_admit(self, r: Request) -> bool:
        try:
            mid = self.eng.add(r.case)
        except MemoryError:
            self.refused += 1
            return False
        r._mid = mid
        return True

    def _harvest(self, r: Request):
        out = self.eng.read(r._mid, fields=self.keep)
        self.eng.release(r._mid)
        r.result = out

    def serve(self, requests, speed: float = 1.0, clock=time.perf_counter):
        """Runs the trace.  Request k arrives t_arrival / speed wall seconds
        after the start (speed = inf: all at once); admit and done times are
        wall seconds after the start, and latency = done - arrival."""
        for r in requests:
            r.t_arrival_wall = r.t_arrival / speed if np.isfinite(speed) else 0.0
        pending = deque(sorted(requests, key=lambda r: r.t_arrival_wall))
        waiting: deque = deque()
        active = []
        t0 = clock()
        while pending or waiting or active:
            t = clock() - t0
            while pending and pending[0].t_arrival_wall <= t:
                waiting.append(pending.popleft())
            while waiting and self._try_admit(waiting[0]):
                r = waiting.popleft()
                r.t_admit = clock() - t0
                active.append(r)
            self.max_active = max(self.max_active, len(active))
            if not active:
                if waiting:
                    raise RuntimeError(f"request {waiting[0].rid} does not fit the engine budget alone")
                if pending:
                    time.sleep(max(0.0, min(0.002, pending[0].t_arrival_wall - (clock() - t0))))
                continue
            self.eng.step(self.chunk)
            self.eng.sync()
            still = []
            for r in active:
                if self.eng.done(r._mid):
                    self._harvest(r)
                    r.t_done = clock() - t0
                else:
                    still.append(r)
            active = still
        return requests


def percentiles(x, qs=(50, 99)):
    x = np.sort(np.asarray(x, dtype=np.float64))
    return {f"p{q}": float(np.percentile(x, q)) for q in qs}


def fifo_latencies(arrivals, service):
    """one-request-at-a-time server: completion of k = max(arrival_k, done_{k-1}) + service_k"""
    done = 0.0
    lat = []
    for a, s in sorted(zip(arrivals, service)):
        start = max(a, done)
        done = start + s
        lat.append(done - a)
    return np.array(lat), done
