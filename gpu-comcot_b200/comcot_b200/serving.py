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
products are in host memory.  Finished requests' products are copied from
the device behind the running steps into page-locked host memory
(Engine.read_async); the loop takes them when the copy's event completes and
hands them to the file writer's thread, so neither the copies nor the files
hold up the next chunk.

Failure handling (all on the host; nothing faults a GPU): a request the
engine refuses as malformed, or one larger than the whole budget, is marked
"rejected" and the loop goes on; a
request can be cancelled (``cancel_at`` seconds after its arrival, or
``cancel(rid)``) and its memory is freed at the next harvest; a finished
request whose surface held a NaN/Inf or exceeded ``blowup_m`` metres is
marked "diverged" and its products are not returned as a forecast.
"""
from __future__ import annotations

import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from . import outputs
from .engine import Engine


@dataclass
class Request:
    rid: int
    t_arrival: float          # seconds after the start of the trace
    case: object              # synth.Case: layers (shared per class), Z0, gauges, nsteps
    faults: list | None = None  # fault planes: the initial state is generated on the device
    t_admit: float = -1.0
    t_done: float = -1.0
    result: dict = field(default_factory=dict)
    cancel_at: float = float("inf")   # seconds after arrival (wall) to cancel it
    status: str = "pending"           # done | rejected | cancelled | diverged
    error: str = ""
    t_arrival_wall: float = 0.0

    @property
    def latency(self) -> float:
        return self.t_done - self.t_arrival_wall


class ForecastServer:
    """Continuous-batching request loop on one GPU."""

    def __init__(self, budget_bytes: int, chunk: int = 32, variant: int = -1, keep_fields=("zmax", "arrival", "ts"),
                 engine=None, blowup_m: float = 100.0, out_dir: str | None = None):
        """engine: an object with Engine's add/step/sync/done/read/release
        (default: a new Engine with this budget)"""
        self.eng = engine if engine is not None else Engine(budget=budget_bytes)
        self.eng.config(variant=variant, use_graphs=1, chunk=chunk)
        self.chunk = chunk
        self.budget = budget_bytes
        self.keep = keep_fields
        self.max_active = 0
        self.refused = 0      # admission attempts that found no room
        self.blowup_m = blowup_m
        self.idle_retries = 20   # refusals with nothing running before a request is rejected
        self._cancel = set()
        # products of finished requests go to out_dir/req_<rid>/ on a writer thread
        self.out_dir = out_dir
        self.writer = outputs.AsyncWriter() if out_dir else None

    def close(self):
        if self.writer:
            self.writer.close()
        self.eng.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def cancel(self, rid: int):
        """cancels request rid (waiting or running) at the next harvest"""
        self._cancel.add(rid)

    def _try_admit(self, r: Request) -> bool:
        """True when the request left the queue (admitted or rejected)"""
        try:
            mid = self.eng.add_faults(r.case, r.faults) if r.faults else self.eng.add(r.case)
        except MemoryError:
            self.refused += 1
            return False
        except (RuntimeError, ValueError) as exc:
            r.status, r.error = "rejected", str(exc)
            return True
        r._mid = mid
        r.status = "running"
        return True

    def _harvest(self, r: Request) -> bool:
        """True when the request is finished here; False when its results
        are still on their way to host memory (r._pending)"""
        h = self.eng.health(r._mid, self.blowup_m)
        if h:
            r.status = "diverged"
            r.error = ("non-finite surface" if h & 1 else "") + (" |eta| above %g m" % self.blowup_m if h & 2 else "")
            self.eng.release(r._mid)
            return True
        if hasattr(self.eng, "read_async"):
            # copied behind the steps into page-locked memory; the loop goes on
            r._pending = self.eng.read_async(r._mid, fields=self.keep)
            self.eng.release(r._mid)
            r.status = "draining"
            return False
        r.result = self.eng.read(r._mid, fields=self.keep)
        self.eng.release(r._mid)
        self._finish(r)
        return True

    def _finish(self, r: Request):
        r.status = "done"
        if self.writer:
            L = r.case.root
            self.writer.submit(outputs.write_forecast, f"{self.out_dir}/req_{r.rid:05d}", r.result, L.H, L.dt)

    def serve(self, requests, speed: float = 1.0, clock=time.perf_counter):
        """Runs the trace.  Request k arrives t_arrival / speed wall seconds
        after the start (speed = inf: all at once); admit and done times are
        wall seconds after the start, and latency = done - arrival."""
        for r in requests:
            r.t_arrival_wall = r.t_arrival / speed if np.isfinite(speed) else 0.0
        pending = deque(sorted(requests, key=lambda r: r.t_arrival_wall))
        waiting: deque = deque()
        active = []
        idle_refusals = 0
        t0 = clock()

        def take_arrivals():
            """queues what has arrived, drops cancelled requests, admits in
            arrival order while the budget has room; returns the admissions"""
            t = clock() - t0
            while pending and pending[0].t_arrival_wall <= t:
                waiting.append(pending.popleft())
            for r in list(waiting):
                if r.rid in self._cancel or t >= r.t_arrival_wall + r.cancel_at:
                    waiting.remove(r)
                    r.status, r.t_done = "cancelled", t
            n = 0
            while waiting and self._try_admit(waiting[0]):
                r = waiting.popleft()
                r.t_admit = clock() - t0
                n += 1
                if r.status == "rejected":
                    r.t_done = r.t_admit
                else:
                    active.append(r)
            self.max_active = max(self.max_active, len(active))
            return n

        draining = []

        def drain(wait=False):
            """finishes requests whose results have reached host memory"""
            nonlocal draining
            still = []
            for r in draining:
                if wait or r._pending.done():
                    r.result = r._pending.take()
                    r.t_done = clock() - t0
                    self._finish(r)
                else:
                    still.append(r)
            draining = still

        while pending or waiting or active or draining:
            drain()
            if take_arrivals():
                idle_refusals = 0
            if not active:
                if waiting:
                    # nothing runs, so nothing will free memory: retry a few times
                    # (an allocator can refuse transiently), then give the head up
                    idle_refusals += 1
                    if idle_refusals > self.idle_retries:
                        r = waiting.popleft()
                        r.status, r.error, r.t_done = "rejected", "does not fit the HBM budget", clock() - t0
                        idle_refusals = 0
                    else:
                        time.sleep(0.001)
                    continue
                if pending:
                    time.sleep(max(0.0, min(0.002, pending[0].t_arrival_wall - (clock() - t0))))
                elif draining:
                    drain(wait=True)
                continue
            self.eng.step(self.chunk)
            # while the chunk runs: arrivals are admitted now (their state is
            # uploaded behind the chunk) and join at the next one
            while not self.eng.idle():
                take_arrivals()
                drain()
                time.sleep(0.0002)
            self.eng.sync()
            still = []
            t = clock() - t0
            for r in active:
                if r.rid in self._cancel or t >= r.t_arrival_wall + r.cancel_at:
                    self.eng.release(r._mid)
                    r.status, r.t_done = "cancelled", clock() - t0
                elif self.eng.done(r._mid):
                    if self._harvest(r):
                        r.t_done = clock() - t0
                    else:
                        draining.append(r)
                else:
                    still.append(r)
            active = still
        drain(wait=True)
        return requests


class PlainServer:
    """The plain path a warning centre runs without batching: one request at
    a time, in arrival order, through the reference C ABI exactly as the
    Fortran driver calls it (layer upload, then per step MASS, OPEN,
    ALL_GRID, MOMENT, MAX_AMP and the gauge stencils, one kernel per phase),
    products read back when the run ends.  Serves the same traces as
    ForecastServer so their latencies compare on equal terms."""

    def __init__(self, fusion: bool = False):
        from .abi import ReferenceSession

        self._session = ReferenceSession
        self.fusion = fusion
        self.host_cache = {}   # Fortran-order arrays per layer, as the caller holds them

    def prepare(self, requests):
        """builds the callers' host arrays of every grid class in the trace"""
        for r in requests:
            s = self._session(r.case, fusion=self.fusion, init_layers=False, host_cache=self.host_cache)
            s.close()

    def run_one(self, r: Request) -> dict:
        s = self._session(r.case, fusion=self.fusion, arrival=True, host_cache=self.host_cache)
        try:
            st = s.drive(r.case.nsteps, maxamp=True)
            res = {"zmax": s.getzmax(1), "arrival": s.getarrival(1), "ts": gauge_series(st, r.case.gauges)}
        finally:
            s.close()
        return res

    def serve(self, requests, speed: float = 1.0, clock=time.perf_counter):
        for r in requests:
            r.t_arrival_wall = r.t_arrival / speed if np.isfinite(speed) else 0.0
        t0 = clock()
        for r in sorted(requests, key=lambda q: q.t_arrival_wall):
            wait = r.t_arrival_wall - (clock() - t0)
            if wait > 0:
                time.sleep(wait)
            r.t_admit = clock() - t0
            r.result = self.run_one(r)
            r.status = "done"
            r.t_done = clock() - t0
        return requests


def gauge_series(stencils, gauges):
    """GET_TS (output.f90:1078-1090): bilinear interpolation of the 2x2
    stencils [nsteps, ngauges, 4] in float32, left to right"""
    st = np.asarray(stencils, dtype=np.float32)
    out = np.zeros(st.shape[:2], np.float32)
    one = np.float32(1.0)
    for g, (_lid, _ki, _kj, cx, cy) in enumerate(gauges):
        cx, cy = np.float32(cx), np.float32(cy)
        l1, l2, l3, l4 = (st[:, g, q] for q in range(4))
        out[:, g] = l1 * (one - cx) * (one - cy) + l2 * cx * (one - cy) + l3 * (one - cx) * cy + l4 * cx * cy
    return out


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
