"""The serving loop's host logic (admission by HBM footprint, FIFO order,
continuous batching, harvesting) driven by a fake engine on the CPU, and the
one-request-at-a-time queue model."""
import time

import numpy as np
import pytest

from comcot_b200.serving import ForecastServer, Request, fifo_latencies, percentiles


class FakeCase:
    def __init__(self, nsteps, nbytes, bad=0):
        self.nsteps = nsteps
        self.nbytes = nbytes
        self.bad = bad            # health bits the fake device reports at the end


class FakeEngine:
    """members advance one step per step() unit; memory is counted in bytes"""

    def __init__(self, budget, step_seconds=0.0):
        self.budget, self.used = budget, 0
        self.step_seconds = step_seconds
        self.exhausted = 0        # the next n allocations fail as if the pool were exhausted
        self.members = {}
        self.next_id = 0
        self.log = []
        self.steps = 0

    def config(self, **kw):
        pass

    def add(self, case):
        if case.nbytes <= 0:
            raise RuntimeError("gc_engine_add_member failed: -1")
        if self.used + case.nbytes > self.budget or self.exhausted > 0:
            self.exhausted = max(0, self.exhausted - 1)
            raise MemoryError
        mid = self.next_id
        self.next_id += 1
        self.members[mid] = [case, 0]
        self.used += case.nbytes
        self.log.append(("add", mid, self.steps))
        return mid

    def step(self, n):
        time.sleep(self.step_seconds * n)
        self.steps += n
        for m in self.members.values():
            m[1] = min(m[0].nsteps, m[1] + n)

    def sync(self):
        pass

    def idle(self):
        return True     # step() above runs to completion before it returns

    def done(self, mid):
        c, k = self.members[mid]
        return k >= c.nsteps

    def read(self, mid, fields=()):
        return {"steps_run": self.members[mid][1]}

    def health(self, mid, bound):
        return self.members[mid][0].bad

    def release(self, mid):
        self.used -= self.members[mid][0].nbytes
        del self.members[mid]
        self.log.append(("release", mid, self.steps))

    def close(self):
        pass


def test_admission_by_footprint_and_fifo():
    eng = FakeEngine(budget=100)
    reqs = [Request(k, 0.0, FakeCase(nsteps=n, nbytes=b)) for k, (n, b) in
            enumerate([(40, 60), (10, 30), (20, 50), (8, 10)])]
    srv = ForecastServer(100, chunk=4, engine=eng)
    srv.serve(reqs, speed=float("inf"))
    assert all(r.result["steps_run"] == r.case.nsteps for r in reqs)
    order = [m for a, m, _ in eng.log if a == "add"]
    # FIFO: request 2 (50 B) waits for room, request 3 may not overtake it
    assert order == [0, 1, 2, 3]
    adds = {m: s for a, m, s in eng.log if a == "add"}
    rels = {m: s for a, m, s in eng.log if a == "release"}
    assert adds[2] >= rels[1]                  # admitted only after request 1 freed its memory
    assert srv.refused >= 1
    assert srv.max_active == 2
    assert eng.used == 0


def test_oversized_and_malformed_requests_are_rejected_and_the_rest_served():
    eng = FakeEngine(budget=10)
    reqs = [Request(0, 0.0, FakeCase(5, 11)), Request(1, 0.0, FakeCase(5, -1)), Request(2, 0.0, FakeCase(5, 4))]
    ForecastServer(10, engine=eng).serve(reqs, speed=float("inf"))
    assert [r.status for r in reqs] == ["rejected", "rejected", "done"]
    assert "budget" in reqs[0].error and reqs[2].result["steps_run"] == 5
    assert eng.used == 0


def test_cancellation_frees_memory_for_waiting_requests():
    eng = FakeEngine(budget=10, step_seconds=1e-3)
    long_run = Request(0, 0.0, FakeCase(100000, 8), cancel_at=0.05)
    queued = Request(1, 0.0, FakeCase(10, 8))
    never = Request(2, 0.0, FakeCase(10, 8), cancel_at=0.0)
    srv = ForecastServer(10, chunk=4, engine=eng)
    srv.serve([long_run, never, queued], speed=float("inf"))
    assert long_run.status == "cancelled" and never.status == "cancelled"
    assert queued.status == "done" and queued.t_admit >= long_run.t_done
    assert eng.used == 0


def test_diverged_request_is_not_returned_as_a_forecast():
    eng = FakeEngine(budget=100)
    reqs = [Request(0, 0.0, FakeCase(8, 10, bad=1)), Request(1, 0.0, FakeCase(8, 10, bad=2)),
            Request(2, 0.0, FakeCase(8, 10))]
    ForecastServer(100, engine=eng).serve(reqs, speed=float("inf"))
    assert [r.status for r in reqs] == ["diverged", "diverged", "done"]
    assert reqs[0].result == {} and "non-finite" in reqs[0].error and "above" in reqs[1].error


def test_allocator_exhaustion_is_retried_not_fatal():
    eng = FakeEngine(budget=100, step_seconds=1e-4)
    eng.exhausted = 3                            # the pool refuses the next three attempts
    reqs = [Request(0, 0.0, FakeCase(20, 10)), Request(1, 0.0, FakeCase(20, 10))]
    srv = ForecastServer(100, chunk=2, engine=eng)
    srv.serve(reqs, speed=float("inf"))
    assert [r.status for r in reqs] == ["done", "done"]
    assert srv.refused == 3


def test_arrivals_join_a_running_batch():
    eng = FakeEngine(budget=1000, step_seconds=1e-3)
    reqs = [Request(0, 0.0, FakeCase(200, 10)), Request(1, 0.02, FakeCase(10, 10))]
    srv = ForecastServer(1000, chunk=2, engine=eng)
    srv.serve(reqs, speed=1.0)
    # the second request was admitted while the first was still running
    assert reqs[1].t_admit < reqs[0].t_done
    assert reqs[1].t_done < reqs[0].t_done
    assert all(r.latency >= 0 for r in reqs)


def test_fifo_model_and_percentiles():
    lat, end = fifo_latencies([0.0, 0.5, 0.6], [1.0, 1.0, 1.0])
    assert np.allclose(lat, [1.0, 1.5, 2.4]) and end == 3.0
    p = percentiles(np.arange(101))
    assert p["p50"] == 50.0 and p["p99"] == 99.0


def test_finished_requests_products_written_in_background(tmp_path):
    import types

    class Eng(FakeEngine):
        def read(self, mid, fields=()):
            return {"zmax": np.full((2, 3), 0.25, np.float32), "ts": np.zeros((2, 1), np.float32),
                    "arrival": np.full((2, 3), -1, np.int32)}

    case = FakeCase(4, 10)
    case.root = types.SimpleNamespace(H=np.ones((2, 3), np.float32), dt=2.0)
    with ForecastServer(100, engine=Eng(budget=100), out_dir=str(tmp_path)) as srv:
        srv.serve([Request(7, 0.0, case)], speed=float("inf"))
    import os
    assert sorted(os.listdir(tmp_path / "req_00007")) == ["arrival_layer01.dat", "ts_record0001.dat",
                                                          "zmax_layer01.dat"]
