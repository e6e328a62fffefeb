"""The serving loop's host logic (admission by HBM footprint, FIFO order,
continuous batching, harvesting) driven by a fake engine on the CPU, and the
one-request-at-a-time queue model."""
import time

import numpy as np
import pytest

from comcot_b200.serving import ForecastServer, Request, fifo_latencies, percentiles


class FakeCase:
    def __init__(self, nsteps, nbytes):
        self.nsteps = nsteps
        self.nbytes = nbytes


class FakeEngine:
    """members advance one step per step() unit; memory is counted in bytes"""

    def __init__(self, budget, step_seconds=0.0):
        self.budget, self.used = budget, 0
        self.step_seconds = step_seconds
        self.members = {}
        self.next_id = 0
        self.log = []
        self.steps = 0

    def config(self, **kw):
        pass

    def add(self, case):
        if self.used + case.nbytes > self.budget:
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

    def done(self, mid):
        c, k = self.members[mid]
        return k >= c.nsteps

    def read(self, mid, fields=()):
        return {"steps_run": self.members[mid][1]}

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


def test_request_larger_than_budget_is_an_error():
    srv = ForecastServer(10, engine=FakeEngine(budget=10))
    with pytest.raises(RuntimeError):
        srv.serve([Request(0, 0.0, FakeCase(5, 11))], speed=float("inf"))


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
