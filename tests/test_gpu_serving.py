"""Serving: requests that arrive while others run are admitted by HBM
footprint and batched; each request's products (gauge series, max-eta,
arrival steps) are the same alone and in the mix, and equal the oracle's."""
import numpy as np
import pytest

from comcot_b200 import synth
from comcot_b200.engine import Engine
from comcot_b200.serving import ForecastServer, Request

pytestmark = pytest.mark.gpu

SIZES = ((161, 121), (181, 131))


def _trace():
    tpl = synth.config_c5_templates(seed=70, sizes=SIZES)
    rng = np.random.default_rng(71)
    reqs = []
    t = 0.0
    for k in range(8):
        t += float(rng.exponential(0.01))
        size = SIZES[k % 2]
        nested = k % 3 == 1
        nsteps = int(rng.integers(30, 70))
        reqs.append(Request(k, t, synth.c5_request_case(tpl, size, nsteps, nested, seed=1000 + k)))
    return reqs


def _alone(case):
    with Engine(budget=1 << 30) as eng:
        mid = eng.add(case)
        eng.step(case.nsteps + 1)
        eng.sync()
        return eng.read(mid, fields=("zmax", "arrival", "ts"))


def test_served_results_equal_alone_and_oracle(oracle_mod):
    reqs = _trace()
    # every request arrives at once; the budget holds the grid classes and
    # only some of the requests, so the rest wait for memory to free up
    with ForecastServer(budget_bytes=10 << 20, chunk=8) as srv:
        srv.serve(reqs, speed=float("inf"))
        assert srv.refused > 0            # some requests waited for memory
        assert srv.max_active >= 2        # and others overlapped on the GPU
    for r in reqs:
        assert r.t_done >= r.t_admit >= r.t_arrival_wall
        a = _alone(r.case)
        for k in ("zmax", "ts"):
            assert np.array_equal(r.result[k].view(np.uint32), a[k].view(np.uint32)), (r.rid, k)
        assert np.array_equal(r.result["arrival"], a["arrival"])
    for r in (reqs[0], reqs[1]):
        o = oracle_mod.OracleRun(r.case)
        ts = o.run(r.case.nsteps)
        ref = o.layer(0)
        assert np.array_equal(r.result["zmax"].view(np.uint32), ref["zmax"].view(np.uint32))
        assert np.array_equal(r.result["arrival"], ref["arrival"])
        assert np.array_equal(r.result["ts"].view(np.uint32), ts.view(np.uint32))
