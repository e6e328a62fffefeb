"""Failure detection on the GPU, in the forms that fault nothing:
  - a bounded pipeline wait that runs out: the two-step kernel is told to
    wait for a row no copy delivers (no copy is issued for it); the wait gives
    up after a short poll limit, the kernel returns, gc_engine_sync reports
    GC_ETIMEOUT, and the context keeps working;
  - a member whose initial surface holds a NaN: gc_engine_member_health sets
    bit 0 and the forecast server marks the request "diverged" while the
    other request in the batch completes.
"""
import math
import time

import numpy as np
import pytest

from comcot_b200 import _lib, serving, synth
from comcot_b200.engine import Engine

pytestmark = pytest.mark.gpu

GC_ETIMEOUT = -5


def _case(nx, ny, seed, nsteps):
    return synth.single_layer_case("f", nx, ny, 2.0, 2.0, nsteps, seed=seed, n_seamounts=3,
                                   shelf_cols=max(2, nx // 10), land_cols=max(1, nx // 30), source="dipole",
                                   ngauges=2)


def test_bounded_wait_gives_up_and_is_reported():
    lib = _lib.load()
    n1 = 2 * lib.gc_engine_num_variants()
    case = _case(300, 140, 5, 30)
    try:
        with Engine(budget=1 << 30) as eng:
            eng.config(variant=n1, use_graphs=0, chunk=8)   # a two-step candidate, eager launches
            eng.add(case)
            eng.step(2)
            assert lib.gc_engine_sync(eng.h) == 0
            lib.gcomcot_set_wait_limit(2000)
            lib.gcomcot_inject_stall()
            t0 = time.perf_counter()
            eng.step(2)                                     # one two-step launch, its first warp stalls
            rc = lib.gc_engine_sync(eng.h)
            waited = time.perf_counter() - t0
            assert rc == GC_ETIMEOUT
            assert waited < 30.0
            # the flag was taken; the context keeps working
            eng.step(4)
            assert lib.gc_engine_sync(eng.h) == 0
    finally:
        lib.gcomcot_set_wait_limit(0)


def test_nan_member_is_flagged_and_served_as_diverged():
    case = _case(97, 81, 6, 20)
    L = case.root
    j, i = np.argwhere(L.H > 100.0)[len(np.argwhere(L.H > 100.0)) // 2]
    z_bad = L.Z0.copy()
    z_bad[j, i] = np.nan
    with Engine(budget=1 << 30) as eng:
        bad = eng.add(case, z0=z_bad)
        good = eng.add(case)
        eng.step(22)
        eng.sync()
        assert eng.health(bad) & 1
        assert eng.health(good) == 0
    bad_case = synth.Case("bad", [synth.LayerSpec(**{**L.__dict__, "Z0": z_bad})], case.nsteps,
                          gauges=case.gauges)
    reqs = [serving.Request(0, 0.0, bad_case), serving.Request(1, 0.0, case)]
    with serving.ForecastServer(1 << 30, chunk=8) as srv:
        srv.serve(reqs, speed=math.inf)
    assert reqs[0].status == "diverged" and "non-finite" in reqs[0].error
    assert reqs[1].status == "done" and reqs[1].result["zmax"].shape == (L.ny, L.nx)
