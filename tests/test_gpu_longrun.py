"""Parity over whole forecasts, not a few dozen steps.

C1 (361 x 301 at 2', Gaussian hump, OPEN on four sides, dt 2 s) runs its full
3600 steps; the float stepping's own error against an FP64 twin reaches
2.4e-2 of max eta there (the radiation boundary's sign flips), which is where
a divergence between the device and the oracle would show.  C3's nested pair
(1201 x 1001 linear spherical outer grid, 601 x 501 nonlinear Cartesian child
with wet/dry and Manning friction, ratio 5) runs 600 outer steps.  Each runs
through the batched engine and through the reference C ABI (the call sequence
of comcot.f90:359-439), and is compared with the FP32 oracle run for the same
number of steps: surface, fluxes, max-eta, arrival steps and gauge series, at
the stated tolerance (max|d eta| <= 1e-4 max|eta|, max|d(M,N)| <= 1e-4
max|M,N|, masks and arrival exact) and bit for bit.
"""
import os

import numpy as np
import pytest

from comcot_b200 import synth
from comcot_b200.abi import ReferenceSession
from comcot_b200.engine import Engine

pytestmark = pytest.mark.gpu

TOL = 1e-4
F32 = np.float32
THREADS = os.cpu_count() or 1


def _check(got, want, what):
    """tolerance first (the stated bar), then bit equality (the design point)"""
    assert got.shape == want.shape, what
    scale = max(float(np.abs(want).max()), 1e-30)
    err = float(np.abs(got.astype(np.float64) - want.astype(np.float64)).max())
    assert err <= TOL * scale, f"{what}: max|diff| {err} > {TOL} x {scale}"
    bad = np.flatnonzero(got.view(np.uint32) != want.view(np.uint32))
    assert bad.size == 0, f"{what}: {bad.size} cells differ in their bits, first at {bad[0]}"


def _interp(stencils, gauges):
    """GET_TS (output.f90:1078-1090) on the 2x2 stencils gcomcot_drive returns"""
    out = np.zeros(stencils.shape[:2], F32)
    one = F32(1.0)
    for g, (_lid, _ki, _kj, cx, cy) in enumerate(gauges):
        cx, cy = F32(cx), F32(cy)
        l1, l2, l3, l4 = (stencils[:, g, q] for q in range(4))
        out[:, g] = l1 * (one - cx) * (one - cy) + l2 * cx * (one - cy) + l3 * (one - cx) * cy + l4 * cx * cy
    return out


def test_c1_full_forecast_engine_and_reference_abi(oracle_mod):
    nsteps = 3600
    case = synth.config_c1(nsteps=nsteps)
    case.gauges = synth.wet_gauges(case.root, 8, np.random.default_rng(11))
    o = oracle_mod.OracleRun(case)
    ots = o.run(nsteps, threads=THREADS)
    ref = o.layer(0)
    assert (ref["arrival"] > 0).sum() > 1000  # the wave crossed most of the basin

    with Engine(budget=2 << 30) as eng:
        mid = eng.add(case)
        eng.step(nsteps + 2)  # the launch after the last step takes its gauge sample
        eng.sync()
        assert eng.steps_done(mid) == nsteps
        got = eng.read(mid)
    for k in ("z", "m", "n", "zmax"):
        _check(got[k], ref[k], "engine " + k)
    assert np.array_equal(got["arrival"], ref["arrival"])
    _check(got["ts"], ots, "engine gauges")

    for fusion in (True, False):
        s = ReferenceSession(case, fusion=fusion, arrival=True)
        try:
            ts = _interp(s.drive(nsteps, maxamp=True), case.gauges)
            z, (m, n), zmax, arr = s.getz(1), s.getmn(1), s.getzmax(1), s.getarrival(1)
        finally:
            s.close()
        tag = "abi fused " if fusion else "abi per-phase "
        for a, b, k in ((z, ref["z"], "z"), (m, ref["m"], "m"), (n, ref["n"], "n"), (zmax, ref["zmax"], "zmax")):
            _check(a, b, tag + k)
        assert np.array_equal(arr, ref["arrival"]), tag + "arrival"
        H = case.root.H
        assert np.array_equal(z + H > 1e-5, ref["z"] + H > 1e-5), tag + "wet mask"
        _check(ts, ots, tag + "gauges")


def test_c1_drive_two_steps_per_launch(oracle_mod):
    """gcomcot_drive's two-step path (a lone linear spherical layer, fused,
    max-eta on, arrival off): a run of odd length that crosses the 1024-step
    stencil history twice ends with one single step; fields, max-eta and the
    raw gauge stencils against the oracle and against the per-phase path, bit
    for bit"""
    nsteps = 2051
    case = synth.config_c1(nsteps=nsteps)
    case.gauges = synth.wet_gauges(case.root, 8, np.random.default_rng(12))
    o = oracle_mod.OracleRun(case)
    ots = o.run(nsteps, threads=THREADS, arrival=False)
    ref = o.layer(0)
    got = {}
    for fusion in (True, False):
        s = ReferenceSession(case, fusion=fusion, arrival=False)
        try:
            st = s.drive(nsteps, maxamp=True)
            got[fusion] = (st, s.getz(1), s.getmn(1), s.getzmax(1))
        finally:
            s.close()
    st, z, (m, n), zmax = got[True]
    for a, b, k in ((z, ref["z"], "z"), (m, ref["m"], "m"), (n, ref["n"], "n"), (zmax, ref["zmax"], "zmax")):
        _check(a, b, "drive pairs " + k)
    _check(_interp(st, case.gauges), ots, "drive pairs gauges")
    assert np.array_equal(st.view(np.uint32), got[False][0].view(np.uint32))


@pytest.mark.parametrize("nsteps", [2, 3, 4, 40])
def test_drive_two_steps_short_runs(nsteps):
    """short gcomcot_drive runs on the two-step path: one history chunk that
    ends on a launch's second step (even lengths) or on a single step (odd);
    the raw gauge stencils and the fields equal the per-phase path's bit for
    bit"""
    case = synth.config_c1(nsteps=nsteps)
    case.gauges = synth.wet_gauges(case.root, 8, np.random.default_rng(13))
    got = {}
    for fusion in (True, False):
        s = ReferenceSession(case, fusion=fusion, arrival=False)
        try:
            st = s.drive(nsteps, maxamp=True)
            got[fusion] = (st, s.getz(1), *s.getmn(1), s.getzmax(1))
        finally:
            s.close()
    assert got[True][0].shape[0] == nsteps
    for a, b in zip(got[True], got[False]):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_c3_nested_600_steps_engine_and_reference_abi(oracle_mod):
    nsteps = 600
    case = synth.config_c3(nsteps=nsteps)
    # a 0.5 m hump in the child's own initial surface (wet cells): CONMASS,
    # CONMOME's wet/dry front and the JNZ feedback work from the first step
    Cl = case.layers[1]
    jj, ii = np.mgrid[0:Cl.ny, 0:Cl.nx]
    hump = 0.5 * np.exp(-((ii - Cl.nx / 2.0) ** 2 + (jj - Cl.ny / 2.0) ** 2) / (2.0 * 60.0 ** 2))
    Cl.Z0 = np.where(Cl.H > 0.0, Cl.Z0 + hump, 0.0).astype(np.float32)
    o = oracle_mod.OracleRun(case)
    o.run(nsteps, threads=THREADS)
    ref, rc = o.layer(0), o.layer(1)
    assert np.abs(rc["m"]).max() > 0

    with Engine(budget=8 << 30) as eng:
        mid = eng.add(case)
        eng.step(nsteps + 2)
        eng.sync()
        assert eng.steps_done(mid) == nsteps
        got = eng.read(mid)
    for k in ("z", "m", "n", "zmax"):
        _check(got[k], ref[k], "engine " + k)
    assert np.array_equal(got["arrival"], ref["arrival"])
    for k in ("z", "m", "n"):
        _check(got["child_" + k], rc[k], "engine child " + k)
    Hc = Cl.H
    # the child's wet/dry state: total depth above GX, exactly as the oracle has it
    assert np.array_equal(got["child_z"] + Hc > 1e-5, rc["z"] + Hc > 1e-5)

    s = ReferenceSession(case, fusion=True, arrival=True)
    try:
        s.drive(nsteps, maxamp=True)
        z, (m, n), zmax = s.getz(1), s.getmn(1), s.getzmax(1)
        zc, (mc, nc) = s.getz(2), s.getmn(2)
        arr = s.getarrival(1)
    finally:
        s.close()
    for a, b, k in ((z, ref["z"], "z"), (m, ref["m"], "m"), (n, ref["n"], "n"), (zmax, ref["zmax"], "zmax"),
                    (zc, rc["z"], "child z"), (mc, rc["m"], "child m"), (nc, rc["n"], "child n")):
        _check(a, b, "abi " + k)
    assert np.array_equal(arr, ref["arrival"])
