"""Parity at the full workload sizes: the 2401x2001 single grid (through the
engine and through the reference C ABI), the 1201x1001 + 601x501 nested pair
and two members of the 1201x1001 ensemble grid sharing one bathymetry, each
bitwise against the FP32 oracle.  The oracle runs these few dozen steps in
seconds on the host.  Humps placed on the open boundary, in a corner and
against the land strip make the edge tiles, OPEN and the shallow-cell clamp
work from the first step."""
import numpy as np
import pytest

from comcot_b200 import synth
from comcot_b200.abi import ReferenceSession
from comcot_b200.engine import Engine

pytestmark = pytest.mark.gpu


def _with_edge_humps(L, nsteps_unused=None):
    """adds 0.5 m Gaussian humps at the west and south boundaries, the
    south-west corner and 30 cells off the land strip, on wet cells"""
    z0 = L.Z0.astype(np.float64).copy()
    land = np.where((L.H <= 0.0).all(axis=0))[0]
    i_shore = (int(land.min()) if land.size else L.nx) - 30
    for (i, j) in ((0, L.ny // 2), (L.nx // 2, 0), (2, 2), (i_shore, L.ny // 3)):
        z0 += synth.gaussian_hump(L.x, L.y, float(L.x[i]), float(L.y[j]), 0.5, 25.0)
    z0[L.H <= 0.0] = 0.0
    L.Z0 = z0.astype(np.float32)


def _bits_equal(a, b, what):
    assert a.shape == b.shape, what
    bad = np.flatnonzero(a.view(np.uint32) != b.view(np.uint32))
    assert bad.size == 0, f"{what}: {bad.size} cells differ, first at flat index {bad[0]}"


def test_c2_full_size_engine_and_reference_abi(oracle_mod):
    nsteps = 40
    case = synth.config_c2(nsteps=nsteps)
    _with_edge_humps(case.root)
    o = oracle_mod.OracleRun(case)
    ots = o.run(nsteps)
    ref = o.layer(0)
    with Engine(budget=8 << 30) as eng:
        mid = eng.add(case)
        eng.step(nsteps + 2)  # the step after the last takes its gauge sample
        eng.sync()
        assert eng.done(mid)
        got = eng.read(mid)
    for k in ("z", "m", "n", "zmax"):
        _bits_equal(got[k], ref[k], "engine " + k)
    assert np.array_equal(got["arrival"], ref["arrival"])
    _bits_equal(got["ts"], ots, "engine gauges")
    assert (ref["arrival"] >= 0).sum() > 1000
    # the reference ABI's fused path on the same case
    s = ReferenceSession(case, fusion=True, arrival=True)
    try:
        for _ in range(nsteps):
            s.step(maxamp=True)
        z, (m, n), zmax, arr = s.getz(1), s.getmn(1), s.getzmax(1), s.getarrival(1)
    finally:
        s.close()
    for a, b, what in ((z, ref["z"], "abi z"), (m, ref["m"], "abi m"), (n, ref["n"], "abi n"),
                       (zmax, ref["zmax"], "abi zmax")):
        _bits_equal(a, b, what)
    assert np.array_equal(arr, ref["arrival"])


def test_c3_full_size_nested(oracle_mod):
    nsteps = 20
    case = synth.config_c3(nsteps=nsteps)
    # a 0.5 m hump in the child's own initial surface (wet cells), so its
    # CONMASS / CONMOME and the JNZ feedback work from the first step
    Cl = case.layers[1]
    jj, ii = np.mgrid[0:Cl.ny, 0:Cl.nx]
    hump = 0.5 * np.exp(-((ii - Cl.nx / 2.0) ** 2 + (jj - Cl.ny / 2.0) ** 2) / (2.0 * 60.0 ** 2))
    Cl.Z0 = np.where(Cl.H > 0.0, Cl.Z0 + hump, 0.0).astype(np.float32)
    with Engine(budget=8 << 30) as eng:
        mid = eng.add(case)
        eng.step(nsteps + 2)
        eng.sync()
        assert eng.done(mid)
        got = eng.read(mid)
    o = oracle_mod.OracleRun(case)
    o.run(nsteps)
    ref, rc = o.layer(0), o.layer(1)
    assert np.abs(rc["m"]).max() > 0
    for k in ("z", "m", "n", "zmax"):
        _bits_equal(got[k], ref[k], k)
    for k in ("z", "m", "n"):
        _bits_equal(got["child_" + k], rc[k], "child " + k)


def test_c4_full_size_members_share_bathymetry(oracle_mod):
    nsteps = 20
    L = synth.config_c4_grid()
    srcs = synth.ensemble_sources(L.x, L.y, 2, seed=40)
    cases = []
    for z in srcs:
        Lm = synth.LayerSpec(**{**L.__dict__, "Z0": np.ascontiguousarray(z, dtype=np.float32)})
        cases.append(synth.Case("C4", [Lm], nsteps))
    with Engine(budget=8 << 30) as eng:
        cls = eng.add_class(L)
        ids = [eng.add(c, cls=cls, arrival_thr=0.05) for c in cases]
        eng.step(nsteps + 2)
        eng.sync()
        got = [eng.read(i) for i in ids]
    for g, c in zip(got, cases):
        o = oracle_mod.OracleRun(c)
        o.run(nsteps)
        ref = o.layer(0)
        for k in ("z", "m", "n", "zmax"):
            _bits_equal(g[k], ref[k], k)
        assert np.array_equal(g["arrival"], ref["arrival"])
