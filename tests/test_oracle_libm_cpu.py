"""The float oracle's exp and pow (WAVE_BREAKING's EXP(-A*REF),
moment.f90:1323, and Manning's DF**(2.3333333), moment.f90:460,657) are the
deterministic functions of comcot_math.h, which the CUDA library also uses so
that both round alike.  Sharing them could hide an error in them.  This test
runs a second float build of the oracle whose exp and pow are the C library's
expf and powf (oracle/Makefile, OCL_LIBM) and checks that it agrees:
  - over 300 steps of the C3 nested pair (1201 x 1001 outer grid, 601 x 501
    nonlinear Cartesian child with Manning n = 0.025 and a 0.5 m hump in the
    child): the child's wet/dry mask is identical, eta, M and N within 1e-4
    of their maxima on both layers;
  - on violent child states that reach the breaking damping and the
    velocity limiter, one CONMASS + CONMOME step: fluxes within 1e-4 and the
    same zero pattern.
"""
import ctypes as C
import os

import numpy as np
import pytest

from comcot_b200 import synth

F = np.float32
TOL = 1e-4


def _rel(a, b):
    scale = max(float(np.abs(b).max()), 1e-30)
    return float(np.abs(a.astype(np.float64) - b.astype(np.float64)).max()) / scale


def test_c3_libm_build_agrees(oracle_mod):
    nsteps = 300
    case = synth.config_c3(nsteps=nsteps)
    Cl = case.layers[1]
    jj, ii = np.mgrid[0:Cl.ny, 0:Cl.nx]
    hump = 0.5 * np.exp(-((ii - Cl.nx / 2.0) ** 2 + (jj - Cl.ny / 2.0) ** 2) / (2.0 * 60.0 ** 2))
    Cl.Z0 = np.where(Cl.H > 0.0, Cl.Z0 + hump, 0.0).astype(F)
    runs = []
    for libm in (False, True):
        o = oracle_mod.OracleRun(case, libm=libm)
        o.run(nsteps, threads=os.cpu_count() or 1)
        runs.append((o.layer(0), o.layer(1)))
    (p0, c0), (p1, c1) = runs
    assert float(np.abs(c0["m"]).max()) > 0.0  # the child's fluxes (and its friction) are live
    H = Cl.H
    assert np.array_equal(c0["z"] + H > F(1e-5), c1["z"] + H > F(1e-5))
    for a, b, what in ((p1, p0, "outer"), (c1, c0, "child")):
        for k in ("z", "m", "n"):
            assert _rel(a[k], b[k]) <= TOL, f"{what} {k}"
    assert np.array_equal(p0["zmax"], p1["zmax"]) or _rel(p1["zmax"], p0["zmax"]) <= TOL
    assert np.array_equal(p0["arrival"], p1["arrival"])


@pytest.mark.parametrize("scale,fric", [(300.0, 0), (3000.0, 0)])
def test_violent_child_step_libm_build_agrees(oracle_mod, scale, fric):
    case = synth.nested_case("nl", 97, 81, 2.0, 2.0, [60, 79, 30, 49], 3, 0, seed=4, rel_time=2, child_laygov=1)
    Cl = case.layers[1]
    Cl.fric_switch = fric
    out = []
    for libm in (False, True):
        o = oracle_mod.OracleRun(case, libm=libm)
        f = o.fields[1]
        rng = np.random.default_rng(int(scale) + 3)
        f["z1"][...] = rng.uniform(-0.5, 0.5, f["z1"].shape).astype(F)
        for k in ("m1", "n1", "m2", "n2"):
            f[k][...] = rng.uniform(-scale, scale, f[k].shape).astype(F)
        o.lib.ocl_mass(C.byref(o.arr[1]))
        o.lib.ocl_moment(C.byref(o.arr[1]))
        out.append({k: f[k].copy() for k in ("z2", "dz2", "m2", "n2")})
    a, b = out
    assert np.array_equal(a["z2"].view(np.uint32), b["z2"].view(np.uint32))  # CONMASS has no exp/pow
    assert np.array_equal(a["dz2"] > 0, b["dz2"] > 0)
    for k in ("m2", "n2"):
        assert np.array_equal(a[k] == 0, b[k] == 0), k
        assert _rel(b[k], a[k]) <= TOL, k
