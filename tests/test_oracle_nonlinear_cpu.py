"""The oracle's CONMASS / CONMOME and CONMASS_S / CONMOME_S (with
WAVE_BREAKING) against a second restatement written cell by cell from the
Fortran (tests/nonlinear_restatement.py), bit for bit, on randomised child
states: mild ones and violent ones that reach the breaking damping and the
velocity limiter."""
import ctypes as C

import numpy as np
import pytest

import nonlinear_restatement as nl
from comcot_b200 import synth

F = np.float32


@pytest.mark.parametrize("sph", [False, True])
@pytest.mark.parametrize("scale,fric,modscm", [(3.0, 0, 1), (3000.0, 0, 1), (300.0, 1, 0)])
def test_nonlinear_child_step_bitwise(oracle_mod, sph, scale, fric, modscm):
    kw = {"child_laycord": 0} if sph else {}
    case = synth.nested_case("nl", 97, 81, 2.0, 2.0, [60, 79, 30, 49], 3, 0, seed=4, rel_time=2,
                             child_laygov=1, **kw)
    Cl = case.layers[1]
    Cl.fric_switch, Cl.modscm = fric, modscm
    o = oracle_mod.OracleRun(case)
    lib, f = o.lib, o.fields[1]
    rng = np.random.default_rng(int(scale) + 7 * fric + (1 if sph else 0))
    f["z1"][...] = rng.uniform(-0.5, 0.5, f["z1"].shape).astype(F)
    for k in ("m1", "n1", "m2", "n2"):
        f[k][...] = rng.uniform(-scale, scale, f[k].shape).astype(F)
    s = {"nx": Cl.nx, "ny": Cl.ny, "dt": Cl.dt, "fric_switch": fric, "fric_coef": Cl.fric_coef,
         "linchk": Cl.linchk, "modscm": modscm, "rx": Cl.rx, "ry": Cl.ry, "grx": Cl.grx, "gry": Cl.gry}
    for k in ("h", "hp", "hq", "z1", "m1", "n1", "m2", "n2", "z2", "dz2"):
        s[k] = f[k].copy()
    for k in ("r1", "r11", "r6", "r3", "r5", "r0", "r22"):
        s[k] = f[k].copy()
    s["cx"], s["cy"] = f["r2"][:, 0].copy(), f["r4"][:, 0].copy()

    lib.ocl_mass(C.byref(o.arr[1]))
    nl.conmass(s, sph, root=False)
    for k in ("z2", "dz2"):
        assert np.array_equal(f[k][1:, 1:].view(np.uint32), s[k][1:, 1:].view(np.uint32)), k
    # both sides continue from the same surface
    s["z2"][...] = f["z2"]
    s["dz2"][...] = f["dz2"]
    lib.ocl_moment(C.byref(o.arr[1]))
    nl.conmome(s, sph, False, lib.ocl_powf, lib.ocl_expf)
    for k in ("m2", "n2"):
        assert np.array_equal(f[k].view(np.uint32), s[k].view(np.uint32)), k
