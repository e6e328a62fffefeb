"""The oracle's restatements of the dispersion forms, the sponge and the
SC_OPTION = 1 coupling against a second, independent numpy restatement,
bit for bit, on randomised states (test infrastructure checking test
infrastructure: neither is the product)."""
import ctypes as C

import numpy as np
import pytest

import numpy_restatement as nr
from comcot_b200 import precompute as pc
from comcot_b200 import synth

F = np.float32


def _fill(f, rng, keys, lo, hi):
    for k in keys:
        f[k][...] = rng.uniform(lo, hi, f[k].shape).astype(F)


@pytest.mark.parametrize("laygov", [2, 3])
def test_dispersion_spherical_outer_layer(oracle_mod, laygov):
    case = synth.single_layer_case("d", 53, 41, 2.0, 2.0, 0, seed=3, n_seamounts=3, shelf_cols=6, land_cols=3,
                                   laygov=laygov)
    o = oracle_mod.OracleRun(case)
    lib, f, L = o.lib, o.fields[0], case.root
    rng = np.random.default_rng(laygov)
    _fill(f, rng, ("z1", "z2"), -1.0, 1.0)
    _fill(f, rng, ("m1", "n1"), -50.0, 50.0)
    z1, m1, n1 = f["z1"].copy(), f["m1"].copy(), f["n1"].copy()
    lib.ocl_mass(C.byref(o.arr[0]))
    want = nr.mass_d(z1, m1, n1, f["h"], True, True, f["r1"], f["r11"], f["r6"])
    assert np.array_equal(f["z2"][1:-1, 1:-1].view(np.uint32), want[1:-1, 1:-1].view(np.uint32))
    z2 = f["z2"].copy()
    lib.ocl_moment(C.byref(o.arr[0]))
    wm, wn = nr.momt_s_d(z2, m1, n1, f["h"], f["r2"], f["r3"], f["r4"], f["r5"], L.modscm, True)
    assert np.array_equal(f["m2"][:, :-1].view(np.uint32), wm[:, :-1].view(np.uint32))
    assert np.array_equal(f["n2"][:-1, :].view(np.uint32), wn[:-1, :].view(np.uint32))


@pytest.mark.parametrize("modscm,fric", [(1, 0), (0, 0), (0, 1)])
def test_dispersion_cartesian_child(oracle_mod, modscm, fric):
    case = synth.nested_case("d", 97, 81, 2.0, 2.0, [60, 79, 30, 49], 3, 0, seed=5, rel_time=2, child_laygov=2)
    Cl = case.layers[1]
    Cl.modscm, Cl.fric_switch = modscm, fric
    o = oracle_mod.OracleRun(case)
    lib, f = o.lib, o.fields[1]
    rng = np.random.default_rng(7 + modscm)
    _fill(f, rng, ("z1", "z2"), -1.0, 1.0)
    _fill(f, rng, ("m1", "n1", "m2", "n2"), -20.0, 20.0)
    z1, m1, n1 = f["z1"].copy(), f["m1"].copy(), f["n1"].copy()
    m2_old, n2_old = f["m2"].copy(), f["n2"].copy()
    lib.ocl_mass(C.byref(o.arr[1]))
    want = nr.mass_d(z1, m1, n1, f["h"], False, False, rx=Cl.rx, ry=Cl.ry)
    assert np.array_equal(f["z2"][1:, 1:].view(np.uint32), want[1:, 1:].view(np.uint32))
    z2 = f["z2"].copy()
    lib.ocl_moment(C.byref(o.arr[1]))
    wm, wn = nr.momt_c_d(z2, m1, n1, f["h"], f["hp"], Cl.grx, Cl.gry, Cl.dt, Cl.fric_switch, Cl.fric_coef, modscm,
                         False, m2_old, n2_old, lib.ocl_powf)
    assert np.array_equal(f["m2"].view(np.uint32), wm.view(np.uint32))
    assert np.array_equal(f["n2"].view(np.uint32), wn.view(np.uint32))


def test_sponge(oracle_mod):
    case = synth.single_layer_case("s", 61, 47, 2.0, 2.0, 0, seed=2, n_seamounts=3, shelf_cols=6, land_cols=3)
    L = case.root
    L.sponge = pc.sponge_coef(np.arange(L.nx) * 20000.0, np.arange(L.ny) * 20000.0, L.H, 1)
    o = oracle_mod.OracleRun(case)
    lib, f = o.lib, o.fields[0]
    rng = np.random.default_rng(11)
    _fill(f, rng, ("m1", "n1", "m2", "n2"), -20.0, 20.0)
    m2, n2, m1, n1 = f["m2"].copy(), f["n2"].copy(), f["m1"].copy(), f["n1"].copy()
    lib.ocl_sponge(C.byref(o.arr[0]))
    wm, wn = nr.sponge(m2, n2, m1, n1, f["spx"], f["spy"], L.dt)
    assert np.array_equal(f["m2"].view(np.uint32), wm.view(np.uint32))
    assert np.array_equal(f["n2"].view(np.uint32), wn.view(np.uint32))


def _sc_state(oracle_mod, fix_top=False, rel_time=2, seed=0):
    case = synth.nested_sc_case("sc", 97, 81, 2.0, 2.0, [60, 79, 30, 49], 3, 0, seed=3, rel_time=rel_time,
                                fix_top=fix_top)
    o = oracle_mod.OracleRun(case)
    P, Cf = o.fields
    rng = np.random.default_rng(seed)
    _fill(P, rng, ("z2", "m1", "n1", "m2", "n2"), -5.0, 5.0)
    _fill(Cf, rng, ("z2", "m1", "n1"), -1.0, 1.0)
    return case, o, P, Cf


def test_sc_edges_first_substep(oracle_mod):
    case, o, P, Cf = _sc_state(oracle_mod, seed=1)
    sc = case.layers[1].sc
    want = nr.edge_sc(P["m1"], P["n1"], Cf["h"], Cf["z2"], Cf["m1"], Cf["n1"], sc.pos, sc.cxy)
    o.lib.ocl_edge_sc(C.byref(o.arr[0]), C.byref(o.arr[1]))
    assert np.array_equal(Cf["m1"].view(np.uint32), want[0].view(np.uint32))
    assert np.array_equal(Cf["n1"].view(np.uint32), want[1].view(np.uint32))


@pytest.mark.parametrize("fix_top,t", [(False, 2), (True, 3)])
def test_sc_newq_forecast_and_blend(oracle_mod, fix_top, t):
    case, o, P, Cf = _sc_state(oracle_mod, fix_top=fix_top, rel_time=3, seed=2 + t)
    Pl, Cl = case.layers
    sc = Cl.sc
    pm1, pn1, pz2 = P["m1"].copy(), P["n1"].copy(), P["z2"].copy()
    cm1, cn1 = Cf["m1"].copy(), Cf["n1"].copy()
    o.lib.ocl_newq_sc(C.byref(o.arr[0]), C.byref(o.arr[1]), t)
    # the band forecast of the parent's fluxes (all_grids.f90:1130-1266), restated here
    h, r2, r4, r3, r5 = P["h"], P["r2"], P["r4"], P["r3"], P["r5"]
    ny, nx = h.shape
    c0, c1, c2, c3 = Cl.corners
    pos = sc.pos

    def band_m(i0, i1, j0, j1):
        out = {}
        for j in range(j0, j1 + 1):
            for i in range(i0, i1 + 1):
                I, J = i - 1, j - 1
                if h[J, I] > nr.GX and h[J, I + 1] > nr.GX:
                    jm, jp = max(J - 1, 0), min(J + 1, ny - 1)
                    tot = pn1[J, I] + pn1[J, I + 1] + pn1[jm, I] + pn1[jm, I + 1]
                    xm = pm1[J, I] - r2[J, I] * (pz2[J, I + 1] - pz2[J, I]) + r3[J] * tot
                    if Pl.modscm == 0:
                        xm = xm - r2[J, I] * nr.TWLVTH * ((pz2[jp, I + 1] - F(2) * pz2[J, I + 1] + pz2[jm, I + 1])
                                                          - (pz2[jp, I] - F(2) * pz2[J, I] + pz2[jm, I]))
                    out[(J, I)] = F(0) if abs(xm) < nr.EPS else F(xm)
                else:
                    out[(J, I)] = F(0)
        return out

    def band_n(i0, i1, j0, j1):
        out = {}
        for j in range(j0, j1 + 1):
            for i in range(i0, i1 + 1):
                I, J = i - 1, j - 1
                if h[J, I] > nr.GX and h[J + 1, I] > nr.GX:
                    im, ip = max(I - 1, 0), min(I + 1, nx - 1)
                    tot = pm1[J, im] + pm1[J + 1, im] + pm1[J, I] + pm1[J + 1, I]
                    xn = pn1[J, I] - r4[J, I] * (pz2[J + 1, I] - pz2[J, I]) - r5[J] * tot
                    if Pl.modscm == 0:
                        xn = xn - r4[J, I] * nr.TWLVTH * ((pz2[J + 1, ip] - F(2) * pz2[J + 1, I] + pz2[J + 1, im])
                                                          - (pz2[J, ip] - F(2) * pz2[J, I] + pz2[J, im]))
                    out[(J, I)] = F(0) if abs(xn) < nr.EPS else F(xn)
                else:
                    out[(J, I)] = F(0)
        return out

    fm = {}
    for a, b in ((pos[0, 0, 0], pos[-1, 0, 0]), (pos[0, -1, 0], pos[-1, -1, 0])):
        fm.update(band_m(min(a, b) - 2, max(a, b) + 2, c2 - 2, c3 + 2))
    fn = {}
    for a, b in ((pos[-1, 0, 1], pos[-1, -1, 1]), (pos[0, 0, 1], pos[0, -1, 1])):
        fn.update(band_n(c0 - 2, c1 + 2, min(a, b) - 2, max(a, b) + 2))
    for (J, I), v in fm.items():
        assert P["m2"][J, I].view(np.uint32) == v.view(np.uint32)
    for (J, I), v in fn.items():
        assert P["n2"][J, I].view(np.uint32) == v.view(np.uint32)
    want = nr.newq_sc_blend(pm1, pn1, P["m2"], P["n2"], Cf["h"], Cf["z2"], cm1, cn1, sc.pos, sc.cxy, t, Cl.rel_time,
                            fix_top)
    assert np.array_equal(Cf["m1"].view(np.uint32), want[0].view(np.uint32))
    assert np.array_equal(Cf["n1"].view(np.uint32), want[1].view(np.uint32))


def test_sc_jnz(oracle_mod):
    case, o, P, Cf = _sc_state(oracle_mod, seed=9)
    Cl = case.layers[1]
    want = nr.jnz_sc(P["z2"], Cf["h"], Cf["z2"], Cl.sc.pos, Cl.corners, Cl.rel_size)
    o.lib.ocl_jnz_sc(C.byref(o.arr[0]), C.byref(o.arr[1]))
    assert np.array_equal(P["z2"].view(np.uint32), want.view(np.uint32))
