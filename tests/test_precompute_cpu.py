"""Once-per-run set-up restatements against the oracle's REAL versions."""
import ctypes as C

import numpy as np

from comcot_b200 import precompute as pc
from comcot_b200 import synth


def test_pq_depth_bitwise(oracle_mod):
    lib = oracle_mod.load(np.float32)
    rng = np.random.default_rng(0)
    H = rng.uniform(-50, 4000, (37, 53)).astype(np.float32)
    H[rng.uniform(size=H.shape) < 0.2] = 0.0
    hp, hq = pc.pq_depth(H)
    ohp = np.zeros_like(H)
    ohq = np.zeros_like(H)
    lib.ocl_pq_depth(53, 37, H.ctypes.data, ohp.ctypes.data, ohq.ctypes.data)
    assert np.array_equal(hp, ohp) and np.array_equal(hq, ohq)


def test_para_close_to_real_restatement_and_factorable(oracle_mod):
    lib = oracle_mod.load(np.float32)
    case = synth.single_layer_case("p", 41, 33, 2.0, 2.0, 0, seed=4, n_seamounts=2, shelf_cols=4, land_cols=2)
    L = case.root
    c = L.coefs
    ny, nx = L.H.shape
    lat = L.y.astype(np.float64)
    dely = np.full(ny, 2.0)
    out = {k: np.zeros(ny, np.float32) for k in ("r1", "r11", "r3", "r5", "r6")}
    r2 = np.zeros((ny, nx), np.float32)
    r4 = np.zeros((ny, nx), np.float32)
    lib.ocl_para(nx, ny, 0, 2.0, 2.0, lat.ctypes.data, dely.ctypes.data, L.hp.ctypes.data, L.hq.ctypes.data,
                 out["r1"].ctypes.data, out["r11"].ctypes.data, r2.ctypes.data, out["r3"].ctypes.data,
                 r4.ctypes.data, out["r5"].ctypes.data, out["r6"].ctypes.data)
    for k in out:
        assert np.allclose(getattr(c, k), out[k], rtol=2e-6, atol=0), k
    assert np.allclose(c.r2, r2, rtol=2e-6) and np.allclose(c.r4, r4, rtol=2e-6)
    # the FP32 R2 field is exactly CX(J) * max(HP,0): the device may rebuild it
    assert np.array_equal(c.r2, (c.cx[:, None] * np.maximum(L.hp, np.float32(0))).astype(np.float32))
    assert np.array_equal(c.r4, (c.cy[:, None] * np.maximum(L.hq, np.float32(0))).astype(np.float32))


def test_rel_time_rule_matches(oracle_mod):
    lib = oracle_mod.load(np.float32)
    for dtp, dx, dy, hmax, nl in ((2.0, 740.0, 741.0, 200.0, 1), (2.0, 150.0, 150.0, 200.0, 1),
                                  (1.0, 90.0, 95.0, 4000.0, 0), (4.0, 500.0, 500.0, 10.0, 0)):
        dtc = C.c_double()
        ir = lib.ocl_rel_time(dtp, dx, dy, hmax, nl, C.byref(dtc))
        ir2, dt2 = pc.rel_time(dtp, dx, dy, hmax, bool(nl))
        assert ir == ir2 and abs(dtc.value - dt2) < 1e-12


def test_corners_match(oracle_mod):
    lib = oracle_mod.load(np.float32)
    x, y = pc.axes(140.0, 20.0, 120, 100, 2.0)
    xs, xe, ys, ye = float(x[30]) + 0.01, float(x[60]) + 0.02, float(y[20]) + 0.01, float(y[50]) + 0.02
    c = np.zeros(4, np.int32)
    lib.ocl_corners(120, x.astype(np.float64).ctypes.data, 100, y.astype(np.float64).ctypes.data, xs, xe, ys, ye,
                    c.ctypes.data)
    assert list(c) == pc.corners(x, y, xs, xe, ys, ye)


def test_gauge_locate_weights():
    x, y = pc.axes(140.0, 20.0, 50, 40, 2.0)
    ki, kj, cx, cy = pc.locate_gauge(x, y, float(x[10]) + 0.25 * (x[11] - x[10]), float(y[7]) + 0.5 * (y[8] - y[7]))
    assert (ki, kj) == (11, 8)
    # REAL degree coordinates near 140 E carry ~1e-5 relative error (as in GET_TS)
    assert abs(cx - 0.25) < 1e-3 and abs(cy - 0.5) < 1e-3


def test_c3_geometry():
    case = synth.config_c3(nsteps=1)
    P, C_ = case.layers
    assert (P.nx, P.ny) == (1201, 1001) and (C_.nx, C_.ny) == (601, 501)
    assert C_.rel_size == 5 and C_.laycord == 1 and C_.laygov == 1
    assert C_.rel_time == 1  # 200 m shelf, CR 0.35
    assert C_.H.min() >= -20.0 - 1e-3 and C_.H.max() <= 200.0 + 1e-3


def test_sponge_coef_bitwise_and_separable(oracle_mod):
    """SPONGE_COEF + H_CALC (boundaries.f90:250-385) against the oracle's
    REAL restatement, on spherical and Cartesian axes"""
    for seed, (nx, ny) in enumerate([(97, 81), (160, 45), (33, 200)]):
        case = synth.single_layer_case("s", nx, ny, 2.0, 2.0, 0, seed=seed, n_seamounts=4, shelf_cols=8,
                                       land_cols=3)
        L = case.root
        for laycord, x, y in ((0, L.x, L.y), (1, np.arange(nx) * 20000.0, np.arange(ny) * 18000.0)):
            cx, cy = pc.sponge_coef(x, y, L.H, laycord)
            ox, oy = oracle_mod.sponge_coef(laycord, x, y, L.H)
            assert np.array_equal(cx.view(np.uint32), ox.view(np.uint32))
            assert np.array_equal(cy.view(np.uint32), oy.view(np.uint32))
            assert (cx == cx[:1, :]).all() and (cy == cy[:, :1]).all()
            if laycord == 0:
                # the band is converted to degrees but divided by metres: no damping at all
                assert not cx.any() and not cy.any()
            else:
                assert cx[:, 0] .max() > 0 and cy[0, :].max() > 0 and cx[:, nx // 2].max() == 0


def test_bc_wall_sides():
    H = np.full((10, 12), 100.0, np.float32)
    w = pc.bc_wall(H)
    assert (w[:, :2] == -999).all() and (w[:, -2:] == -999).all() and (w[:2, :] == -999).all()
    assert (w[-2:, :] == -999).all() and (w[2:-2, 2:-2] == 100).all()
    # a wave maker entering from side INCIDENT keeps that side open (boundaries.f90:395-419)
    for inc, open_view in ((1, lambda a: a[-2:, 2:-2]), (2, lambda a: a[:2, 2:-2]), (3, lambda a: a[2:-2, :2]),
                           (4, lambda a: a[2:-2, -2:])):
        w = pc.bc_wall(H, ini_switch=2, incident=inc)
        assert (open_view(w) == 100).all()
        assert (w == -999).sum() == H.size - 6 * 8 - open_view(w).size
    assert (pc.bc_wall(H, ini_switch=2, incident=5) == H).all()
    assert (H == 100).all()   # the input is not modified


def test_utm_round_trip_and_sc_tables():
    """SPH_TO_UTM / UTM_TO_SPH (initialization.f90:1390-1590) invert each
    other, and the SC_OPTION = 1 tables place every child node inside the
    parent cell they name, with weights summing to 1"""
    rng = np.random.default_rng(4)
    for _ in range(20):
        lon0 = float(rng.uniform(3.0, 357.0))
        lon = lon0 + rng.uniform(-2.5, 2.5, 50)
        lat = rng.uniform(-70.0, 70.0, 50)
        x, y = pc.sph_to_utm(lon, lat, lon0)
        lo, la = pc.utm_to_sph(x, y, lon0)
        assert np.abs(lo - lon).max() < 1e-6 and np.abs(la - lat).max() < 1e-6
    assert pc.utm_zone_meridian(140.2) == 141.0 and pc.utm_zone_meridian(-10.0) == 0.0
    xp, yp = pc.axes(140.0, 20.0, 97, 81, 2.0)
    g = pc.sc_child_geometry(xp, yp, [60, 79, 30, 49], 3, 2.0)
    assert g.pos.shape == (61, 61, 2) and (g.pos >= 2).all()
    lon, lat = pc.coord_convert_to_sph(*np.meshgrid(g.x, g.y), g.xs, g.ys)
    ki, kj = g.pos[..., 0] - 1, g.pos[..., 1] - 1
    assert (xp[ki] <= lon).all() and (lon < xp[ki + 1]).all()
    assert (yp[kj] <= lat).all() and (lat < yp[kj + 1]).all()
    assert np.abs(g.cxy.sum(-1) - 1.0).max() < 1e-6 and (g.cxy >= 0).all()
    assert g.corners == [int(g.pos[..., 0].min()), int(g.pos[..., 0].max()), int(g.pos[..., 1].min()),
                         int(g.pos[..., 1].max())]
