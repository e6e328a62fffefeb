"""Seeded synthetic inputs for the benchmark configurations.

The reference's sample deck needs a bathymetry file it does not ship and no
public dataset is named for these configurations, so seeded generators with
the configurations' shapes and value ranges stand in for real data:

* bathymetry: abyssal plain, Gaussian seamounts that shoal it, a linear
  shelf on the east side and a land strip (negative depth) at the east edge;
* sources: a Gaussian hump or an elliptical uplift/subsidence dipole;
* nested child: a Cartesian shelf window whose depth runs from -20 m (land)
  to 200 m with smooth random slopes, and whose parent cells carry the block
  mean of the child depth;
* gauges: seeded wet interior points.

Arrays are [ny, nx] row-major, which is the Fortran NX x NY column-major layout.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import precompute as pc

F32 = np.float32
KM_PER_DEG_LAT = 110.57


@dataclass
class LayerSpec:
    id: int
    parent: int
    level: int
    nx: int
    ny: int
    H: np.ndarray
    Z0: np.ndarray
    x: np.ndarray
    y: np.ndarray
    dt: float
    dx: float                # arc-minutes (spherical) or metres (Cartesian)
    dy: float
    laycord: int = 0
    laygov: int = 0
    rel_size: int = 1
    rel_time: int = 1
    corners: list = field(default_factory=lambda: [1, 1, 1, 1])
    coefs: pc.Coefs | None = None
    rx: float = 0.0
    ry: float = 0.0
    grx: float = 0.0
    gry: float = 0.0
    fric_switch: int = 1
    fric_coef: float = 0.0
    linchk: int = 1
    modscm: int = 1
    hp: np.ndarray | None = None
    hq: np.ndarray | None = None
    sponge: tuple | None = None  # (COEFX, COEFY) [ny, nx] of SPONGE_COEF, outer layer only
    sc: "ScSpec | None" = None  # SC_OPTION = 1 coupling tables of a Cartesian child of a spherical parent


@dataclass
class ScSpec:
    pos: np.ndarray      # [ny, nx, 2] int32, 1-based (KI, KJ) in the parent
    cxy: np.ndarray      # [ny, nx, 4] float32 bilinear weights
    fix_top: bool = False


@dataclass
class Case:
    name: str
    layers: list
    nsteps: int
    gauges: list = field(default_factory=list)   # (layer_id, KI, KJ, CX, CY)
    arrival_thr: float = 0.05

    @property
    def root(self) -> LayerSpec:
        return self.layers[0]

    def cells_per_step(self) -> int:
        n = 0
        for L in self.layers:
            mult = 1
            p = L
            while p.parent != -1:
                mult *= p.rel_time
                p = next(q for q in self.layers if q.id == p.parent)
            n += L.nx * L.ny * mult
        return n


def _dist_km(x, y, lon_c, lat_c):
    dxk = (x[None, :] - lon_c) * 111.32 * math.cos(math.radians(lat_c))
    dyk = (y[:, None] - lat_c) * KM_PER_DEG_LAT
    return dxk, dyk


def bathymetry(x, y, rng, depth=4000.0, n_seamounts=20, shelf_cols=40, land_cols=10,
               shelf_depth=50.0):
    nx, ny = len(x), len(y)
    h = np.full((ny, nx), depth, dtype=np.float64)
    dlon = float(x[1] - x[0])
    dlat = float(y[1] - y[0])
    for _ in range(n_seamounts):
        lon_c = rng.uniform(x[0], x[-1])
        lat_c = rng.uniform(y[0], y[-1])
        amp = rng.uniform(500.0, 2000.0)
        rad = rng.uniform(20.0, 80.0)
        # evaluate inside +-5 radii only (the Gaussian is < 4e-6 of amp beyond)
        wy = int(5.0 * rad / KM_PER_DEG_LAT / dlat) + 2
        wx = int(5.0 * rad / (111.32 * max(math.cos(math.radians(lat_c)), 0.05)) / dlon) + 2
        ic = int((lon_c - x[0]) / dlon)
        jc = int((lat_c - y[0]) / dlat)
        i0, i1 = max(0, ic - wx), min(nx, ic + wx + 1)
        j0, j1 = max(0, jc - wy), min(ny, jc + wy + 1)
        dxk, dyk = _dist_km(x[i0:i1], y[j0:j1], lon_c, lat_c)
        h[j0:j1, i0:i1] -= amp * np.exp(-(dxk ** 2 + dyk ** 2) / (2.0 * rad ** 2))
    h = np.maximum(h, 200.0)
    if shelf_cols > 0:
        i0 = nx - land_cols - shelf_cols
        for k in range(shelf_cols):
            w = (k + 1) / shelf_cols
            col = i0 + k
            h[:, col] = (1.0 - w) * h[:, col] + w * shelf_depth
    if land_cols > 0:
        ramp = np.linspace(-5.0, -200.0, land_cols)
        h[:, nx - land_cols:] = ramp[None, :]
    return h.astype(np.float32)


def gaussian_hump(x, y, lon_c, lat_c, amp=1.0, radius_km=50.0):
    dxk, dyk = _dist_km(x, y, lon_c, lat_c)
    return (amp * np.exp(-(dxk ** 2 + dyk ** 2) / (2.0 * radius_km ** 2))).astype(np.float32)


def dipole(x, y, lon_c, lat_c, amp, strike_deg, offset_km=40.0, a_km=150.0, b_km=50.0):
    dxk, dyk = _dist_km(x, y, lon_c, lat_c)
    th = math.radians(strike_deg)
    along = dxk * math.sin(th) + dyk * math.cos(th)
    across = dxk * math.cos(th) - dyk * math.sin(th)

    def lobe(shift):
        return np.exp(-((along / a_km) ** 2 + ((across - shift) / b_km) ** 2))

    z = amp * lobe(-0.5 * offset_km) - 0.5 * amp * lobe(0.5 * offset_km)
    return z.astype(np.float32)


def spherical_layer(lid, x, y, H, Z0, dt, dx_min, parent=-1, level=1, laygov=0):
    ny, nx = H.shape
    coefs = pc.para(H, y, dx_min, dt, laygov=laygov)
    rx = dt / dx_min
    L = LayerSpec(id=lid, parent=parent, level=level, nx=nx, ny=ny, H=H, Z0=Z0, x=x, y=y, dt=dt,
                  dx=dx_min, dy=dx_min, laycord=0, laygov=laygov, coefs=coefs, rx=rx, ry=rx,
                  grx=9.807 * rx, gry=9.807 * rx, modscm=0 if parent == -1 else 1)
    L.hp, L.hq = pc.pq_depth(H)
    return L


def wet_gauges(L: LayerSpec, n, rng, first=1, margin=5):
    out = []
    tries = 0
    while len(out) < n and tries < 100000:
        tries += 1
        i = int(rng.integers(margin, L.nx - margin))
        j = int(rng.integers(margin, L.ny - margin))
        if L.H[j, i] <= 10.0:
            continue
        x0 = float(L.x[i] + (L.x[i + 1] - L.x[i]) * rng.uniform(0.1, 0.9))
        y0 = float(L.y[j] + (L.y[j + 1] - L.y[j]) * rng.uniform(0.1, 0.9))
        ki, kj, cx, cy = pc.locate_gauge(L.x, L.y, x0, y0, first=first)
        out.append((L.id, ki, kj, float(cx), float(cy)))
    return out


def single_layer_case(name, nx, ny, dx_min, dt, nsteps, seed, n_seamounts, shelf_cols, land_cols,
                      source="hump", ngauges=0, lon0=140.0, lat0=20.0, amp=None, laygov=0, fric=0.025):
    """One spherical layer: linear (laygov 0), nonlinear with Manning
    friction (laygov 1, CONMASS_S / CONMOME_S), or the dispersion-corrected
    forms (laygov 2 and 3, MASS_S_D / MOMT_S_D)."""
    rng = np.random.default_rng(seed)
    x, y = pc.axes(lon0, lat0, nx, ny, dx_min)
    H = bathymetry(x, y, rng, n_seamounts=n_seamounts, shelf_cols=shelf_cols, land_cols=land_cols)
    lon_c = float(rng.uniform(x[nx // 4], x[nx // 2]))
    lat_c = float(rng.uniform(y[ny // 4], y[3 * ny // 4]))
    if source == "hump":
        Z0 = gaussian_hump(x, y, lon_c, lat_c, 1.0 if amp is None else amp, 50.0)
    else:
        a = float(rng.uniform(0.5, 5.0)) if amp is None else amp
        Z0 = dipole(x, y, lon_c, lat_c, a, float(rng.uniform(0.0, 360.0)))
    L = spherical_layer(1, x, y, H, Z0, dt, dx_min, laygov=laygov)
    if laygov == 1:
        L.fric_switch, L.fric_coef, L.linchk = 0, fric, 1
    if laygov % 2 == 1:
        L.modscm = 1   # comcot.f90:602
    case = Case(name, [L], nsteps)
    if ngauges:
        case.gauges = wet_gauges(L, ngauges, rng)
    return case


def config_c1(nsteps=3600):
    """361x301 at 2', hump source, dt 2 s, OPEN on four sides."""
    return single_layer_case("C1", 361, 301, 2.0, 2.0, nsteps, seed=1, n_seamounts=20, shelf_cols=40,
                             land_cols=10, source="hump")


def config_c2(nsteps=7200, ngauges=32):
    """2401x2001 at 1', 200 seamounts, 2% land, dipole, dt 1 s, max-eta, gauges."""
    land = int(round(0.02 * 2401))
    return single_layer_case("C2", 2401, 2001, 1.0, 1.0, nsteps, seed=2, n_seamounts=200,
                             shelf_cols=80, land_cols=land, source="dipole", ngauges=ngauges)


def nested_case(name, pnx, pny, dx_min, dt, corners, rel_size, nsteps, seed, rel_time=None,
                n_seamounts=40, fric=0.025, lon0=140.0, lat0=20.0, child_laygov=1, ngauges=0, child_laycord=1):
    """Linear spherical parent with one child over an east-side shelf window:
    Cartesian (nonlinear by default, linear with child_laygov=0) or, with
    child_laycord=0, linear spherical (the reference GPU path's only kind)."""
    rng = np.random.default_rng(seed)
    x, y = pc.axes(lon0, lat0, pnx, pny, dx_min)
    is_, ie, js, je = corners
    cnx = (ie - is_ + 1) * rel_size + 1
    cny = (je - js + 1) * rel_size + 1
    # child depth: smooth random field between -20 and 200 m, deepening westward
    cx_ = np.linspace(0.0, 1.0, cnx)[None, :]
    cy_ = np.linspace(0.0, 1.0, cny)[:, None]
    base = 200.0 - 220.0 * cx_ ** 1.5
    wav = np.zeros((cny, cnx))
    for _ in range(6):
        kx, ky = rng.uniform(1.0, 4.0, size=2)
        ph = rng.uniform(0, 2 * math.pi, size=2)
        wav += np.sin(2 * math.pi * kx * cx_ + ph[0]) * np.cos(2 * math.pi * ky * cy_ + ph[1])
    Hc = np.clip(base + 15.0 * wav, -20.0, 200.0).astype(np.float32)
    # parent: deep basin, shelf ramp toward the child window, block means inside it
    H = bathymetry(x, y, rng, n_seamounts=n_seamounts, shelf_cols=0, land_cols=0)
    i_lo = is_ - 1
    for i in range(pnx):
        if i >= i_lo - 60:
            w = min(1.0, (i - (i_lo - 60)) / 60.0)
            H[:, i] = ((1 - w) * H[:, i] + w * 200.0).astype(np.float32)
    for jb in range(je - js + 1):
        for ib in range(ie - is_ + 1):
            blk = Hc[1 + jb * rel_size:1 + (jb + 1) * rel_size, 1 + ib * rel_size:1 + (ib + 1) * rel_size]
            H[js - 1 + jb, is_ - 1 + ib] = F32(blk.mean())
    east = ie + 1
    H[:, east - 1:] = np.minimum(H[:, east - 1:], F32(-10.0))
    lon_c = float(x[max(5, i_lo - 150)])
    lat_c = float(y[(js + je) // 2])
    Z0 = dipole(x, y, lon_c, lat_c, 2.0, float(rng.uniform(0, 360)))
    P = spherical_layer(1, x, y, H, Z0, dt, dx_min)
    # child geometry (Cartesian, metres)
    dxm, dym = pc.child_cartesian_spacing(y, corners, rel_size, dx_min)
    xs = 0.5 * (x[is_ - 1] + x[is_ - 2]) - (dx_min / 60.0 / rel_size) / 2.0
    ys = 0.5 * (y[js - 1] + y[js - 2]) - (dx_min / 60.0 / rel_size) / 2.0
    cxd = (xs + np.arange(cnx) * dx_min / 60.0 / rel_size).astype(np.float32)
    cyd = (ys + np.arange(cny) * dx_min / 60.0 / rel_size).astype(np.float32)
    rt, dtc = pc.rel_time(dt, dxm, dym, float(Hc.max()), nonlinear=(child_laygov == 1))
    if rel_time is not None:
        rt, dtc = rel_time, float(F32(dt) / F32(rel_time))
    Zc = dipole(cxd, cyd, lon_c, lat_c, 2.0, 0.0) * 0.0
    if child_laycord == 0:
        sx, sy = pc.child_axes_spherical(x, y, corners, rel_size, dx_min)
        rt, dtc = pc.rel_time(dt, dxm, dym, float(Hc.max()), nonlinear=(child_laygov == 1))
        if rel_time is not None:
            rt, dtc = rel_time, float(F32(dt) / F32(rel_time))
        C = spherical_layer(2, sx, sy, Hc, np.zeros_like(Hc), dtc, dx_min / rel_size, parent=1, level=2,
                            laygov=child_laygov)
        C.rel_size, C.rel_time, C.corners = rel_size, rt, list(corners)
        if child_laygov == 1:
            C.fric_switch, C.fric_coef, C.linchk = 0, fric, 1
        case = Case(name, [P, C], nsteps)
        if ngauges:
            case.gauges = wet_gauges(P, ngauges, rng)
        return case
    rx, ry = F32(dtc) / F32(dxm), F32(dtc) / F32(dym)
    C = LayerSpec(id=2, parent=1, level=2, nx=cnx, ny=cny, H=Hc, Z0=Zc.astype(np.float32), x=cxd, y=cyd,
                  dt=dtc, dx=dxm, dy=dym, laycord=1, laygov=child_laygov, rel_size=rel_size, rel_time=rt,
                  corners=list(corners), rx=float(rx), ry=float(ry), grx=float(F32(9.807) * rx),
                  gry=float(F32(9.807) * ry), fric_switch=0, fric_coef=fric, linchk=1, modscm=1)
    C.hp, C.hq = pc.pq_depth(Hc)
    case = Case(name, [P, C], nsteps)
    if ngauges:
        case.gauges = wet_gauges(P, ngauges, rng)
    return case


def nested_sc_case(name, pnx, pny, dx_min, dt, corners, rel_size, nsteps, seed, rel_time=None, child_laygov=1,
                   fix_top=False, **kw):
    """nested_case's spherical parent with a Cartesian child coupled by
    SC_OPTION = 1: the child's axes are UTM eastings / northings of its
    window's corners and every child node carries its parent cell and
    bilinear weights (SUBGRID_MATCHING, initialization.f90:996-1123)"""
    case = nested_case(name, pnx, pny, dx_min, dt, corners, rel_size, nsteps, seed, rel_time=rel_time,
                       child_laygov=child_laygov, **kw)
    P, C = case.layers
    g = pc.sc_child_geometry(P.x, P.y, corners, rel_size, dx_min)
    assert (C.ny, C.nx) == g.pos.shape[:2]
    C.x, C.y = g.x.astype(np.float32), g.y.astype(np.float32)
    C.dx, C.dy = g.dx, g.dy
    C.corners = list(g.corners)
    rx, ry = F32(C.dt) / F32(g.dx), F32(C.dt) / F32(g.dy)
    C.rx, C.ry = float(rx), float(ry)
    C.grx, C.gry = float(F32(9.807) * rx), float(F32(9.807) * ry)
    C.sc = ScSpec(pos=g.pos, cxy=g.cxy, fix_top=fix_top)
    return case


def config_c3(nsteps=3600, rel_time=None):
    """1201x1001 2' linear spherical parent, 601x501 nonlinear Cartesian child, r=5."""
    is_ = 1201 - 10 - 120 + 1 - 20
    js = 450
    corners = [is_, is_ + 119, js, js + 99]
    return nested_case("C3", 1201, 1001, 2.0, 2.0, corners, 5, nsteps, seed=3, rel_time=rel_time)


def ensemble_sources(x, y, nscen, seed, zone_km=300.0):
    """C4: seeded dipoles (amplitude U(0.5,5) m, strike U(0,360)) centred in a
    300 km fault zone."""
    rng = np.random.default_rng(seed)
    lon0 = float(x[len(x) // 3])
    lat0 = float(y[len(y) // 2])
    out = []
    for _ in range(nscen):
        dxk = rng.uniform(-zone_km / 2, zone_km / 2)
        dyk = rng.uniform(-zone_km / 2, zone_km / 2)
        lon_c = lon0 + dxk / (111.32 * math.cos(math.radians(lat0)))
        lat_c = lat0 + dyk / KM_PER_DEG_LAT
        out.append(dipole(x, y, lon_c, lat_c, float(rng.uniform(0.5, 5.0)), float(rng.uniform(0, 360))))
    return out


def config_c4_grid(seed=4):
    """the C4 shared grid: 1201x1001 at 2', linear spherical, dt 2 s"""
    rng = np.random.default_rng(seed)
    x, y = pc.axes(140.0, 20.0, 1201, 1001, 2.0)
    H = bathymetry(x, y, rng, n_seamounts=60, shelf_cols=40, land_cols=10)
    L = spherical_layer(1, x, y, H, np.zeros_like(H), 2.0, 2.0)
    return L


def poisson_trace(n=400, rate=2.0, seed=5, sizes=((481, 401), (961, 801), (1921, 1601)),
                  nested_frac=0.3, dt=2.0):
    """C5 arrivals: (t_arrival_s, (nx, ny), nsteps, nested, seed)"""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for k in range(n):
        t += rng.exponential(1.0 / rate)
        sz = sizes[int(rng.integers(0, len(sizes)))]
        minutes = rng.uniform(30.0, 120.0)
        nsteps = int(round(minutes * 60.0 / dt))
        out.append((t, sz, nsteps, bool(rng.uniform() < nested_frac), int(rng.integers(0, 2 ** 31))))
    return out


C5_SIZES = ((481, 401), (961, 801), (1921, 1601))


def config_c5_templates(seed=50, sizes=C5_SIZES, dt=2.0):
    """C5 grid classes: per outer size, a 2' linear spherical grid with an
    east-side shelf and, under it, a 301x251 nonlinear Cartesian child at
    ratio 5 (60 x 50 outer cells); un-nested requests of that size use the
    outer grid alone."""
    out = {}
    for k, (nx, ny) in enumerate(sizes):
        is_ = nx - 90
        js = ny // 2 - 25
        t = nested_case(f"C5t{nx}", nx, ny, 2.0, dt, [is_, is_ + 59, js, js + 49], 5, 0, seed=seed + k,
                        n_seamounts=max(10, nx // 40))
        out[(nx, ny)] = t
    return out


def child_wet_gauges(Cl: LayerSpec, n, rng):
    out = []
    tries = 0
    while len(out) < n and tries < 100000:
        tries += 1
        i = int(rng.integers(3, Cl.nx - 3))
        j = int(rng.integers(3, Cl.ny - 3))
        if Cl.H[j, i] <= 5.0:
            continue
        x0 = float(Cl.x[i] + (Cl.x[i + 1] - Cl.x[i]) * rng.uniform(0.1, 0.9))
        y0 = float(Cl.y[j] + (Cl.y[j + 1] - Cl.y[j]) * rng.uniform(0.1, 0.9))
        ki, kj, cx, cy = pc.locate_gauge(Cl.x, Cl.y, x0, y0, first=2)
        out.append((Cl.id, ki, kj, float(cx), float(cy)))
    return out


def c5_request_case(templates, size, nsteps, nested, seed, ngauges=16, child_gauges=4):
    """one C5 forecast request: its own seeded dipole (amplitude U(0.5,5) m,
    strike U(0,360)) in the western half of the outer grid and 16 gauges
    (4 of them in the child when nested).  Layers are shared with the
    template; only Z0 and the gauges are the request's own."""
    t = templates[size]
    P = t.layers[0]
    rng = np.random.default_rng(seed)
    lon_c = float(rng.uniform(P.x[P.nx // 8], P.x[P.nx // 2]))
    lat_c = float(rng.uniform(P.y[P.ny // 4], P.y[3 * P.ny // 4]))
    z0 = dipole(P.x, P.y, lon_c, lat_c, float(rng.uniform(0.5, 5.0)), float(rng.uniform(0.0, 360.0)))
    Pr = LayerSpec(**{**P.__dict__, "Z0": z0})
    layers = [Pr] + (list(t.layers[1:]) if nested else [])
    case = Case(f"req{seed}", layers, nsteps)
    ng_child = child_gauges if nested else 0
    case.gauges = wet_gauges(P, ngauges - ng_child, rng) + (child_wet_gauges(t.layers[1], ng_child, rng)
                                                           if nested else [])
    return case
