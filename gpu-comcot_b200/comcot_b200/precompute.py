"""Once-per-run set-up of a COMCOT layer: grid axes, still-water depth at the
flux points, spherical coefficients, sub-level time ratio, nesting corners
and gauge interpolation weights.

These restate the reference's initialisation routines:

* ``axes``          DX_CALC, normal spherical grid (initialization.f90:853-870)
* ``pq_depth``      PQ_DEPTH (initialization.f90:2501-2526)
* ``para``          PARA, LAYGOV 0/1 (comcot.f90:694-752)
* ``rel_time``      CR_CHECK sub-level rule (initialization.f90:1210-1237)
* ``corners``       SUBGRID_MATCHING corner search (initialization.f90:913-936)
* ``locate_gauge``  GET_TS index search and weights (output.f90:1054-1080)

PARA's trigonometry is evaluated in float64 and rounded once to float32 (the
reference evaluates it in REAL); R2 and R4 are then formed in float32 as
``CX(J) * max(HP,0)`` exactly like ``RS/COS_M/(DX*RAD_MIN)*AMAX1(HP,0)``, so
the per-row factor CX(J) reproduces every cell of R2 bit for bit.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

GRAV = np.float32(9.807)
GX = np.float32(1.0e-5)
EPS = np.float32(1.0e-10)
R_EARTH = 6378000.0
RAD_DEG = 0.01745329252
RAD_MIN = 0.000290888208665721
CORI_W = 7.2722e-5

F32 = np.float32


def axes(x_start: float, y_start: float, nx: int, ny: int, dx_min: float, dy_min: float | None = None):
    """Longitude/latitude axes in degrees of a normal spherical grid."""
    dy_min = dx_min if dy_min is None else dy_min
    dx = F32(dx_min) / F32(60.0)
    dy = F32(dy_min) / F32(60.0)
    x = (F32(x_start) + np.arange(nx, dtype=np.float32) * dx).astype(np.float32)
    y = (F32(y_start) + np.arange(ny, dtype=np.float32) * dy).astype(np.float32)
    return x, y


def pq_depth(h: np.ndarray):
    """HP, HQ [ny, nx] (row-major view of the column-major field)."""
    h = h.astype(np.float32)
    hp = np.zeros_like(h)
    hq = np.zeros_like(h)
    hip1 = np.concatenate([h[:, 1:], h[:, -1:]], axis=1)
    hjp1 = np.concatenate([h[1:, :], h[-1:, :]], axis=0)
    wet = h > GX
    hp[wet] = (F32(0.5) * (h + hip1))[wet]
    hq[wet] = (F32(0.5) * (h + hjp1))[wet]
    return hp, hq


@dataclass
class Coefs:
    r1: np.ndarray   # [ny] R1(1,J)
    r11: np.ndarray  # [ny]
    r6: np.ndarray   # [ny]
    r3: np.ndarray   # [ny]
    r5: np.ndarray   # [ny]
    cx: np.ndarray   # [ny]  R2 = CX * max(HP,0)
    cy: np.ndarray   # [ny]  R4 = CY * max(HQ,0)
    r2: np.ndarray = field(default=None)  # [ny, nx]
    r4: np.ndarray = field(default=None)
    r0: np.ndarray = field(default=None)  # [ny] RR/(DEL_Y*RAD_MIN), nonlinear advection (comcot.f90:727)
    r22: np.ndarray = field(default=None)  # [ny] RR/COS_N/(DX*RAD_MIN) (comcot.f90:733)

    def rows(self) -> np.ndarray:
        return np.stack([self.r1, self.r11, self.r6, self.r3, self.r5, self.cx, self.cy]).astype(np.float32)


def para(h: np.ndarray, lat: np.ndarray, dx_min: float, dt: float, del_y_min=None, laygov: int = 0) -> Coefs:
    ny, nx = h.shape
    lat = np.asarray(lat, dtype=np.float64)
    dely = np.full(ny, dx_min, dtype=np.float64) if del_y_min is None else np.asarray(del_y_min, np.float64)
    rr = dt / R_EARTH
    rs = 9.807 * rr
    rt = 0.5 * dt * CORI_W
    ang_m = lat * RAD_DEG
    ang_n = (lat + 0.5 * dely / 60.0) * RAD_DEG
    cos_m, cos_n = np.cos(ang_m), np.cos(ang_n)
    sin_m, sin_n = np.sin(ang_m), np.sin(ang_n)
    r1 = (rr / cos_m / (dx_min * RAD_MIN)).astype(np.float32)
    r11 = (rr / cos_m / (dely * RAD_MIN)).astype(np.float32)
    cx = (rs / cos_m / (dx_min * RAD_MIN)).astype(np.float32)
    cy = (rs / (dely * RAD_MIN)).astype(np.float32)
    r3 = (rt * sin_m).astype(np.float32)
    r5 = (rt * sin_n).astype(np.float32)
    r6 = cos_n.astype(np.float32)
    r0 = (rr / (dely * RAD_MIN)).astype(np.float32)
    r22 = (rr / cos_n / (dx_min * RAD_MIN)).astype(np.float32)
    hp, hq = pq_depth(h)
    if laygov in (0, 2):   # LAYGOV 3 and the nonlinear forms carry no depth factor (comcot.f90:733-747,776-795)
        r2 = (cx[:, None] * np.maximum(hp, F32(0))).astype(np.float32)
        r4 = (cy[:, None] * np.maximum(hq, F32(0))).astype(np.float32)
    else:
        r2 = np.repeat(cx[:, None], nx, axis=1).astype(np.float32)
        r4 = np.repeat(cy[:, None], nx, axis=1).astype(np.float32)
    return Coefs(r1, r11, r6, r3, r5, cx, cy, r2, r4, r0, r22)


def rel_time(dt_parent: float, dx_m: float, dy_m: float, hmax: float, nonlinear: bool):
    """(rel_time, dt_child) from the Courant rule with CR 0.5 (0.35 nonlinear)."""
    h_max = max(np.float32(hmax), GX)
    cr = F32(0.35) if nonlinear else F32(0.5)
    dt = cr * F32(min(dx_m, dy_m)) / np.sqrt(GRAV * F32(h_max))
    dtp = F32(dt_parent)
    if dt >= dtp:
        return 1, float(dtp)
    ir = int(math.floor(float(dtp / dt))) + 1
    return ir, float(dtp / F32(ir))


def corners(xp: np.ndarray, yp: np.ndarray, xs: float, xe: float, ys: float, ye: float):
    """[IS, IE, JS, JE] (1-based) of a child window inside the parent axes."""
    c = [1, 1, 1, 1]
    xp = xp.astype(np.float32)
    yp = yp.astype(np.float32)
    for k in range(2, len(xp)):
        lo = (xp[k - 2] + xp[k - 1]) / F32(2)
        hi = (xp[k - 1] + xp[k]) / F32(2)
        if lo <= F32(xs) < hi:
            c[0] = k + 1
        if lo <= F32(xe) < hi:
            c[1] = k - 1
    for k in range(2, len(yp)):
        lo = (yp[k - 2] + yp[k - 1]) / F32(2)
        hi = (yp[k - 1] + yp[k]) / F32(2)
        if lo <= F32(ys) < hi:
            c[2] = k + 1
        if lo <= F32(ye) < hi:
            c[3] = k - 1
    return c


def locate_gauge(x: np.ndarray, y: np.ndarray, x0: float, y0: float, first: int = 1):
    """(KI, KJ, CX, CY) with GET_TS's search (1-based; first=1 layer 1, 2 inner)."""
    nx, ny = len(x), len(y)
    x0, y0 = F32(x0), F32(y0)
    ki = kj = 0
    for i in range(first, nx):
        if x[i - 1] <= x0 < x[i]:
            ki = i
        if x0 < x[first - 1]:
            ki = first
        if x0 >= x[nx - 1]:
            ki = nx - 1
    for j in range(first, ny):
        if y[j - 1] <= y0 < y[j]:
            kj = j
        if y0 < y[first - 1]:
            kj = first
        if y0 >= y[ny - 1]:
            kj = ny - 1
    cx = (x0 - x[ki - 1]) / (x[ki] - x[ki - 1])
    cy = (y0 - y[kj - 1]) / (y[kj] - y[kj - 1])
    return ki, kj, F32(cx), F32(cy)


def child_axes_spherical(xp, yp, corners_, rel_size, dx_min_parent):
    """Child axes for a spherical child of a spherical parent (SUBGRID_MATCHING
    initialization.f90:970-1000), uniform DEL_Y."""
    is_, ie, js, je = corners_
    nx = (ie - is_ + 1) * rel_size + 1
    ny = (je - js + 1) * rel_size + 1
    dx = F32(dx_min_parent) / F32(rel_size) / F32(60.0)
    xs = F32(0.5) * (xp[is_ - 1] + xp[is_ - 2]) - dx / F32(2.0)
    ys = F32(0.5) * (yp[js - 1] + yp[js - 2]) - dx / F32(2.0)
    x = (np.arange(nx, dtype=np.float32) * dx + xs).astype(np.float32)
    y = (np.arange(ny, dtype=np.float32) * dx + ys).astype(np.float32)
    return x, y


def child_cartesian_spacing(yp, corners_, rel_size, dx_min_parent):
    """Metres per child cell of a Cartesian child in a spherical parent: the
    parent cell at the window's south edge divided by the ratio (the reference
    converts the window corners with its UTM routine, initialization.f90:1004-1050;
    this uses the local arc lengths, which agree to <0.1% inside a 1-degree window)."""
    is_, ie, js, je = corners_
    lat = float(0.5 * (yp[js - 1] + yp[js - 2]))
    dlon = dx_min_parent / 60.0 * RAD_DEG
    dx = R_EARTH * math.cos(lat * RAD_DEG) * dlon / rel_size
    dy = R_EARTH * dlon / rel_size
    return dx, dy


def h_mean(h: np.ndarray) -> np.float32:
    """H_CALC (boundaries.f90:351-385): mean of the wet depths (H > GX),
    accumulated in float with I outermost, as the Fortran loops run"""
    hw = np.ascontiguousarray(h, dtype=F32).T.ravel()   # I outer, J inner
    wet = hw[hw > F32(GX)]
    if wet.size == 0:
        return F32(0.0)
    s = np.cumsum(wet, dtype=F32)[-1]                   # sequential float additions
    return F32(s / F32(wet.size))


def sponge_coef(x: np.ndarray, y: np.ndarray, h: np.ndarray, laycord: int):
    """SPONGE_COEF (boundaries.f90:250-345), in float arithmetic: damping
    coefficients [ny, nx] for X and Y over a band of twice the characteristic
    wavelength (20 x mean wet depth) along the edges.  COEFX depends on I only
    and COEFY on J only.  On a spherical layer the band width is converted to
    degrees but the ramp is still divided by the width in metres, so every
    coefficient falls below EPS and is 0, as in the reference."""
    depth = h_mean(h)
    if depth <= F32(GX):
        depth = F32(GX)
    pi, grav = F32(math.pi), F32(9.807)
    wavelength = F32(20.0) * depth
    width = F32(2.0) * wavelength
    alpha_c = F32(10.0)
    t = F32(wavelength / F32(math.sqrt(float(F32(grav * depth)))))
    omega = F32(F32(F32(2.0) * pi) / t)
    if laycord == 0:
        sw = F32(F32(F32(width / F32(6378000.0)) * F32(180.0)) / pi)
    else:
        sw = width
    r_max = width
    xa = np.asarray(x, dtype=F32)
    ya = np.asarray(y, dtype=F32)
    xs, ys = F32(xa[0] + sw), F32(ya[0] + sw)
    xe, ye = F32(xa[-1] - sw), F32(ya[-1] - sw)
    em1 = F32(F32(math.exp(1.0)) - F32(1.0))

    def ramp(v, lo, hi):
        r = np.where(v <= lo, -(v - lo), np.where(v >= hi, v - hi, F32(0.0))).astype(F32)
        r = np.clip(r, F32(0.0), r_max).astype(F32)
        a = (r / r_max).astype(F32)
        e = np.exp((a * a).astype(np.float64)).astype(F32)
        c = ((alpha_c * omega) * (e - F32(1.0))).astype(F32) / em1
        c = c.astype(F32)
        return np.where(c <= F32(EPS), F32(0.0), c).astype(F32)

    cxv = ramp(xa, xs, xe)
    cyv = ramp(ya, ys, ye)
    ny, nx = len(ya), len(xa)
    return (np.ascontiguousarray(np.broadcast_to(cxv[None, :], (ny, nx))),
            np.ascontiguousarray(np.broadcast_to(cyv[:, None], (ny, nx))))


def bc_wall(h: np.ndarray, ini_switch: int = 0, incident: int = 0) -> np.ndarray:
    """BC_WALL (boundaries.f90:388-428): a copy of H with the two outermost
    rows / columns set to -999 m (land), all four sides unless a wave maker
    (INI_SWITCH 2) enters through side INCIDENT (1 top, 2 bottom, 3 left,
    4 right), which stays open"""
    out = np.array(h, dtype=F32, copy=True)
    sides = {"w": True, "s": True, "e": True, "n": True}
    if ini_switch == 2:
        # the Fortran leaves one side commented out per incident direction
        open_side = {1: "n", 2: "s", 3: "w", 4: "e"}.get(incident)
        if open_side is None:
            return out
        sides[open_side] = False
    if sides["w"]:
        out[:, 0:2] = -999.0
    if sides["s"]:
        out[0:2, :] = -999.0
    if sides["e"]:
        out[:, -2:] = -999.0
    if sides["n"]:
        out[-2:, :] = -999.0
    return out


# ---------------------------------------------------------------------
# SC_OPTION = 1: Cartesian child of a spherical parent (UTM coupling)
# ---------------------------------------------------------------------
# WGS84 constants as initialization.f90:1410-1420 / 1520-1530 state them
_UTM_A, _UTM_K0 = 6378137.0, 0.9996
_UTM_ES = 0.006739496756587
_UTM_F2, _UTM_F4, _UTM_F6 = 0.006694380004261, 0.00004481472364144701, 0.0000003000067898417773


def _meridian_arc(lat):
    a, f2, f4, f6 = _UTM_A, _UTM_F2, _UTM_F4, _UTM_F6
    return a * ((1.0 - f2 / 4.0 - 3.0 * f4 / 64.0 - 5.0 * f6 / 256.0) * lat
                - (3.0 * f2 / 8.0 + 3.0 * f4 / 32.0 + 45.0 * f6 / 1024.0) * np.sin(2.0 * lat)
                + (15.0 * f4 / 256.0 + 45.0 * f6 / 1024.0) * np.sin(4.0 * lat)
                - (35.0 * f6 / 3072.0) * np.sin(6.0 * lat))


def _pole():
    return math.pi / 2.0 - 1.0e-10


def sph_to_utm(lon, lat, lon0):
    """SPH_TO_UTM (initialization.f90:1490-1590): transverse Mercator on
    WGS84 about central meridian lon0 (degrees), natural origin on the
    equator, no false easting / northing; double precision"""
    lat = np.clip(np.asarray(lat, np.float64) * RAD_DEG, -_pole(), _pole())
    lon = np.asarray(lon, np.float64) * RAD_DEG
    ln0 = lon0 * RAD_DEG
    cs, sn = np.cos(lat), np.sin(lat)
    tn = sn / cs
    nu = _UTM_A / np.sqrt(1.0 - _UTM_F2 * sn ** 2)
    t = tn ** 2
    c = _UTM_ES * cs ** 2
    p = (lon - ln0) * cs
    s = _meridian_arc(lat)
    es = _UTM_ES
    x = _UTM_K0 * nu * (p + (1.0 - t + c) * p ** 3 / 6.0 + (5.0 - 18.0 * t + t ** 2 + 72.0 * c - 58.0 * es) * p ** 5 / 120.0)
    y = _UTM_K0 * (s + nu * tn * (p ** 2 / 2.0 + (5.0 - t + 9.0 * c + 4.0 * c ** 2) * p ** 4 / 24.0
                                  + (61.0 - 58.0 * t + t ** 2 + 600.0 * c - 330.0 * es) * p ** 6 / 720.0))
    return x, y


def utm_to_sph(x, y, lon0):
    """UTM_TO_SPH (initialization.f90:1390-1487): the inverse, with the
    footpoint latitude series; double precision"""
    a, f2, es, k0 = _UTM_A, _UTM_F2, _UTM_ES, _UTM_K0
    x = np.asarray(x, np.float64)
    y = np.asarray(y, np.float64)
    mu1 = (y / k0) / a / (1.0 - f2 / 4.0 - 3.0 * _UTM_F4 / 64.0 - 5.0 * _UTM_F6 / 256.0)
    e1 = (1.0 - math.sqrt(1.0 - f2)) / (1.0 + math.sqrt(1.0 - f2))
    lt1 = (mu1 + (3.0 * e1 / 2.0 - 27.0 * e1 ** 3 / 32.0) * np.sin(2.0 * mu1)
           + (21.0 * e1 ** 2 / 16.0 - 55.0 * e1 ** 4 / 32.0) * np.sin(4.0 * mu1)
           + (151.0 * e1 ** 3 / 96.0) * np.sin(6.0 * mu1) + (1097.0 * e1 ** 4 / 512.0) * np.sin(8.0 * mu1))
    lt1 = np.clip(lt1, -_pole(), _pole())
    tmp1 = np.sqrt(1.0 - f2 * np.sin(lt1) ** 2)
    nu1 = a / tmp1
    rho1 = a * (1.0 - f2) / tmp1 ** 3
    t1 = np.tan(lt1) ** 2
    c1 = es * np.cos(lt1) ** 2
    d = x / nu1 / k0
    lat = lt1 - nu1 * np.tan(lt1) / rho1 * (d ** 2 / 2.0 - (5.0 + 3.0 * t1 + 10.0 * c1 - 4.0 * c1 ** 2 - 9.0 * es)
                                            * d ** 4 / 24.0 + (61.0 + 90.0 * t1 + 298.0 * c1 + 45.0 * t1 ** 2
                                                               - 252 * es - 3.0 * c1 ** 2) * d ** 6 / 720.0)
    lon = lon0 * RAD_DEG + 1.0 / np.cos(lt1) * (d - (1.0 + 2.0 * t1 + c1) * d ** 3 / 6.0
                                               + (5.0 - 2.0 * c1 + 28.0 * t1 - 3.0 * c1 ** 2 + 8.0 * es
                                                  + 24.0 * t1 ** 2) * d ** 5 / 120.0)
    return lon * 180.0 / math.pi, lat * 180.0 / math.pi


def utm_zone_meridian(olon: float) -> float:
    """COORD_CONVERT (initialization.f90:1340-1350): central meridian of the
    6-degree zone holding olon, zones numbered from 0 E; 0 when none does"""
    lon0 = 0.0
    for i in range(60):
        zc = 3.0 + i * 6.0
        if zc - 3.0 <= olon < zc + 3.0:
            lon0 = zc
    return lon0


def coord_convert_to_utm(lon, lat, olon, olat):
    """COORD_CONVERT option 0: easting / northing with the false offsets"""
    x, y = sph_to_utm(lon, lat, utm_zone_meridian(olon))
    return x + 500000.0, y + (10000000.0 if olat < 0.0 else 0.0)


def coord_convert_to_sph(x, y, olon, olat):
    """COORD_CONVERT option 1"""
    return utm_to_sph(np.asarray(x) - 500000.0, np.asarray(y) - (10000000.0 if olat < 0.0 else 0.0),
                      utm_zone_meridian(olon))


@dataclass
class ScGeometry:
    """a Cartesian child of a spherical parent under SC_OPTION = 1"""
    x: np.ndarray          # [nx] easting (m)
    y: np.ndarray          # [ny] northing (m)
    dx: float
    dy: float
    pos: np.ndarray        # [ny, nx, 2] int32, 1-based (KI, KJ) of the parent cell holding each child node
    cxy: np.ndarray        # [ny, nx, 4] float32 bilinear weights of (KI,KJ),(KI+1,KJ),(KI,KJ+1),(KI+1,KJ+1)
    corners: list          # [IMIN, IMAX, JMIN, JMAX] of pos (the child's corners after matching)
    xs: float
    ys: float


def sc_child_geometry(xp, yp, corners_, rel_size, dx_min_parent, del_y_parent=None) -> ScGeometry:
    """SUBGRID_MATCHING for LAYCORD 0 -> 1 (initialization.f90:996-1123):
    the child's UTM axes from the projected window corners, then the
    position and weight tables of every child node in the parent grid"""
    xp = np.asarray(xp, np.float64)
    yp = np.asarray(yp, np.float64)
    c1, c2, c3, c4 = corners_
    dely = dx_min_parent if del_y_parent is None else del_y_parent[c3 - 1]
    dx = dx_min_parent / 60.0 / rel_size
    dy = dely / 60.0 / rel_size
    xs = 0.5 * (xp[c1 - 1] + xp[c1 - 2]) - dx / 2.0
    xe = 0.5 * (xp[c2 - 1] + xp[c2]) - dx / 2.0
    ys = 0.5 * (yp[c3 - 1] + yp[c3 - 2]) - dy / 2.0
    ye = 0.5 * (yp[c4 - 1] + yp[c4]) - dy / 2.0
    nx = (c2 - c1 + 1) * rel_size + 1
    ny = (c4 - c3 + 1) * rel_size + 1
    x_end, _ = coord_convert_to_utm(xe, ys, xs, ys)
    _, y_end = coord_convert_to_utm(xs, ye, xs, ys)
    x0, y0 = coord_convert_to_utm(xs, ys, xs, ys)
    dxm = (float(x_end) - float(x0)) / (nx - 1)
    dym = (float(y_end) - float(y0)) / (ny - 1)
    x = float(x0) + np.arange(nx) * dxm
    y = float(y0) + np.arange(ny) * dym
    X, Y = np.meshgrid(x, y)
    lon, lat = coord_convert_to_sph(X, Y, xs, ys)
    npx, npy = len(xp), len(yp)
    # KI: the K in 2..NX-1 with X(K) <= lon < X(K+1), else 0 (1-based)
    ki = np.searchsorted(xp, lon, side="right")          # first index with xp > lon -> K+1 (1-based K)
    ok_i = (ki >= 2) & (ki <= npx - 1)
    ki = np.where(ok_i, ki, 0)
    kj = np.searchsorted(yp, lat, side="right")
    ok_j = (kj >= 2) & (kj <= npy - 1)
    kj = np.where(ok_j, kj, 0)
    pos = np.stack([ki, kj], axis=-1).astype(np.int32)
    cxy = np.zeros((ny, nx, 4), np.float32)
    good = ok_i & ok_j
    kk = np.where(good, ki, 1) - 1
    jj = np.where(good, kj, 1) - 1
    cx = (lon - xp[kk]) / (xp[kk + 1] - xp[kk])
    cy = (lat - yp[jj]) / (yp[jj + 1] - yp[jj])
    w = np.stack([(1.0 - cx) * (1.0 - cy), cx * (1.0 - cy), (1.0 - cx) * cy, cx * cy], axis=-1)
    cxy[good] = w[good].astype(np.float32)
    corners_sc = [int(ki.min()), int(ki.max()), int(kj.min()), int(kj.max())]
    return ScGeometry(x=x, y=y, dx=dxm, dy=dym, pos=pos, cxy=cxy, corners=corners_sc, xs=xs, ys=ys)
