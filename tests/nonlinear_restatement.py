"""A second, independent restatement of the nonlinear solvers, written
cell by cell from the Fortran in float32 scalar arithmetic: CONMASS
(mass.f90:162-224), CONMASS_S (mass.f90:227-277), CONMOME (moment.f90:280-780),
CONMOME_S (moment.f90:783-1268) and WAVE_BREAKING (moment.f90:1272-1384).
It is test infrastructure that cross-checks the C oracle; it is slow and
meant for small grids.  Arrays are [ny, nx] numpy float32; indices below are
the Fortran ones (I, J from 1).  The float power and exponential are the
shared definitions (passed in), everything else is plain float32."""
import numpy as np

F = np.float32
GX, EPS, ELMAX, GRAV, VLIM = F(1e-5), F(1e-10), F(-50.0), F(9.807), F(20.0)
MEXP = F(2.3333333)


class Grid:
    def __init__(self, a):
        self.a = a

    def __call__(self, i, j):
        return self.a[j - 1, i - 1]

    def set(self, i, j, v):
        self.a[j - 1, i - 1] = v


def conmass(s, sph, root):
    """s: dict of fields and coefficients; writes s['z2'], s['dz2']"""
    nx, ny = s["nx"], s["ny"]
    h, z1, m1, n1 = Grid(s["h"]), Grid(s["z1"]), Grid(s["m1"]), Grid(s["n1"])
    z2, dz2 = Grid(s["z2"]), Grid(s["dz2"])
    ie, je = (nx - 1, ny - 1) if root else (nx, ny)
    for j in range(2, je + 1):
        for i in range(2, ie + 1):
            hh = h(i, j)
            wet = hh >= ELMAX if sph else hh > ELMAX
            if wet:
                if sph:
                    zz = (z1(i, j) - s["r1"][j - 1] * (m1(i, j) - m1(i - 1, j))
                          - s["r11"][j - 1] * (n1(i, j) * s["r6"][j - 1] - n1(i, j - 1) * s["r6"][j - 2]))
                else:
                    zz = z1(i, j) - F(s["rx"]) * (m1(i, j) - m1(i - 1, j)) - F(s["ry"]) * (n1(i, j) - n1(i, j - 1))
                if abs(zz) < EPS:
                    zz = F(0)
                dd = F(zz + hh)
                if dd >= GX:
                    dz2.set(i, j, dd)
                    z2.set(i, j, zz)
                else:
                    dz2.set(i, j, F(0))
                    z2.set(i, j, -hh)
            else:
                dz2.set(i, j, F(0))
                z2.set(i, j, -hh)


def _breaking(s, i, j, advx, advy, expf):
    dz2, z1, z2 = Grid(s["dz2"]), Grid(s["z1"]), Grid(s["z2"])
    c = np.sqrt(GRAV * dz2(i, j))
    f_, i_ = F(0.08) * c, F(0.65) * c
    dzdt = F(abs(z2(i, j) - z1(i, j)) / F(s["dt"]))
    if dzdt > f_:
        with np.errstate(all="ignore"):   # a dry cell (c = 0) gives REF = inf, COEF = 0, as in float
            ref = (dzdt - f_) / (i_ - f_)
        coef = F(expf(F(-(F(1.0) * ref))))
        advx, advy = coef * advx, coef * advy
    return advx, advy


def conmome(s, sph, root, powf, expf):
    """writes s['m2'], s['n2'] (cells outside the loops keep their values)"""
    nx, ny = s["nx"], s["ny"]
    hz, hp, hq = Grid(s["h"]), Grid(s["hp"]), Grid(s["hq"])
    z, p, q, dz = Grid(s["z2"]), Grid(s["m1"]), Grid(s["n1"]), Grid(s["dz2"])
    m2, n2 = Grid(s["m2"]), Grid(s["n2"])
    dt, fric, fm = F(s["dt"]), s["fric_switch"], F(s["fric_coef"])
    const = F(F(0.5) * dt) * GRAV if fric != 1 else F(0)
    lin, mod = s["linchk"], s["modscm"]

    def row(name, j):
        return F(s[name][j - 1])

    def cx(j):
        return row("cx", j) if sph else F(s["grx"])

    def cy(j):
        return row("cy", j) if sph else F(s["gry"])

    def ax(j):
        return row("r1", j) if sph else F(s["rx"])    # R21 = R1

    def ay(j):
        return row("r0", j) if sph else F(s["ry"])

    def bx(j):
        return row("r22", j) if sph else F(s["rx"])

    # DP/DQ, with DZ(:,:,1) = 0 (never written by the reference)
    DP1, DP2 = np.zeros((ny + 1, nx + 1), F), np.zeros((ny + 1, nx + 1), F)
    DQ1, DQ2 = np.zeros((ny + 1, nx + 1), F), np.zeros((ny + 1, nx + 1), F)
    for i in range(1, nx + 1):
        ip1 = min(i + 1, nx)
        for j in range(1, ny + 1):
            jp1 = min(j + 1, ny)
            d1 = F(0.25) * (dz(i, j) + F(0) + dz(ip1, j) + F(0))
            d2 = F(0.5) * (dz(i, j) + dz(ip1, j))
            e1 = F(0.25) * (dz(i, j) + F(0) + dz(i, jp1) + F(0))
            e2 = F(0.5) * (dz(i, j) + dz(i, jp1))
            DP1[j, i] = F(0) if d1 < GX else d1
            DP2[j, i] = F(0) if d2 < GX else d2
            DQ1[j, i] = F(0) if e1 < GX else e1
            DQ2[j, i] = F(0) if e2 < GX else e2
    dp1 = lambda i, j: DP1[j, i]
    dq1 = lambda i, j: DQ1[j, i]
    span = lambda i, j: 10 < i < nx - 10 and 10 < j < ny - 10

    # x
    if root:
        is_, js, ie, je = 1, 1, nx - 1, ny - 1
    else:
        is_, js, ie, je = 2, 2, nx - 1, ny
    for i in range(is_, ie + 1):
        ip1 = min(i + 1, nx)
        im1 = max(i - 1, 1)
        for j in range(js, je + 1):
            jp1, jm1 = min(j + 1, ny), max(j - 1, 1)
            noflux = False
            dd = df = F(0)
            if hz(i, j) <= ELMAX or hp(i, j) <= ELMAX:
                noflux = True
            else:
                if dz(i, j) > GX and dz(ip1, j) > GX:
                    dd, df = DP2[j, i], DP1[j, i]
                elif dz(i, j) > GX and dz(ip1, j) <= GX and hz(ip1, j) + z(i, j) > GX:
                    dd = hp(i, j) + F(0.5) * (z(i, j) + z(ip1, j)) if sph else F(0.5) * dz(i, j)
                    df = dd
                elif dz(i, j) <= GX and dz(ip1, j) > GX and hz(i, j) + z(ip1, j) > GX:
                    dd = hp(i, j) + F(0.5) * (z(i, j) + z(ip1, j)) if sph else F(0.5) * dz(ip1, j)
                    df = dd
                else:
                    noflux = True
                if not noflux and dd < GX:
                    noflux = True
            if noflux:
                m2.set(i, j, F(0))
                continue
            if df < F(1.0e-3):
                df = F(1.0e-3)
            xqq = F(0.25) * (q(i, j) + q(ip1, j) + q(i, jm1) + q(ip1, jm1))
            ff = const * fm * fm * np.sqrt(p(i, j) * p(i, j) + xqq * xqq) / F(powf(df, MEXP)) if fric != 1 else F(0)
            xp = p(i, j) - cx(j) * dd * (z(ip1, j) - z(i, j))
            if mod == 0 and j < ny:
                xp = xp - cx(j) * dd / F(12.0) * ((z(ip1, jp1) - F(2) * z(ip1, j) + z(ip1, jm1))
                                                   - (z(i, jp1) - F(2) * z(i, j) + z(i, jm1)))
            if fric != 1:
                xp = xp - ff * p(i, j)
            if sph:
                xp = xp + F(4.0) * row("r3", j) * xqq
            if lin == 1 and dp1(i, j) >= GX and span(i, j):
                if p(i, j) < 0:
                    if dp1(ip1, j) < GX or dz(ip1, j) < GX:
                        advx = ax(j) * (-(p(i, j) * p(i, j) / dp1(i, j)))
                    else:
                        advx = ax(j) * (p(ip1, j) * p(ip1, j) / dp1(ip1, j) - p(i, j) * p(i, j) / dp1(i, j))
                else:
                    if dp1(im1, j) < GX or dz(i, j) < GX:
                        advx = ax(j) * (p(i, j) * p(i, j) / dp1(i, j))
                    else:
                        advx = ax(j) * (p(i, j) * p(i, j) / dp1(i, j) - p(im1, j) * p(im1, j) / dp1(im1, j))
                if xqq < 0:
                    if dz(i, jp1) < GX or dz(ip1, jp1) < GX or dp1(i, jp1) < GX:
                        advy = ay(j) * (-(p(i, j) * xqq / dp1(i, j)))
                    else:
                        xqe = F(0.25) * (q(i, jp1) + q(ip1, jp1) + q(i, j) + q(ip1, j))
                        advy = ay(j) * (p(i, jp1) * xqe / dp1(i, jp1) - p(i, j) * xqq / dp1(i, j))
                else:
                    if dz(i, jm1) < GX or dz(ip1, jm1) < GX or dp1(i, jm1) < GX:
                        advy = ay(j) * (p(i, j) * xqq / dp1(i, j))
                    else:
                        xqe = F(0.25) * (q(i, jm1) + q(ip1, jm1) + q(i, j - 2) + q(ip1, j - 2))
                        advy = ay(j) * (p(i, j) * xqq / dp1(i, j) - p(i, jm1) * xqe / dp1(i, jm1))
                advx, advy = _breaking(s, i, j, advx, advy, expf)
                xp = xp - advx - advy
            if fric != 1:
                xp = xp / (F(1.0) + ff)
            if abs(xp) < EPS:
                xp = F(0)
            lim = VLIM * dd
            if xp > lim:
                xp = lim
            if xp < -lim:
                xp = -lim
            m2.set(i, j, F(xp))

    # y
    if root:
        is_, js, ie, je = 1, 1, nx - 1, ny - 1
    else:
        is_, js, ie, je = 2, 2, nx, ny - 1
    for i in range(is_, ie + 1):
        ip1 = min(i + 1, nx)
        im1 = max(i - 1, 1)
        for j in range(js, je + 1):
            jp1, jm1 = min(j + 1, ny), max(j - 1, 1)
            noflux = False
            dd = df = F(0)
            if hz(i, j) <= ELMAX or hq(i, j) <= ELMAX:
                noflux = True
            else:
                if dz(i, j) > GX and dz(i, jp1) > GX:
                    dd, df = DQ2[j, i], DQ1[j, i]
                elif dz(i, j) > GX and dz(i, jp1) <= GX and hz(i, jp1) + z(i, j) > GX:
                    dd = hq(i, j) + F(0.5) * (z(i, j) + z(i, jp1)) if sph else F(0.5) * dz(i, j)
                    df = dd
                elif dz(i, j) <= GX and dz(i, jp1) > GX and hz(i, j) + z(i, jp1) > GX:
                    dd = hq(i, j) + F(0.5) * (z(i, j) + z(i, jp1)) if sph else F(0.5) * dz(i, jp1)
                    df = dd
                else:
                    noflux = True
                if not noflux and dd < GX:
                    noflux = True
            if noflux:
                n2.set(i, j, F(0))
                continue
            if df < F(1.0e-3):
                df = F(1.0e-3)
            xpp = F(0.25) * (p(i, j) + p(i, jp1) + p(im1, j) + p(im1, jp1))
            ff = const * fm * fm * np.sqrt(q(i, j) * q(i, j) + xpp * xpp) / F(powf(df, MEXP)) if fric != 1 else F(0)
            xq = q(i, j) - cy(j) * dd * (z(i, jp1) - z(i, j))
            if mod == 0 and i < nx:
                xq = xq - cy(j) * dd / F(12.0) * ((z(ip1, jp1) - F(2) * z(i, jp1) + z(im1, jp1))
                                                   - (z(ip1, j) - F(2) * z(i, j) + z(im1, j)))
            if sph:
                if fric != 1:
                    xq = xq - ff * q(i, j)
                xq = xq - F(4.0) * row("r5", j) * xpp
            # the Cartesian routine subtracts this friction from XP (moment.f90:672): XQ keeps it
            if lin == 1 and dq1(i, j) >= GX and span(i, j):
                if q(i, j) < 0:
                    if dq1(i, jp1) < GX or dz(i, jp1) < GX:
                        advy = ay(j) * (-(q(i, j) * q(i, j) / dq1(i, j)))
                    else:
                        advy = ay(j) * (q(i, jp1) * q(i, jp1) / dq1(i, jp1) - q(i, j) * q(i, j) / dq1(i, j))
                else:
                    if dq1(i, jm1) < GX or dz(i, j) < GX:
                        advy = ay(j) * (q(i, j) * q(i, j) / dq1(i, j))
                    else:
                        advy = ay(j) * (q(i, j) * q(i, j) / dq1(i, j) - q(i, jm1) * q(i, jm1) / dq1(i, jm1))
                if xpp < 0:
                    if dz(ip1, j) < GX or dz(ip1, jp1) < GX or dq1(ip1, j) < GX:
                        advx = bx(j) * (-(q(i, j) * xpp / dq1(i, j)))
                    else:
                        xpe = F(0.25) * (p(ip1, j) + p(ip1, jp1) + p(i, j) + p(i, jp1))
                        advx = bx(j) * (q(ip1, j) * xpe / dq1(ip1, j) - q(i, j) * xpp / dq1(i, j))
                else:
                    if dz(im1, j) < GX or dz(im1, jp1) < GX or dq1(i - 1, j) < GX:
                        advx = bx(j) * (q(i, j) * xpp / dq1(i, j))
                    else:
                        xpe = F(0.25) * (p(im1, j) + p(im1, jp1) + p(i - 2, j) + p(i - 2, jp1))
                        advx = bx(j) * (q(i, j) * xpp / dq1(i, j) - q(im1, j) * xpe / dq1(im1, j))
                advx, advy = _breaking(s, i, j, advx, advy, expf)
                xq = xq - advx - advy
            if fric != 1:
                xq = xq / (F(1.0) + ff)
            if abs(xq) < EPS:
                xq = F(0)
            lim = VLIM * dd
            if xq > lim:
                xq = lim
            if xq < -lim:
                xq = -lim
            n2.set(i, j, F(xq))
