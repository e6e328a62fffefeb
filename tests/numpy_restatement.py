"""A second, independent restatement of the linear spherical step in
vectorised numpy float32 (MASS_S mass.f90:61-100, OPEN boundaries.f90:22-202,
MOMT_S moment.f90:65-149), used only to cross-check the C oracle.  numpy
float32 operations round like the Fortran REAL ones, so the two agree bit for
bit when both follow the Fortran operation order."""
import numpy as np

F = np.float32
GX, EPS, GRAV, UB = F(1e-5), F(1e-10), F(9.807), F(99.0)


def mass_s(z1, m1, n1, h, r1, r11, r6, root=True):
    ny, nx = h.shape
    z2 = np.zeros_like(z1)
    je = ny - 1 if root else ny
    ie = nx - 1 if root else nx
    J = slice(1, je)
    I = slice(1, ie)
    zz = (z1[J, I] - r1[J, None] * (m1[J, I] - m1[J, 0:ie - 1])
          - r11[J, None] * (n1[J, I] * r6[J, None] - n1[0:je - 1, I] * r6[0:je - 1, None]))
    zz = np.where(np.abs(zz) < EPS, F(0), zz)
    hh = h[J, I]
    zz = np.where(zz + hh <= EPS, -hh, zz)
    z2[J, I] = np.where(hh > GX, zz, F(0))
    return z2


def open_bc(z2, m, n, h):
    ny, nx = h.shape
    z2 = z2.copy()

    def put(j, i, zz, hc):
        zz = np.where(np.abs(zz) > UB, F(0), zz)
        z2[j, i] = np.where(hc > GX, zz, F(0))

    with np.errstate(invalid="ignore", divide="ignore"):
        i = np.arange(1, nx - 1)
        # J = 1
        hc = h[0, i]; cc = np.sqrt(GRAV * hc)
        uh = F(0.5) * (m[0, i] + m[0, i - 1]); uu = np.sqrt(uh * uh + n[0, i] * n[0, i]); zz = uu / cc
        put(0, i, np.where(n[0, i] > 0, -zz, zz), hc)
        # J = NY
        hc = h[-1, i]; cc = np.sqrt(GRAV * hc); ns = n[-2, i]
        uh = F(0.5) * (m[-1, i] + m[-1, i - 1]); uu = np.sqrt(uh * uh + ns * ns); zz = uu / cc
        put(ny - 1, i, np.where(ns < 0, -zz, zz), hc)
        j = np.arange(1, ny - 1)
        # I = 1
        hc = h[j, 0]; cc = np.sqrt(GRAV * hc)
        uh = np.where(h[j - 1, 0] > GX, F(0.5) * (n[j, 0] + n[j - 1, 0]), n[j, 0])
        uu = np.sqrt(uh * uh + m[j, 0] * m[j, 0]); zz = uu / cc
        put(j, 0, np.where(m[j, 0] > 0, -zz, zz), hc)
        # I = NX
        hc = h[j, -1]; cc = np.sqrt(GRAV * hc); mw = m[j, -2]
        uh = F(0.5) * (n[j, -1] + n[j - 1, -1]); uu = np.sqrt(uh * uh + mw * mw); zz = uu / cc
        put(j, nx - 1, np.where(mw < 0, -zz, zz), hc)
        # corners
        for (jj, ii, qx, qy, neg) in ((0, 0, m[0, 0], n[0, 0], lambda a, b: a > 0 or b > 0),
                                      (0, nx - 1, m[0, nx - 2], n[0, nx - 1], lambda a, b: a < 0 or b > 0),
                                      (ny - 1, 0, m[ny - 1, 0], n[ny - 2, 0], lambda a, b: a > 0 or b < 0),
                                      (ny - 1, nx - 1, m[ny - 1, nx - 2], n[ny - 2, nx - 1], lambda a, b: a < 0 or b < 0)):
            hc = h[jj, ii]
            if hc > GX:
                zz = np.sqrt(qx * qx + qy * qy) / np.sqrt(GRAV * hc)
                if neg(qx, qy):
                    zz = -zz
                if abs(zz) > UB:
                    zz = F(0)
                z2[jj, ii] = zz
            else:
                z2[jj, ii] = F(0)
    return z2


def momt_s(z2, m1, n1, h, r2, r3, r4, r5, root=True):
    ny, nx = h.shape
    m2 = np.zeros_like(m1)
    n2 = np.zeros_like(n1)
    lo = 0 if root else 1
    # x: I = lo..NX-2 (0-based), J = lo..NY-1
    J = np.arange(lo, ny)
    Jm = np.maximum(J - 1, 0)
    I = np.arange(lo, nx - 1)
    jj, ii = np.meshgrid(J, I, indexing="ij")
    jm = np.maximum(jj - 1, 0)
    tot_n = n1[jj, ii] + n1[jj, ii + 1] + n1[jm, ii] + n1[jm, ii + 1]
    xm = m1[jj, ii] - r2[jj, ii] * (z2[jj, ii + 1] - z2[jj, ii]) + r3[jj] * tot_n
    xm = np.where(np.abs(xm) < EPS, F(0), xm)
    wet = (h[jj, ii] > GX) & (h[jj, ii + 1] > GX)
    m2[jj, ii] = np.where(wet, xm, F(0))
    # y: J = lo..NY-2, I = lo..NX-1
    J = np.arange(lo, ny - 1)
    I = np.arange(lo, nx)
    jj, ii = np.meshgrid(J, I, indexing="ij")
    im = np.maximum(ii - 1, 0)
    tot_m = m1[jj, im] + m1[jj + 1, im] + m1[jj, ii] + m1[jj + 1, ii]
    xn = n1[jj, ii] - r4[jj, ii] * (z2[jj + 1, ii] - z2[jj, ii]) - r5[jj] * tot_m
    xn = np.where(np.abs(xn) < EPS, F(0), xn)
    wet = (h[jj, ii] > GX) & (h[jj + 1, ii] > GX)
    n2[jj, ii] = np.where(wet, xn, F(0))
    return m2, n2


def run_single(L, nsteps):
    """outer steps of a single linear spherical root layer; returns z, m, n, zmax"""
    c = L.coefs
    z1 = L.Z0.astype(F).copy()
    m1 = np.zeros_like(z1)
    n1 = np.zeros_like(z1)
    zmax = z1.copy()
    for _ in range(nsteps):
        z2 = mass_s(z1, m1, n1, L.H, c.r1, c.r11, c.r6)
        z2 = open_bc(z2, m1, n1, L.H)
        m2, n2 = momt_s(z2, m1, n1, L.H, c.r2, c.r3, c.r4, c.r5)
        zmax = np.where(zmax >= z2, zmax, z2)
        z1, m1, n1 = z2, m2, n2
    return z1, m1, n1, zmax
