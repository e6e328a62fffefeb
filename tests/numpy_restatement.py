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


# ---------------------------------------------------------------------
# dispersion-corrected forms with the reference's all-zero MASK
# (dispersion.f90:239-1692), the sponge (boundaries.f90:206-247) and the
# SC_OPTION = 1 coupling (all_grids.f90:996-1425)
# ---------------------------------------------------------------------
TWLVTH = F(0.08333333333333)


def mass_d(z1, m1, n1, h, root, sph, r1=None, r11=None, r6=None, rx=None, ry=None):
    """MASS_S_D / MASS_C_D: linear continuity, land clamp ZZ+H <= 0"""
    ny, nx = h.shape
    z2 = z1.copy() if not root else np.zeros_like(z1)
    je = ny - 1 if root else ny
    ie = nx - 1 if root else nx
    J, I = slice(1, je), slice(1, ie)
    if sph:
        zz = (z1[J, I] - r1[J, None] * (m1[J, I] - m1[J, 0:ie - 1])
              - r11[J, None] * (n1[J, I] * r6[J, None] - n1[0:je - 1, I] * r6[0:je - 1, None]))
    else:
        zz = z1[J, I] - F(rx) * (m1[J, I] - m1[J, 0:ie - 1]) - F(ry) * (n1[J, I] - n1[0:je - 1, I])
    zz = np.where(np.abs(zz) < EPS, F(0), zz)
    hh = h[J, I]
    zz = np.where(zz + hh <= F(0), -hh, zz)
    z2[J, I] = np.where(hh > GX, zz, F(0))
    if root:
        z2[0, :] = z1[0, :]; z2[-1, :] = z1[-1, :]; z2[:, 0] = z1[:, 0]; z2[:, -1] = z1[:, -1]
    return z2


def momt_s_d(z2, m1, n1, h, r2, r3, r4, r5, modscm, root):
    """MOMT_S_D: MOMT_S, the modified-scheme term when MODSCM = 0, y wet test > 0"""
    ny, nx = h.shape
    m2 = np.zeros_like(m1)
    n2 = np.zeros_like(n1)
    lo = 0 if root else 1
    jj, ii = np.meshgrid(np.arange(lo, ny), np.arange(lo, nx - 1), indexing="ij")
    jm, jp = np.maximum(jj - 1, 0), np.minimum(jj + 1, ny - 1)
    tot_n = n1[jj, ii] + n1[jj, ii + 1] + n1[jm, ii] + n1[jm, ii + 1]
    xm = m1[jj, ii] - r2[jj, ii] * (z2[jj, ii + 1] - z2[jj, ii]) + r3[jj] * tot_n
    if modscm == 0:
        scm = r2[jj, ii] * TWLVTH * ((z2[jp, ii + 1] - F(2) * z2[jj, ii + 1] + z2[jm, ii + 1])
                                     - (z2[jp, ii] - F(2) * z2[jj, ii] + z2[jm, ii]))
        xm = xm - scm
    xm = np.where(np.abs(xm) < EPS, F(0), xm)
    m2[jj, ii] = np.where((h[jj, ii] > GX) & (h[jj, ii + 1] > GX), xm, F(0))
    jj, ii = np.meshgrid(np.arange(lo, ny - 1), np.arange(lo, nx), indexing="ij")
    im, ip = np.maximum(ii - 1, 0), np.minimum(ii + 1, nx - 1)
    tot_m = m1[jj, im] + m1[jj + 1, im] + m1[jj, ii] + m1[jj + 1, ii]
    xn = n1[jj, ii] - r4[jj, ii] * (z2[jj + 1, ii] - z2[jj, ii]) - r5[jj] * tot_m
    if modscm == 0:
        scm = r4[jj, ii] * TWLVTH * ((z2[jj + 1, ip] - F(2) * z2[jj + 1, ii] + z2[jj + 1, im])
                                     - (z2[jj, ip] - F(2) * z2[jj, ii] + z2[jj, im]))
        xn = xn - scm
    xn = np.where(np.abs(xn) < EPS, F(0), xn)
    n2[jj, ii] = np.where((h[jj, ii] > F(0)) & (h[jj + 1, ii] > F(0)), xn, F(0))
    return m2, n2


def momt_c_d(z2, m1, n1, h, hp, grx, gry, dt, fric_switch, fm, modscm, root, m2_old, n2_old, powf):
    """MOMT_C_D: total face depth, Manning friction, modified-scheme term;
    dry faces keep m2_old / n2_old; powf is the shared float power"""
    ny, nx = h.shape
    m2 = m2_old.copy()
    n2 = n2_old.copy()
    lo = 0 if root else 1
    konst = F(0.5) * F(dt) * GRAV
    fm, grx, gry, mexp = F(fm), F(grx), F(gry), F(2.3333333)
    def _pow(a):
        with np.errstate(all="ignore"):
            return np.float32(powf(np.float32(a), mexp))
    vpow = np.vectorize(_pow, otypes=[np.float32])
    jj, ii = np.meshgrid(np.arange(lo, ny), np.arange(lo, nx - 1), indexing="ij")
    jm, jp = np.maximum(jj - 1, 0), np.minimum(jj + 1, ny - 1)
    hm = hp[jj, ii] + F(0.5) * (z2[jj, ii] + z2[jj, ii + 1])
    ff = np.zeros_like(hm)
    if fric_switch != 1:
        xqq = F(0.25) * (n1[jj, ii] + n1[jj, ii + 1] + n1[jm, ii] + n1[jm, ii + 1])
        with np.errstate(all="ignore"):   # the masked-off branch may divide by 0
            ff = np.where(hm >= F(1.0e-3), konst * fm * fm * np.sqrt(m1[jj, ii] * m1[jj, ii] + xqq * xqq)
                          / vpow(hm), F(0))
    xm = (F(1) - ff) * m1[jj, ii] - grx * hm * (z2[jj, ii + 1] - z2[jj, ii])
    if modscm == 0:
        xm = xm - grx * TWLVTH * hm * ((z2[jp, ii + 1] - F(2) * z2[jj, ii + 1] + z2[jm, ii + 1])
                                       - (z2[jp, ii] - F(2) * z2[jj, ii] + z2[jm, ii]))
    if fric_switch != 1:
        xm = xm / (F(1) + ff)
    xm = np.where(np.abs(xm) < EPS, F(0), xm)
    wet = (h[jj, ii] > GX) & (h[jj, ii + 1] > GX)
    m2[jj[wet], ii[wet]] = xm[wet]
    jj, ii = np.meshgrid(np.arange(lo, ny - 1), np.arange(lo, nx), indexing="ij")
    im, ip = np.maximum(ii - 1, 0), np.minimum(ii + 1, nx - 1)
    hn = F(0.5) * (h[jj, ii] + h[jj + 1, ii] + z2[jj, ii] + z2[jj + 1, ii])
    ff = np.zeros_like(hn)
    if fric_switch != 1:
        xpp = F(0.25) * (m1[jj, ii] + m1[jj + 1, ii] + m1[jj, im] + m1[jj + 1, im])
        with np.errstate(all="ignore"):
            ff = np.where(hn >= F(1.0e-5), konst * fm * fm * np.sqrt(n1[jj, ii] * n1[jj, ii] + xpp * xpp)
                          / vpow(hn), F(0))
    xn = (F(1) - ff) * n1[jj, ii] - gry * hn * (z2[jj + 1, ii] - z2[jj, ii])
    if modscm == 0:
        xn = xn - gry * TWLVTH * hn * ((z2[jj + 1, ip] - F(2) * z2[jj + 1, ii] + z2[jj + 1, im])
                                       - (z2[jj, ip] - F(2) * z2[jj, ii] + z2[jj, im]))
    if fric_switch != 1:
        xn = xn / (F(1) + ff)
    xn = np.where(np.abs(xn) < EPS, F(0), xn)
    wet = (h[jj, ii] > GX) & (h[jj + 1, ii] > GX)
    n2[jj[wet], ii[wet]] = xn[wet]
    return m2, n2


def sponge(m2, n2, m1, n1, cx, cy, dt):
    """SPONGE_LAYER: M2 += CX*DT*M1, N2 += CY*DT*N1 where CX or CY > 0"""
    on = (cx > 0) | (cy > 0)
    dt = F(dt)
    return (np.where(on, m2 + cx * dt * m1, m2).astype(F), np.where(on, n2 + cy * dt * n1, n2).astype(F))


def _bilin(f, ps, w):
    """Z1+Z2+Z3+Z4 of the weighted 2x2 parent values; ps 1-based (KI, KJ)"""
    i, j = ps[..., 0] - 1, ps[..., 1] - 1
    return f[j, i] * w[..., 0] + f[j, i + 1] * w[..., 1] + f[j + 1, i] * w[..., 2] + f[j + 1, i + 1] * w[..., 3]


def edge_sc(pm1, pn1, ch, cz2, cm1, cn1, pos, cxy):
    """EDGE_INTERP_SC with the wet test at the edge node"""
    cm1, cn1 = cm1.copy(), cn1.copy()
    for sl in (np.s_[:, 0], np.s_[:, -1]):
        wet = ch[sl] + cz2[sl] > GX
        cm1[sl] = np.where(wet, _bilin(pm1, pos[sl], cxy[sl]), F(0))
    for sl in (np.s_[0, :], np.s_[-1, :]):
        wet = ch[sl] + cz2[sl] > GX
        cn1[sl] = np.where(wet, _bilin(pn1, pos[sl], cxy[sl]), F(0))
    return cm1, cn1


def newq_sc_blend(pm1, pn1, pm2, pn2, ch, cz2, cm1, cn1, pos, cxy, t, rel_time, fix_top):
    """NEWQ_SC's edge blend C1*X2 + C2*X1 (the top edge: C1*X1 unless fixed)"""
    c1 = (F(t) - F(1)) / F(rel_time)
    c2 = F(1) - c1
    cm1, cn1 = cm1.copy(), cn1.copy()
    for sl in (np.s_[:, 0], np.s_[:, -1]):
        wet = ch[sl] + cz2[sl] > GX
        cm1[sl] = np.where(wet, c1 * _bilin(pm2, pos[sl], cxy[sl]) + c2 * _bilin(pm1, pos[sl], cxy[sl]), F(0))
    for k, sl in enumerate((np.s_[0, :], np.s_[-1, :])):
        wet = ch[sl] + cz2[sl] > GX
        w1 = c1 if (k == 1 and not fix_top) else c2
        cn1[sl] = np.where(wet, c1 * _bilin(pn2, pos[sl], cxy[sl]) + w1 * _bilin(pn1, pos[sl], cxy[sl]), F(0))
    return cm1, cn1


def jnz_sc(pz2, ch, cz2, pos, corners, rel_size):
    """JNZ_SC: per parent cell the mean of the wet child surfaces in it,
    summed in child I-outer order, where more than r*r/2 contributed"""
    out = pz2.copy()
    zs = np.zeros_like(pz2)
    cs = np.zeros_like(pz2)
    ny, nx = ch.shape
    for i in range(nx):
        for j in range(ny):
            if ch[j, i] + cz2[j, i] > GX:
                ki, kj = pos[j, i] - 1
                zs[kj, ki] = F(zs[kj, ki] + cz2[j, i])
                cs[kj, ki] = F(cs[kj, ki] + F(1))
    half = F(rel_size * rel_size) / F(2)
    c0, c1, c2, c3 = corners
    blk = np.s_[c2 - 1:c3, c0 - 1:c1]
    out[blk] = np.where(cs[blk] > half, zs[blk] / np.where(cs[blk] > 0, cs[blk], F(1)), out[blk])
    return out
