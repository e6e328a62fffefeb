/*
 * Per-phase sm_100a kernels of the COMCOT time stepper: one launch per phase
 * and layer.  These are the building blocks of the nested sub-cycle and the
 * "plain" path the fused and batched kernels are measured against.
 *
 * Every kernel evaluates the Fortran expression in the Fortran order with
 * separately rounded float operations (the library is built with
 * -fmad=false; IEEE division and square root), so results are bit-identical
 * to the REAL arithmetic of the reference solvers cited per kernel.
 * Indices are 0-based: Fortran (I,J) = (i+1, j+1).
 */
#include <utility>
#include <algorithm>

#include "gc_internal.h"

namespace {

constexpr int BX = 32, BY = 8;

__device__ __forceinline__ float fabs_(float x) { return x < 0.0f ? -x : x; }

/* a / b bit for bit, without the division where a is a signed zero and b
 * positive (IEEE 754 gives a itself there).  Still water makes many zero
 * numerators, and a correctly rounded division costs far more than the
 * test.  NaN or non-positive b always takes the division. */
__device__ __forceinline__ float qdiv(float a, float b) {
    if (a == 0.0f && b > 0.0f) return a;
    return a / b;
}
/* a / (1 + ff) for the friction divisor: also without the division where
 * 1 + ff rounded to exactly 1 (friction below 2^-24, as in deep water) and
 * a is a number */
__device__ __forceinline__ float fdiv1(float a, float onepff) {
    if (onepff == 1.0f && a == a) return a;
    return qdiv(a, onepff);
}

/* ---------------------------------------------------------------- */
/* continuity                                                        */
/* ---------------------------------------------------------------- */
/* Programmatic dependent launch: a kernel launched with it may be scheduled
 * while its predecessor still runs; griddepcontrol.wait then blocks until
 * the predecessor has completed and its writes are visible, so it comes
 * before any global access.  launch_dependents lets the next kernel in the
 * stream be scheduled early.  Both are no-ops for an ordinary launch. */
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

/* MASS_S (mass.f90:61-100) and, NONLIN, CONMASS_S (mass.f90:226-278).  Child
 * edge rows i==0 / j==0 are not computed by the reference; they keep the
 * value of time level 1 (the UPDATE edge copy of all_grids.f90:323-324 made
 * them equal), so they are carried over here. */
template <bool NONLIN>
__global__ void k_mass_s(GcLayerDev L) {
    pdl_enter();
    int i = blockIdx.x * BX + threadIdx.x;
    int j = blockIdx.y * BY + threadIdx.y;
    if (i >= L.nx || j >= L.ny) return;
    size_t c = (size_t)j * L.pitch + i;
    if (L.root) {
        if (i < 1 || i > L.nx - 2 || j < 1 || j > L.ny - 2) return;
    } else if (i == 0 || j == 0) {
        L.z2[c] = L.z1[c];
        return;
    }
    float h = L.h[c];
    if (NONLIN) {
        float dz, z;
        if (h >= CC_ELMAX) {
            float r1 = GC_ROW(L, GC_R1, j), r11 = GC_ROW(L, GC_R11, j);
            float r6 = GC_ROW(L, GC_R6, j), r6m = GC_ROW(L, GC_R6, j - 1);
            float zz = L.z1[c] - r1 * (L.m1[c] - L.m1[c - 1])
                       - r11 * (L.n1[c] * r6 - L.n1[c - L.pitch] * r6m);
            if (fabsf(zz) < CC_EPS) zz = 0.0f;
            float dd = zz + h;
            if (dd >= CC_GX) { dz = dd; z = zz; }
            else { dz = 0.0f; z = -h; }
        } else {
            dz = 0.0f; z = -h;
        }
        L.dz2[c] = dz;
        L.z2[c] = z;
        return;
    }
    float out;
    if (h > CC_GX) {
        float r1 = GC_ROW(L, GC_R1, j), r11 = GC_ROW(L, GC_R11, j);
        float r6 = GC_ROW(L, GC_R6, j), r6m = GC_ROW(L, GC_R6, j - 1);
        float zz = L.z1[c] - r1 * (L.m1[c] - L.m1[c - 1])
                   - r11 * (L.n1[c] * r6 - L.n1[c - L.pitch] * r6m);
        if (fabsf(zz) < CC_EPS) zz = 0.0f;
        if ((zz + h) <= CC_EPS) zz = -h;
        out = zz;
    } else {
        out = 0.0f;
    }
    L.z2[c] = out;
}

/* MASS_C (mass.f90:103-157) and CONMASS (mass.f90:162-224) */
template <bool NONLIN>
__global__ void k_mass_c(GcLayerDev L) {
    pdl_enter();
    int i = blockIdx.x * BX + threadIdx.x;
    int j = blockIdx.y * BY + threadIdx.y;
    if (i >= L.nx || j >= L.ny) return;
    size_t c = (size_t)j * L.pitch + i;
    if (L.root) {
        if (i < 1 || i > L.nx - 2 || j < 1 || j > L.ny - 2) return;
    } else if (i == 0 || j == 0) {
        L.z2[c] = L.z1[c];
        return;
    }
    float h = L.h[c];
    float zz = L.z1[c] - L.rx * (L.m1[c] - L.m1[c - 1]) - L.ry * (L.n1[c] - L.n1[c - L.pitch]);
    if (fabsf(zz) < CC_EPS) zz = 0.0f;
    if (!NONLIN) {
        float out;
        if (h > CC_GX) {
            if ((zz + h) <= CC_EPS) zz = -h;
            out = zz;
        } else {
            out = 0.0f;
        }
        L.z2[c] = out;
    } else {
        float dz, z;
        if (h > CC_ELMAX) {
            float dd = zz + h;
            if (dd >= CC_GX) { dz = dd; z = zz; }
            else { dz = 0.0f; z = -h; }
        } else {
            dz = 0.0f; z = -h;
        }
        L.dz2[c] = dz;
        L.z2[c] = z;
    }
}

/* ---------------------------------------------------------------- */
/* linear spherical momentum (moment.f90:65-149)                     */
/* ---------------------------------------------------------------- */
__device__ __forceinline__ float r2_at(const GcLayerDev &L, int i, int j, size_t c, float h,
                                       float hp1) {
    if (L.explicit_r24) return L.r2[c];
    /* R2 = RS/COS_M/(DX*RAD_MIN) * AMAX1(HP,0) with HP from PQ_DEPTH; the
     * caller only needs it where H(i)>GX and H(i+1)>GX, so HP>0 there. */
    return GC_ROW(L, GC_CX, j) * (0.5f * (h + hp1));
}
__device__ __forceinline__ float r4_at(const GcLayerDev &L, int i, int j, size_t c, float h,
                                       float hq1) {
    if (L.explicit_r24) return L.r4[c];
    return GC_ROW(L, GC_CY, j) * (0.5f * (h + hq1));
}

/* MASS_S_D / MASS_C_D (dispersion.f90:239-543), LAYGOV 2 and 3.  The
 * reference's ALPHA clears its whole MASK inside the cell loop
 * (dispersion.f90:125), so every cell takes the non-dispersive branch
 * (:333-337, :460-462): linear continuity with the land clamp ZZ+H <= ZERO. */
template <bool SPH>
__global__ void k_mass_d(GcLayerDev L) {
    pdl_enter();
    int i = blockIdx.x * BX + threadIdx.x;
    int j = blockIdx.y * BY + threadIdx.y;
    if (i >= L.nx || j >= L.ny) return;
    size_t c = (size_t)j * L.pitch + i;
    if (L.root) {
        if (i < 1 || i > L.nx - 2 || j < 1 || j > L.ny - 2) return;
    } else if (i == 0 || j == 0) {
        L.z2[c] = L.z1[c];
        return;
    }
    const float h = L.h[c];
    float out = 0.0f;
    if (h > CC_GX) {
        float zz;
        if (SPH)
            zz = L.z1[c] - GC_ROW(L, GC_R1, j) * (L.m1[c] - L.m1[c - 1])
                 - GC_ROW(L, GC_R11, j) * (L.n1[c] * GC_ROW(L, GC_R6, j) - L.n1[c - L.pitch] * GC_ROW(L, GC_R6, j - 1));
        else
            zz = L.z1[c] - L.rx * (L.m1[c] - L.m1[c - 1]) - L.ry * (L.n1[c] - L.n1[c - L.pitch]);
        if (fabsf(zz) < CC_EPS) zz = 0.0f;
        if ((zz + h) <= 0.0f) zz = -h;
        out = zz;
    }
    L.z2[c] = out;
}

/* MOMT_S_D / MOMT_C_D (dispersion.f90:544-1692), LAYGOV 2 and 3, with the
 * reference's MASK = 0.  Spherical (:681-692, :812-823): MOMT_S plus the
 * modified-scheme term when MODSCM = 0, the y wet test against ZERO (:706).
 * Cartesian (:1225-1233, :1560-1568): face depth HM = HP + (Z + Z(I+1))/2,
 * HN = (H + H(J+1) + Z + Z(J+1))/2, Manning friction, the modified-scheme
 * term; a dry face is not written by the reference (:922, :1255), so it
 * keeps its level-2 value, which equals level 1 after CHANGE / UPDATE. */
template <bool SPH>
__global__ void k_momt_d(GcLayerDev L) {
    pdl_enter();
    const int i = blockIdx.x * BX + threadIdx.x;
    const int j = blockIdx.y * BY + threadIdx.y;
    const int nx = L.nx, ny = L.ny, P = L.pitch;
    if (i >= nx || j >= ny) return;
    const size_t c = (size_t)j * P + i;
    const int lo = L.root ? 0 : 1;
    const float *z = L.z2;
    const float konst = 0.5f * L.dt * CC_GRAV, fm = L.fric_coef;
    /* x: I = IS..NX-1, J = JS..NY; cells outside are never written by the
     * reference and stay 0 */
    if (!(i >= lo && i <= nx - 2 && j >= lo)) {
        L.m2[c] = 0.0f;
    } else {
        const size_t cp = c + 1;
        const int jm1 = j > 0 ? j - 1 : 0, jp1 = j < ny - 1 ? j + 1 : ny - 1;
        const size_t cm = (size_t)jm1 * P + i, cu = (size_t)jp1 * P + i;
        const float h = L.h[c], hp1 = L.h[cp];
        if (SPH) {
            float xm = 0.0f;
            if (h > CC_GX && hp1 > CC_GX) {
                const float tot_n = L.n1[c] + L.n1[cp] + L.n1[cm] + L.n1[cm + 1];
                const float r2 = r2_at(L, i, j, c, h, hp1);
                xm = L.m1[c] - r2 * (z[cp] - z[c]) + GC_ROW(L, GC_R3, j) * tot_n;
                if (L.modscm == 0) {
                    const float scm = r2 * CC_TWLVTH * ((z[cu + 1] - 2.0f * z[cp] + z[cm + 1]) - (z[cu] - 2.0f * z[c] + z[cm]));
                    xm = xm - scm;
                }
                if (fabsf(xm) < CC_EPS) xm = 0.0f;
            }
            L.m2[c] = xm;
        } else if (h > CC_GX && hp1 > CC_GX) {
            const float hm = L.hp[c] + 0.5f * (z[c] + z[cp]);
            float ff = 0.0f;
            if (L.fric_switch != 1) {
                const float xqq = 0.25f * (L.n1[c] + L.n1[cp] + L.n1[cm] + L.n1[cm + 1]);
                if (hm >= 1.0e-3f)
                    {
                    /* the guard above keeps hm >= 1e-3, so the power is positive */
                    const float fnum = konst * fm * fm * sqrtf(L.m1[c] * L.m1[c] + xqq * xqq);
                    ff = (fnum == 0.0f) ? fnum : fnum / cc_powf(hm, CC_MANNEXP);
                }
            }
            float xm = (1.0f - ff) * L.m1[c] - L.grx * hm * (z[cp] - z[c]);
            if (L.modscm == 0) {
                const float scm = L.grx * CC_TWLVTH * hm * ((z[cu + 1] - 2.0f * z[cp] + z[cm + 1]) - (z[cu] - 2.0f * z[c] + z[cm]));
                xm = xm - scm;
            }
            if (L.fric_switch != 1) xm = fdiv1(xm, 1.0f + ff);
            if (fabsf(xm) < CC_EPS) xm = 0.0f;
            L.m2[c] = xm;
        } else {
            L.m2[c] = L.m1[c];
        }
    }
    /* y: J = JS..NY-1, I = IS..NX */
    if (!(j >= lo && j <= ny - 2 && i >= lo)) {
        L.n2[c] = 0.0f;
    } else {
        const size_t cq = c + P;
        const int im1 = i > 0 ? i - 1 : 0, ip1 = i < nx - 1 ? i + 1 : nx - 1;
        const size_t cw = (size_t)j * P + im1, ce = (size_t)j * P + ip1;
        const float h = L.h[c], hq1 = L.h[cq];
        if (SPH) {
            float xn = 0.0f;
            if (h > 0.0f && hq1 > 0.0f) {
                const float tot_m = L.m1[cw] + L.m1[cw + P] + L.m1[c] + L.m1[cq];
                /* R4 = C(J) * AMAX1(HQ,0), HQ = 0 where H <= GX (PQ_DEPTH) */
                const float r4 = L.explicit_r24 ? L.r4[c] : (h > CC_GX ? r4_at(L, i, j, c, h, hq1) : 0.0f);
                xn = L.n1[c] - r4 * (z[cq] - z[c]) - GC_ROW(L, GC_R5, j) * tot_m;
                if (L.modscm == 0) {
                    const float scm = r4 * CC_TWLVTH * ((z[ce + P] - 2.0f * z[cq] + z[cw + P]) - (z[ce] - 2.0f * z[c] + z[cw]));
                    xn = xn - scm;
                }
                if (fabsf(xn) < CC_EPS) xn = 0.0f;
            }
            L.n2[c] = xn;
        } else if (h > CC_GX && hq1 > CC_GX) {
            const float hn = 0.5f * (h + hq1 + z[c] + z[cq]);
            float ff = 0.0f;
            if (L.fric_switch != 1) {
                const float xpp = 0.25f * (L.m1[c] + L.m1[cq] + L.m1[cw] + L.m1[cw + P]);
                if (hn >= 1.0e-5f)
                    {
                    /* the guard above keeps hn >= 1e-5, so the power is positive */
                    const float fnum = konst * fm * fm * sqrtf(L.n1[c] * L.n1[c] + xpp * xpp);
                    ff = (fnum == 0.0f) ? fnum : fnum / cc_powf(hn, CC_MANNEXP);
                }
            }
            float xn = (1.0f - ff) * L.n1[c] - L.gry * hn * (z[cq] - z[c]);
            if (L.modscm == 0) {
                const float scm = L.gry * CC_TWLVTH * hn * ((z[ce + P] - 2.0f * z[cq] + z[cw + P]) - (z[ce] - 2.0f * z[c] + z[cw]));
                xn = xn - scm;
            }
            if (L.fric_switch != 1) xn = fdiv1(xn, 1.0f + ff);
            if (fabsf(xn) < CC_EPS) xn = 0.0f;
            L.n2[c] = xn;
        } else {
            L.n2[c] = L.n1[c];
        }
    }
}

/* over the cells i0 <= i < i0+ni, j0 <= j < j0+nj (the whole layer, or a
 * window whose level-2 surface changed after the layer's step) */
__global__ void k_momt_s(GcLayerDev L, int i0, int j0, int ni, int nj) {
    pdl_enter();
    int i = i0 + blockIdx.x * BX + threadIdx.x;
    int j = j0 + blockIdx.y * BY + threadIdx.y;
    if (i >= i0 + ni || j >= j0 + nj || i >= L.nx || j >= L.ny) return;
    const int P = L.pitch;
    size_t c = (size_t)j * P + i;
    int lo = L.root ? 0 : 1;
    /* x-momentum: i in [lo, nx-2], j in [lo, ny-1]; 0 elsewhere */
    float xm = 0.0f;
    if (i >= lo && i <= L.nx - 2 && j >= lo) {
        float h = L.h[c], hp1 = L.h[c + 1];
        if (h > CC_GX && hp1 > CC_GX) {
            size_t cm = (j > 0) ? c - P : c;  /* JM1 = max(J-1,1) */
            float tot_n = L.n1[c] + L.n1[c + 1] + L.n1[cm] + L.n1[cm + 1];
            xm = L.m1[c] - r2_at(L, i, j, c, h, hp1) * (L.z2[c + 1] - L.z2[c])
                 + GC_ROW(L, GC_R3, j) * tot_n;
            if (fabsf(xm) < CC_EPS) xm = 0.0f;
        }
    }
    L.m2[c] = xm;
    /* y-momentum: j in [lo, ny-2], i in [lo, nx-1]; 0 elsewhere */
    float xn = 0.0f;
    if (j >= lo && j <= L.ny - 2 && i >= lo) {
        float h = L.h[c], hq1 = L.h[c + P];
        if (h > CC_GX && hq1 > CC_GX) {
            size_t cw = (i > 0) ? c - 1 : c;  /* IM1 = max(I-1,1) */
            float tot_m = L.m1[cw] + L.m1[cw + P] + L.m1[c] + L.m1[c + P];
            xn = L.n1[c] - r4_at(L, i, j, c, h, hq1) * (L.z2[c + P] - L.z2[c])
                 - GC_ROW(L, GC_R5, j) * tot_m;
            if (fabsf(xn) < CC_EPS) xn = 0.0f;
        }
    }
    L.n2[c] = xn;
}

/* ---------------------------------------------------------------- */
/* linear Cartesian momentum (moment.f90:152-277)                    */
/* ---------------------------------------------------------------- */
__global__ void k_momt_c(GcLayerDev L) {
    pdl_enter();
    int i = blockIdx.x * BX + threadIdx.x;
    int j = blockIdx.y * BY + threadIdx.y;
    if (i >= L.nx || j >= L.ny) return;
    const int P = L.pitch, nx = L.nx, ny = L.ny;
    size_t c = (size_t)j * P + i;
    int lo = L.root ? 0 : 1;
    const float konst = 0.5f * L.dt * CC_GRAV;
    const float fm = L.fric_coef;
    const float *z = L.z2;
    float xm = 0.0f;
    if (i >= lo && i <= nx - 2 && j >= lo) {
        float h = L.h[c], hp1 = L.h[c + 1];
        if (h > CC_GX && hp1 > CC_GX) {
            int jm1 = j > 0 ? j - 1 : 0, jp1 = j < ny - 1 ? j + 1 : ny - 1;
            size_t cm = (size_t)jm1 * P + i, cpj = (size_t)jp1 * P + i;
            float ff = 0.0f;
            float hm = L.hp[c] + 0.5f * (z[c] + z[c + 1]);
            xm = L.m1[c] - L.grx * hm * (z[c + 1] - z[c]);
            if (L.fric_switch != 1) {
                float xqq = 0.25f * (L.n1[c] + L.n1[c + 1] + L.n1[cm] + L.n1[cm + 1]);
                if (hm >= 1.0e-3f)
                    {
                    /* the guard above keeps hm >= 1e-3, so the power is positive */
                    const float fnum = konst * fm * fm * sqrtf(L.m1[c] * L.m1[c] + xqq * xqq);
                    ff = (fnum == 0.0f) ? fnum : fnum / cc_powf(hm, CC_MANNEXP);
                }
                else
                    ff = 0.0f;
                xm = xm - ff * L.m1[c];
            }
            if (L.modscm == 0) {
                float scm = L.grx * CC_TWLVTH * hm
                            * ((z[cpj + 1] - 2.0f * z[c + 1] + z[cm + 1])
                               - (z[cpj] - 2.0f * z[c] + z[cm]));
                xm = xm - scm;
            }
            if (L.fric_switch != 1) xm = fdiv1(xm, 1.0f + ff);
            if (fabsf(xm) < CC_EPS) xm = 0.0f;
        }
    }
    L.m2[c] = xm;
    float xn = 0.0f;
    if (j >= lo && j <= ny - 2 && i >= lo) {
        float h = L.h[c], hq1 = L.h[c + P];
        if (h > CC_GX && hq1 > CC_GX) {
            int im1 = i > 0 ? i - 1 : 0, ip1 = i < nx - 1 ? i + 1 : nx - 1;
            size_t cq = c + P;
            float ff = 0.0f;
            float hn = L.hq[c] + 0.5f * (z[c] + z[cq]);
            xn = L.n1[c] - L.gry * hn * (z[cq] - z[c]);
            if (L.fric_switch != 1) {
                float xpp = 0.25f * (L.m1[c] + L.m1[cq] + L.m1[(size_t)j * P + im1]
                                     + L.m1[(size_t)(j + 1) * P + im1]);
                if (hn >= 1.0e-5f)
                    {
                    /* the guard above keeps hn >= 1e-5, so the power is positive */
                    const float fnum = konst * fm * fm * sqrtf(L.n1[c] * L.n1[c] + xpp * xpp);
                    ff = (fnum == 0.0f) ? fnum : fnum / cc_powf(hn, CC_MANNEXP);
                }
                else
                    ff = 0.0f;
                xn = xn - ff * L.n1[c];
            }
            if (L.modscm == 0) {
                size_t r0 = (size_t)j * P, r1 = (size_t)(j + 1) * P;
                float scm = L.gry * CC_TWLVTH * hn
                            * ((z[r1 + ip1] - 2.0f * z[r1 + i] + z[r1 + im1])
                               - (z[r0 + ip1] - 2.0f * z[r0 + i] + z[r0 + im1]));
                xn = xn - scm;
            }
            if (L.fric_switch != 1) xn = fdiv1(xn, 1.0f + ff);
            if (fabsf(xn) < CC_EPS) xn = 0.0f;
        }
    }
    L.n2[c] = xn;
}

/* ---------------------------------------------------------------- */
/* nonlinear Cartesian momentum: CONMOME (moment.f90:280-780) with    */
/* WAVE_BREAKING (moment.f90:1272-1384).  DZ(:,:,1) is identically    */
/* zero in the reference, so DP1 = 0.25*(DZ2(I)+DZ2(I+1)) etc.         */
/* ---------------------------------------------------------------- */
/* face depths from two total depths (moment.f90:345-366): the x form
 * DP1/DP2 of cells (I,J),(I+1,J), the y form DQ1/DQ2 of (I,J),(I,J+1) */
__device__ __forceinline__ float face1(float a, float b) {
    float v = 0.25f * (a + 0.0f + b + 0.0f);
    return v < CC_GX ? 0.0f : v;
}
__device__ __forceinline__ float face2(float a, float b) {
    float v = 0.50f * (a + b);
    return v < CC_GX ? 0.0f : v;
}

/* WAVE_BREAKING (moment.f90:1302-1335) on one cell's total depth, new and
 * old surface */
__device__ __forceinline__ void wave_breaking(float dz2c, float z2c, float z1c, float dt, float &advx,
                                              float &advy) {
    float cc = sqrtf(CC_GRAV * dz2c);
    float dzdt_f = CC_BRK_F * cc;
    float dzdt_i = CC_BRK_I * cc;
    float dzdt = qdiv(fabs_(z2c - z1c), dt);
    if (dzdt > dzdt_f) {
        float ref = (dzdt - dzdt_f) / (dzdt_i - dzdt_f);
        float coef = cc_expf(-(1.0f * ref));
        advx = coef * advx;
        advy = coef * advy;
    }
}

/* CONMOME (moment.f90:280-780) and, SPH, CONMOME_S (moment.f90:783-1268):
 * the same structure; the spherical form takes the wet/dry face depth as
 * HP + (Z + Z(I+1))/2, the pressure coefficient R2 / R4 of its row, Coriolis
 * +4 R3 XQQ / -4 R5 XPP, advection coefficients R21 (= R1) / R0 / R22 per
 * row, and applies the y friction to XQ (the Cartesian routine subtracts it
 * from XP, moment.f90:672).
 *
 * Every value a face can need (its stencil reaches two cells back along the
 * face normal's neighbour axis and one cell forward) is loaded first, as
 * one batch of independent loads at clamped, in-bounds indices; the
 * branches then run on registers.  Clamped indices coincide with the
 * reference's wherever a value is used: the two-back neighbours are read
 * only inside the advection span, whose cells are at least 10 from every
 * edge. */
/* the stencil of one x face (I,J)-(I+1,J): names give the cell relative to
 * (I,J): p = I+1, m = I-1, p2 = I+2, n = J+1, s = J-1, s2 = J-2; zpn etc.
 * are the surface's corners for the modified-scheme term */
struct XFace {
    float h_c, h_p, hp_c, d_c, d_p, d_p2, d_m, d_cn, d_pn, d_cs, d_ps;
    float z_c, z_p, z1_c, q_c, q_p, q_cs, q_ps, q_cn, q_pn, q_cs2, q_ps2;
    float p_c, p_p, p_m, p_n, p_s;
    float z_pn, z_ps, z_cn, z_cs;
};
/* the stencil of one y face (I,J)-(I,J+1): q = J+1, q2 = J+2, s = J-1,
 * e = I+1, w = I-1, w2 = I-2 */
struct YFace {
    float h_c, h_q, hq_c, d_c, d_q, d_q2, d_s, d_e, d_eq, d_w, d_wq;
    float z_c, z_q, z1_c, p_c, p_q, p_w, p_wq, p_e, p_eq, p_w2, p_w2q;
    float q_c, q_q, q_s, q_e, q_w;
    float z_eq, z_wq, z_e, z_w;
};

/* CONMOME / CONMOME_S x direction at one face (moment.f90:409-568,
 * 1272-1384); `span`: inside the advection span */
template <bool SPH>
__device__ __forceinline__ float conmome_x(const GcLayerDev &L, const XFace &f, int j, int jy, bool span) {
    const float konst = (L.fric_switch != 1) ? 0.5f * L.dt * CC_GRAV : 0.0f;
    const float fm = L.fric_coef;
    float dd = 0.0f, df = 0.0f, ff;
    bool noflux = false;
    if (f.h_c <= CC_ELMAX || f.hp_c <= CC_ELMAX) {
        noflux = true;
    } else {
        if (f.d_c > CC_GX && f.d_p > CC_GX) {
            dd = face2(f.d_c, f.d_p); df = face1(f.d_c, f.d_p);
        } else if (f.d_c > CC_GX && f.d_p <= CC_GX && f.h_p + f.z_c > CC_GX) {
            dd = SPH ? f.hp_c + 0.5f * (f.z_c + f.z_p) : 0.5f * f.d_c; df = dd;
        } else if (f.d_c <= CC_GX && f.d_p > CC_GX && f.h_c + f.z_p > CC_GX) {
            dd = SPH ? f.hp_c + 0.5f * (f.z_c + f.z_p) : 0.5f * f.d_p; df = dd;
        } else {
            noflux = true;
        }
        if (!noflux && dd < CC_GX) noflux = true;
    }
    if (noflux) return 0.0f;
    if (df < CC_DFMIN) df = CC_DFMIN;
    float xqq = 0.25f * (f.q_c + f.q_p + f.q_cs + f.q_ps);
    if (L.fric_switch != 1) {
        /* df >= DFMIN here unless it is NaN, so the power is positive */
        const float fnum = konst * fm * fm * sqrtf(f.p_c * f.p_c + xqq * xqq);
        ff = (fnum == 0.0f && df >= CC_DFMIN) ? fnum : fnum / cc_powf(df, CC_MANNEXP);
    } else {
        ff = 0.0f;
    }
    const float cpx = SPH ? GC_ROW(L, GC_CX, j) : L.grx;
    float xp = f.p_c - cpx * dd * (f.z_p - f.z_c);
    if (L.modscm == 0 && j + 1 < jy) {
        float scm = qdiv(cpx * dd, 12.0f) * ((f.z_pn - 2.0f * f.z_p + f.z_ps) - (f.z_cn - 2.0f * f.z_c + f.z_cs));
        xp = xp - scm;
    }
    if (L.fric_switch != 1) xp = xp - ff * f.p_c;
    if (SPH) xp = xp + 4.0f * GC_ROW(L, GC_R3, j) * xqq;
    const float ax = SPH ? GC_ROW(L, GC_R1, j) : L.rx;   /* R21 = R1 */
    const float ay = SPH ? L.rows2[2 * (size_t)j] : L.ry; /* R0 */
    float dp1c = face1(f.d_c, f.d_p);
    if (L.linchk == 1 && dp1c >= CC_GX && span) {
        float advx, advy;
        if (f.p_c < 0.0f) {
            float dp1p = face1(f.d_p, f.d_p2);
            if (dp1p < CC_GX || f.d_p < CC_GX)
                advx = ax * (-(qdiv(f.p_c * f.p_c, dp1c)));
            else
                advx = ax * (qdiv(f.p_p * f.p_p, dp1p) - qdiv(f.p_c * f.p_c, dp1c));
        } else {
            float dp1m = face1(f.d_m, f.d_c);
            if (dp1m < CC_GX || f.d_c < CC_GX)
                advx = ax * (qdiv(f.p_c * f.p_c, dp1c));
            else
                advx = ax * (qdiv(f.p_c * f.p_c, dp1c) - qdiv(f.p_m * f.p_m, dp1m));
        }
        if (xqq < 0.0f) {
            if (f.d_cn < CC_GX || f.d_pn < CC_GX) {
                advy = ay * (-(qdiv(f.p_c * xqq, dp1c)));
            } else if (face1(f.d_cn, f.d_pn) < CC_GX) {
                advy = ay * (-(qdiv(f.p_c * xqq, dp1c)));
            } else {
                float xqe = 0.25f * (f.q_cn + f.q_pn + f.q_c + f.q_p);
                advy = ay * (qdiv(f.p_n * xqe, face1(f.d_cn, f.d_pn)) - qdiv(f.p_c * xqq, dp1c));
            }
        } else {
            if (f.d_cs < CC_GX || f.d_ps < CC_GX) {
                advy = ay * (qdiv(f.p_c * xqq, dp1c));
            } else if (face1(f.d_cs, f.d_ps) < CC_GX) {
                advy = ay * (qdiv(f.p_c * xqq, dp1c));
            } else {
                float xqe = 0.25f * (f.q_cs + f.q_ps + f.q_cs2 + f.q_ps2);
                advy = ay * (qdiv(f.p_c * xqq, dp1c) - qdiv(f.p_s * xqe, face1(f.d_cs, f.d_ps)));
            }
        }
        wave_breaking(f.d_c, f.z_c, f.z1_c, L.dt, advx, advy);
        xp = xp - advx - advy;
    }
    if (L.fric_switch != 1) xp = fdiv1(xp, 1.0f + ff);
    if (fabsf(xp) < CC_EPS) xp = 0.0f;
    float lim = CC_VLIMIT * dd;
    if (xp > lim) xp = lim;
    if (xp < -lim) xp = -lim;
    return xp;
}

/* CONMOME / CONMOME_S y direction at one face (moment.f90:570-780) */
template <bool SPH>
__device__ __forceinline__ float conmome_y(const GcLayerDev &L, const YFace &f, int i, int j, int ix, bool span) {
    const float konst = (L.fric_switch != 1) ? 0.5f * L.dt * CC_GRAV : 0.0f;
    const float fm = L.fric_coef;
    float dd = 0.0f, df = 0.0f, ff;
    bool noflux = false;
    if (f.h_c <= CC_ELMAX || f.hq_c <= CC_ELMAX) {
        noflux = true;
    } else {
        if (f.d_c > CC_GX && f.d_q > CC_GX) {
            dd = face2(f.d_c, f.d_q); df = face1(f.d_c, f.d_q);
        } else if (f.d_c > CC_GX && f.d_q <= CC_GX && f.h_q + f.z_c > CC_GX) {
            dd = SPH ? f.hq_c + 0.5f * (f.z_c + f.z_q) : 0.5f * f.d_c; df = dd;
        } else if (f.d_c <= CC_GX && f.d_q > CC_GX && f.h_c + f.z_q > CC_GX) {
            dd = SPH ? f.hq_c + 0.5f * (f.z_c + f.z_q) : 0.5f * f.d_q; df = dd;
        } else {
            noflux = true;
        }
        if (!noflux && dd < CC_GX) noflux = true;
    }
    if (noflux) return 0.0f;
    if (df < CC_DFMIN) df = CC_DFMIN;
    float xpp = 0.25f * (f.p_c + f.p_q + f.p_w + f.p_wq);
    if (L.fric_switch != 1) {
        /* df >= DFMIN here unless it is NaN, so the power is positive */
        const float fnum = konst * fm * fm * sqrtf(f.q_c * f.q_c + xpp * xpp);
        ff = (fnum == 0.0f && df >= CC_DFMIN) ? fnum : fnum / cc_powf(df, CC_MANNEXP);
    } else {
        ff = 0.0f;
    }
    const float cqy = SPH ? GC_ROW(L, GC_CY, j) : L.gry;
    float xq = f.q_c - cqy * dd * (f.z_q - f.z_c);
    if (L.modscm == 0 && i + 1 < ix) {
        float scm = qdiv(cqy * dd, 12.0f) * ((f.z_eq - 2.0f * f.z_q + f.z_wq) - (f.z_e - 2.0f * f.z_c + f.z_w));
        xq = xq - scm;
    }
    /* CONMOME applies -FF*Q to XP, which is unused (moment.f90:672):
     * no term on XQ; CONMOME_S applies it to XQ (moment.f90:1150) */
    if (SPH && L.fric_switch != 1) xq = xq - ff * f.q_c;
    if (SPH) xq = xq - 4.0f * GC_ROW(L, GC_R5, j) * xpp;
    const float by = SPH ? L.rows2[2 * (size_t)j] : L.ry;     /* R0 */
    const float bx = SPH ? L.rows2[2 * (size_t)j + 1] : L.rx; /* R22 */
    float dq1c = face1(f.d_c, f.d_q);
    if (L.linchk == 1 && dq1c >= CC_GX && span) {
        float advx, advy;
        if (f.q_c < 0.0f) {
            float dq1q = face1(f.d_q, f.d_q2);
            if (dq1q < CC_GX || f.d_q < CC_GX)
                advy = by * (-(qdiv(f.q_c * f.q_c, dq1c)));
            else
                advy = by * (qdiv(f.q_q * f.q_q, dq1q) - qdiv(f.q_c * f.q_c, dq1c));
        } else {
            float dq1m = face1(f.d_s, f.d_c);
            if (dq1m < CC_GX || f.d_c < CC_GX)
                advy = by * (qdiv(f.q_c * f.q_c, dq1c));
            else
                advy = by * (qdiv(f.q_c * f.q_c, dq1c) - qdiv(f.q_s * f.q_s, dq1m));
        }
        if (xpp < 0.0f) {
            if (f.d_e < CC_GX || f.d_eq < CC_GX) {
                advx = bx * (-(qdiv(f.q_c * xpp, dq1c)));
            } else if (face1(f.d_e, f.d_eq) < CC_GX) {
                advx = bx * (-(qdiv(f.q_c * xpp, dq1c)));
            } else {
                float xpe = 0.25f * (f.p_e + f.p_eq + f.p_c + f.p_q);
                advx = bx * (qdiv(f.q_e * xpe, face1(f.d_e, f.d_eq)) - qdiv(f.q_c * xpp, dq1c));
            }
        } else {
            if (f.d_w < CC_GX || f.d_wq < CC_GX) {
                advx = bx * (qdiv(f.q_c * xpp, dq1c));
            } else if (face1(f.d_w, f.d_wq) < CC_GX) {
                advx = bx * (qdiv(f.q_c * xpp, dq1c));
            } else {
                float xpe = 0.25f * (f.p_w + f.p_wq + f.p_w2 + f.p_w2q);
                advx = bx * (qdiv(f.q_c * xpp, dq1c) - qdiv(f.q_w * xpe, face1(f.d_w, f.d_wq)));
            }
        }
        wave_breaking(f.d_c, f.z_c, f.z1_c, L.dt, advx, advy);
        xq = xq - advx - advy;
    }
    if (L.fric_switch != 1) xq = fdiv1(xq, 1.0f + ff);
    if (fabsf(xq) < CC_EPS) xq = 0.0f;
    float lim = CC_VLIMIT * dd;
    if (xq > lim) xq = lim;
    if (xq < -lim) xq = -lim;
    return xq;
}

/* a face's stencil from a field accessor get(field, di, dj), di/dj relative
 * to the face's cell; the accessor clamps to the grid */
template <typename Get>
__device__ __forceinline__ void load_x(XFace &f, const Get &get) {
    f.d_c = get(0, 0, 0); f.d_p = get(0, 1, 0); f.d_p2 = get(0, 2, 0); f.d_m = get(0, -1, 0);
    f.d_cn = get(0, 0, 1); f.d_pn = get(0, 1, 1); f.d_cs = get(0, 0, -1); f.d_ps = get(0, 1, -1);
    f.z_c = get(1, 0, 0); f.z_p = get(1, 1, 0);
    f.z_pn = get(1, 1, 1); f.z_ps = get(1, 1, -1); f.z_cn = get(1, 0, 1); f.z_cs = get(1, 0, -1);
    f.q_c = get(3, 0, 0); f.q_p = get(3, 1, 0); f.q_cs = get(3, 0, -1); f.q_ps = get(3, 1, -1);
    f.q_cn = get(3, 0, 1); f.q_pn = get(3, 1, 1); f.q_cs2 = get(3, 0, -2); f.q_ps2 = get(3, 1, -2);
    f.p_c = get(2, 0, 0); f.p_p = get(2, 1, 0); f.p_m = get(2, -1, 0); f.p_n = get(2, 0, 1); f.p_s = get(2, 0, -1);
}
template <typename Get>
__device__ __forceinline__ void load_y(YFace &f, const Get &get) {
    f.d_c = get(0, 0, 0); f.d_q = get(0, 0, 1); f.d_q2 = get(0, 0, 2); f.d_s = get(0, 0, -1);
    f.d_e = get(0, 1, 0); f.d_eq = get(0, 1, 1); f.d_w = get(0, -1, 0); f.d_wq = get(0, -1, 1);
    f.z_c = get(1, 0, 0); f.z_q = get(1, 0, 1);
    f.z_eq = get(1, 1, 1); f.z_wq = get(1, -1, 1); f.z_e = get(1, 1, 0); f.z_w = get(1, -1, 0);
    f.p_c = get(2, 0, 0); f.p_q = get(2, 0, 1); f.p_w = get(2, -1, 0); f.p_wq = get(2, -1, 1);
    f.p_e = get(2, 1, 0); f.p_eq = get(2, 1, 1); f.p_w2 = get(2, -2, 0); f.p_w2q = get(2, -2, 1);
    f.q_c = get(3, 0, 0); f.q_q = get(3, 0, 1); f.q_s = get(3, 0, -1); f.q_e = get(3, 1, 0); f.q_w = get(3, -1, 0);
}

/* Fortran spans: I > 10 .AND. I < IX-10 with I = i+1 */
__device__ __forceinline__ bool adv_span(int i, int j, int ix, int jy) {
    return (i + 1 > CC_SPAN) && (i + 1 < ix - CC_SPAN) && (j + 1 > CC_SPAN) && (j + 1 < jy - CC_SPAN);
}

/* CONMOME, one face per thread, the x and y directions as two grid layers.
 * Every value a face can need (its stencil reaches two cells back along the
 * face normal's neighbour axis and one cell forward) is loaded first, as
 * one batch of independent loads at clamped, in-bounds indices; the
 * branches then run on registers.  Clamped indices coincide with the
 * reference's wherever a value is used: the two-back neighbours are read
 * only inside the advection span, whose cells are at least 10 from every
 * edge. */
template <bool SPH>
__global__ void k_conmome(GcLayerDev L, int upd) {
    pdl_enter();
    int i = blockIdx.x * BX + threadIdx.x;
    int j = blockIdx.y * BY + threadIdx.y;
    if (i >= L.nx || j >= L.ny) return;
    const int P = L.pitch, ix = L.nx, jy = L.ny;
    const size_t c = (size_t)j * P + i;
    /* upd: UPDATE's edge copy of a child (all_grids.f90:323-324), done here
     * by the threads of row and column 0, which compute no face.  The host
     * sets it only where no face reads the surface on row or column 0 (a
     * child without the MODSCM term), and the copy reads rows and columns
     * >= 1, which nothing in this launch writes. */
    if (upd && blockIdx.z == 0) {
        if (j == 0) L.z2[i] = L.z2[(size_t)P + (i == 0 ? 1 : i)];
        else if (i == 0) L.z2[c] = L.z2[c + 1];
    }
    const float *fields[4] = {L.dz2, L.z2, L.m1, L.n1};
    auto get = [&](int f, int di, int dj) {
        const int ii = min(max(i + di, 0), ix - 1), jj = min(max(j + dj, 0), jy - 1);
        return __ldg(fields[f] + (size_t)jj * P + ii);
    };
    const bool span = adv_span(i, j, ix, jy);
    if (blockIdx.z == 0) {
        const bool inx = L.root ? (i <= ix - 2 && j <= jy - 2) : (i >= 1 && i <= ix - 2 && j >= 1);
        float out = 0.0f;
        if (inx) {
            XFace f;
            load_x(f, get);
            f.h_c = __ldg(L.h + c); f.h_p = __ldg(L.h + c + 1); f.hp_c = __ldg(L.hp + c);
            f.z1_c = __ldg(L.z1 + c);
            out = conmome_x<SPH>(L, f, j, jy, span);
        }
        L.m2[c] = out;
    } else {
        const bool iny = L.root ? (i <= ix - 2 && j <= jy - 2) : (i >= 1 && j >= 1 && j <= jy - 2);
        float out = 0.0f;
        if (iny) {
            YFace f;
            load_y(f, get);
            f.h_c = __ldg(L.h + c); f.h_q = __ldg(L.h + c + P); f.hq_c = __ldg(L.hq + c);
            f.z1_c = __ldg(L.z1 + c);
            out = conmome_y<SPH>(L, f, i, j, ix, span);
        }
        L.n2[c] = out;
    }
}

/* CONMOME with both directions per thread, the stencil staged through
 * shared memory: a block stages its (BX+4) x (TY+4) window of DZ, Z, M and
 * N (two cells of halo, at the same clamped indices the one-face kernel
 * reads) with one batch of independent loads, then each thread computes
 * its cell's x and y faces from shared memory.  Same values, same
 * arithmetic (conmome_x / conmome_y): the same bits. */
template <bool SPH, int TY>
__device__ __forceinline__ void conmome_tile_body(const GcLayerDev &L, int upd) {
    pdl_enter();
    constexpr int TW = BX + 4, TH = TY + 4;
    __shared__ float tile[4][TH][TW];
    const int P = L.pitch, ix = L.nx, jy = L.ny;
    const int i0 = blockIdx.x * BX, j0 = blockIdx.y * TY;
    const float *fields[4] = {L.dz2, L.z2, L.m1, L.n1};
    for (int t = threadIdx.y * BX + threadIdx.x; t < TW * TH; t += BX * TY) {
        const int tj = t / TW, ti = t - tj * TW;
        const int ii = min(max(i0 + ti - 2, 0), ix - 1), jj = min(max(j0 + tj - 2, 0), jy - 1);
        const size_t g = (size_t)jj * P + ii;
#pragma unroll
        for (int f = 0; f < 4; f++) tile[f][tj][ti] = __ldg(fields[f] + g);
    }
    __syncthreads();
    const int i = i0 + threadIdx.x, j = j0 + threadIdx.y;
    if (i >= ix || j >= jy) return;
    const size_t c = (size_t)j * P + i;
    /* UPDATE's edge copy as in k_conmome: row and column 0 feed no face here */
    if (upd) {
        if (j == 0) L.z2[i] = L.z2[(size_t)P + (i == 0 ? 1 : i)];
        else if (i == 0) L.z2[c] = L.z2[c + 1];
    }
    /* the tile holds the clamped neighbour of every in-grid cell it covers;
     * for a cell near the grid edge the clamp is repeated on the offset.  A
     * block whose window lies inside the grid clamps nothing: its cells read
     * the tile at fixed offsets from their own slot. */
    auto get = [&](int f, int di, int dj) {
        const int ii = min(max(i + di, 0), ix - 1) - i0 + 2, jj = min(max(j + dj, 0), jy - 1) - j0 + 2;
        return tile[f][jj][ii];
    };
    const float *own = &tile[0][threadIdx.y + 2][threadIdx.x + 2];
    auto get_in = [&](int f, int di, int dj) { return own[(f * TH + dj) * TW + di]; };
    const bool inside = i0 >= 2 && i0 + TW - 3 <= ix - 1 && j0 >= 2 && j0 + TH - 3 <= jy - 1;
    const bool span = adv_span(i, j, ix, jy);
    const bool inx = L.root ? (i <= ix - 2 && j <= jy - 2) : (i >= 1 && i <= ix - 2 && j >= 1);
    const bool iny = L.root ? (i <= ix - 2 && j <= jy - 2) : (i >= 1 && j >= 1 && j <= jy - 2);
    const float h_c = __ldg(L.h + c), z1_c = __ldg(L.z1 + c);
    float outx = 0.0f, outy = 0.0f;
    if (inx) {
        XFace f;
        if (inside) load_x(f, get_in);
        else load_x(f, get);
        f.h_c = h_c; f.h_p = __ldg(L.h + c + 1); f.hp_c = __ldg(L.hp + c);
        f.z1_c = z1_c;
        outx = conmome_x<SPH>(L, f, j, jy, span);
    }
    if (iny) {
        YFace f;
        if (inside) load_y(f, get_in);
        else load_y(f, get);
        f.h_c = h_c; f.h_q = __ldg(L.h + c + P); f.hq_c = __ldg(L.hq + c);
        f.z1_c = z1_c;
        outy = conmome_y<SPH>(L, f, i, j, ix, span);
    }
    L.m2[c] = outx;
    L.n2[c] = outy;
}
template <bool SPH, int TY, int MINB>
__global__ void __launch_bounds__(BX * TY, MINB) k_conmome_tile(GcLayerDev L, int upd) {
    conmome_tile_body<SPH, TY>(L, upd);
}

/* ---------------------------------------------------------------- */
/* OPEN radiation boundary (boundaries.f90:22-202), outermost layer  */
/* ---------------------------------------------------------------- */
__device__ float open_cell(const GcLayerDev &L, int i, int j) {
    const int nx = L.nx, ny = L.ny, P = L.pitch;
    const float *m = L.m1, *n = L.n1, *h = L.h;
    size_t c = (size_t)j * P + i;
    float hc = h[c];
    if (!(hc > CC_GX)) return 0.0f;
    float cc = sqrtf(CC_GRAV * hc);
    float zz;
    bool corner = (i == 0 || i == nx - 1) && (j == 0 || j == ny - 1);
    if (!corner) {
        if (j == 0) {
            float uh = 0.5f * (m[c] + m[c - 1]);
            float uu = sqrtf(uh * uh + n[c] * n[c]);
            zz = uu / cc;
            if (n[c] > 0.0f) zz = -zz;
        } else if (j == ny - 1) {
            float ns = n[c - P];
            float uh = 0.5f * (m[c] + m[c - 1]);
            float uu = sqrtf(uh * uh + ns * ns);
            zz = uu / cc;
            if (ns < 0.0f) zz = -zz;
        } else if (i == 0) {
            float uh = (h[c - P] > CC_GX) ? 0.5f * (n[c] + n[c - P]) : n[c];
            float uu = sqrtf(uh * uh + m[c] * m[c]);
            zz = uu / cc;
            if (m[c] > 0.0f) zz = -zz;
        } else { /* i == nx-1 */
            float mw = m[c - 1];
            float uh = 0.5f * (n[c] + n[c - P]);
            float uu = sqrtf(uh * uh + mw * mw);
            zz = uu / cc;
            if (mw < 0.0f) zz = -zz;
        }
    } else {
        float qx, qy;
        bool neg;
        if (i == 0 && j == 0) {
            qx = m[c]; qy = n[c];
        } else if (i == nx - 1 && j == 0) {
            qx = m[c - 1]; qy = n[c];
        } else if (i == 0) {
            qx = m[c]; qy = n[c - P];
        } else {
            qx = m[c - 1]; qy = n[c - P];
        }
        float uh = sqrtf(qx * qx + qy * qy);
        zz = uh / cc;
        if (i == 0 && j == 0) neg = (qx > 0.0f || qy > 0.0f);
        else if (j == 0) neg = (qx < 0.0f || qy > 0.0f);
        else if (i == 0) neg = (qx > 0.0f || qy < 0.0f);
        else neg = (qx < 0.0f || qy < 0.0f);
        if (neg) zz = -zz;
    }
    if (fabsf(zz) > CC_UB) zz = 0.0f;
    return zz;
}

/* one thread per perimeter cell: index k walks J=1 row, J=NY row, I=1, I=NX */
__global__ void k_open(GcLayerDev L) {
    pdl_enter();
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int nx = L.nx, ny = L.ny;
    int i, j;
    if (k < nx) { i = k; j = 0; }
    else if (k < 2 * nx) { i = k - nx; j = ny - 1; }
    else if (k < 2 * nx + (ny - 2)) { i = 0; j = k - 2 * nx + 1; }
    else if (k < 2 * nx + 2 * (ny - 2)) { i = nx - 1; j = k - 2 * nx - (ny - 2) + 1; }
    else return;
    L.z2[(size_t)j * L.pitch + i] = open_cell(L, i, j);
}

/* UPDATE edge copy (all_grids.f90:323-324): Z2(1,:) = Z2(2,:), then
 * Z2(:,1) = Z2(:,2), so Z2(1,1) = Z2(2,2). */
__global__ void k_update_edges(GcLayerDev L) {
    pdl_enter();
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    const size_t P = L.pitch;
    if (k < L.ny) {
        int j = k;
        if (j >= 1) L.z2[(size_t)j * P] = L.z2[(size_t)j * P + 1];
        else L.z2[0] = L.z2[P + 1];
    } else if (k < L.ny + L.nx - 1) {
        int i = k - L.ny + 1;
        L.z2[i] = L.z2[P + i];
    }
}

/* ---------------------------------------------------------------- */
/* nesting: JNQ / NEWQ edge fluxes (all_grids.f90:452-801)           */
/* one CTA per child side; phase 1 forms the parent flux profile in   */
/* shared memory (with the T==2 forecast), phase 2 interpolates.      */
/* ---------------------------------------------------------------- */
constexpr int EDGE_THREADS = 256;

__global__ void k_edges(GcLayerDev Pl, GcLayerDev C, int ir, int rel_time, int is, int ie,
                        int js, int je, int t, int smem_len) {
    pdl_enter();
    extern __shared__ float prof[];
    const int side = blockIdx.x; /* 0 left(M), 1 right(M), 2 bottom(N), 3 top(N) */
    const bool vert = side < 2;
    const int sd = side & 1;
    /* parent line and range in Fortran 1-based indices */
    const int line = vert ? (sd == 0 ? is - 1 : ie) : (sd == 0 ? js - 1 : je);
    const int lo = vert ? js - 2 : is - 2, hi = vert ? je + 2 : ie + 2;
    const int n = hi - lo + 1;
    const int Pp = Pl.pitch;
    const float c1 = ((float)t - 1.0f) / (float)rel_time;
    const float c2 = 1.0f - c1;
    for (int k = threadIdx.x; k < n && k < smem_len; k += blockDim.x) {
        int a = lo + k;                      /* running index along the line */
        int I = vert ? line : a, J = vert ? a : line;
        size_t c = (size_t)(J - 1) * Pp + (I - 1);
        float v;
        if (t == 1) {
            v = vert ? Pl.m1[c] : Pl.n1[c];
        } else {
            v = 0.0f;
            size_t cn = vert ? c + 1 : c + Pp;   /* IP1 or JP1 neighbour */
            if ((Pl.h[c] + Pl.z2[c] > CC_GX) && (Pl.h[cn] + Pl.z2[cn] > CC_GX)) {
                float *cache = vert ? Pl.yflux + (size_t)sd * Pl.ny + (J - 1)
                                    : Pl.xflux + (size_t)sd * Pl.nx + (I - 1);
                if (t == 2) {
                    float x;
                    if (Pl.laycord == 0) {
                        if (vert) {
                            size_t cm = c - Pp; /* JM1 = J-1 */
                            float tot_n = Pl.n1[c] + Pl.n1[c + 1] + Pl.n1[cm] + Pl.n1[cm + 1];
                            float r2 = Pl.explicit_r24 ? Pl.r2[c]
                                       : GC_ROW(Pl, GC_CX, J - 1) * fmaxf(Pl.hp ? Pl.hp[c] :
                                         ((Pl.h[c] > CC_GX) ? 0.5f * (Pl.h[c] + Pl.h[c + 1]) : 0.0f), 0.0f);
                            x = Pl.m1[c] - r2 * (Pl.z2[c + 1] - Pl.z2[c]) + GC_ROW(Pl, GC_R3, J - 1) * tot_n;
                        } else {
                            size_t cw = c - 1; /* IM1 = I-1 */
                            float tot_m = Pl.m1[cw] + Pl.m1[cw + Pp] + Pl.m1[c] + Pl.m1[c + Pp];
                            float r4 = Pl.explicit_r24 ? Pl.r4[c]
                                       : GC_ROW(Pl, GC_CY, J - 1) * fmaxf(Pl.hq ? Pl.hq[c] :
                                         ((Pl.h[c] > CC_GX) ? 0.5f * (Pl.h[c] + Pl.h[c + Pp]) : 0.0f), 0.0f);
                            x = Pl.n1[c] - r4 * (Pl.z2[c + Pp] - Pl.z2[c]) - GC_ROW(Pl, GC_R5, J - 1) * tot_m;
                        }
                    } else {
                        if (vert) {
                            float hm = Pl.hp[c] + 0.5f * (Pl.z2[c] + Pl.z2[c + 1]);
                            x = Pl.m1[c] - Pl.grx * hm * (Pl.z2[c + 1] - Pl.z2[c]);
                        } else {
                            float hn = Pl.hq[c] + 0.5f * (Pl.z2[c] + Pl.z2[c + Pp]);
                            x = Pl.n1[c] - Pl.gry * hn * (Pl.z2[c + Pp] - Pl.z2[c]);
                        }
                    }
                    if (fabsf(x) < CC_EPS) x = 0.0f;
                    *cache = x;
                }
                v = c1 * (*cache) + c2 * (vert ? Pl.m1[c] : Pl.n1[c]);
            }
        }
        prof[k] = v;
    }
    __syncthreads();
    /* EDGEINTERP_VERT / _HORI (all_grids.f90:502-604) */
    const int a0 = vert ? js : is, a1 = vert ? je : ie;
    const int nn = 2 * ir;
    const int fixed = vert ? (sd == 0 ? 0 : C.nx - 1) : (sd == 0 ? 0 : C.ny - 1);
    const int total = (a1 - a0 + 1) * ir;
    const int Pc = C.pitch;
    for (int w = threadIdx.x; w < total; w += blockDim.x) {
        int a = a0 + w / ir;
        int kk = w % ir + 1;
        int o = a - lo; /* profile offset of F(a) */
        float fs = 0.5f * (prof[o - 1] + prof[o]);
        float fe = 0.5f * (prof[o + 1] + prof[o]);
        float cc1 = (float)((double)(fe - fs) / (double)nn);
        float cc2 = -cc1 + fs;
        int run = (a - a0) * ir + kk; /* 0-based child index along the edge */
        size_t cc = vert ? (size_t)run * Pc + fixed : (size_t)fixed * Pc + run;
        float val = 2.0f * (float)kk * cc1 + cc2;
        if (C.h[cc] + C.z1[cc] <= CC_GX) val = 0.0f;
        if (vert) C.m1w[cc] = val;
        else C.n1w[cc] = val;
    }
}

/* one value of JNQ's edge interpolation at its first sub-step
 * (EDGEINTERP_VERT / _HORI, all_grids.f90:502-604, on the parent's level-1
 * flux as JNQ passes it, all_grids.f90:484-487): the child edge node `run`
 * (1-based along the edge) of side `side` (0 left M, 1 right M, 2 bottom N,
 * 3 top N), zero where the child is dry.  The arithmetic of k_edges, node
 * by node. */
__device__ __forceinline__ float jnq_node(const GcLayerDev &Pl, const GcLayerDev &C, int side, int run, int ir,
                                          int is, int ie, int js, int je) {
    const bool vert = side < 2;
    const int sd = side & 1;
    const int line = vert ? (sd == 0 ? is - 1 : ie) : (sd == 0 ? js - 1 : je);
    const int a0 = vert ? js : is;
    const int a = a0 + (run - 1) / ir, kk = (run - 1) % ir + 1;
    const int Pp = Pl.pitch;
    auto prof = [&](int b) {
        const int I = vert ? line : b, J = vert ? b : line;
        const size_t c = (size_t)(J - 1) * Pp + (I - 1);
        return vert ? Pl.m1[c] : Pl.n1[c];
    };
    const float pm = prof(a - 1), p0 = prof(a), pp = prof(a + 1);
    const float fs = 0.5f * (pm + p0);
    const float fe = 0.5f * (pp + p0);
    const float cc1 = (float)((double)(fe - fs) / (double)(2 * ir));
    const float cc2 = -cc1 + fs;
    const int fixed = vert ? (sd == 0 ? 0 : C.nx - 1) : (sd == 0 ? 0 : C.ny - 1);
    const size_t cc = vert ? (size_t)run * C.pitch + fixed : (size_t)fixed * C.pitch + run;
    float val = 2.0f * (float)kk * cc1 + cc2;
    if (C.h[cc] + C.z1[cc] <= CC_GX) val = 0.0f;
    return val;
}

/* CONMASS / MASS_C of one child cell from its fluxes (mass.f90:103-160) */
template <bool NONLIN>
__device__ __forceinline__ void mass_c_store(const GcLayerDev &L, size_t c, float z1, float m_c, float m_w,
                                             float n_c, float n_s, float h) {
    float zz = z1 - L.rx * (m_c - m_w) - L.ry * (n_c - n_s);
    if (fabsf(zz) < CC_EPS) zz = 0.0f;
    if (!NONLIN) {
        float out;
        if (h > CC_GX) {
            if ((zz + h) <= CC_EPS) zz = -h;
            out = zz;
        } else {
            out = 0.0f;
        }
        L.z2[c] = out;
    } else {
        float dz, z;
        if (h > CC_ELMAX) {
            float dd = zz + h;
            if (dd >= CC_GX) { dz = dd; z = zz; }
            else { dz = 0.0f; z = -h; }
        } else {
            dz = 0.0f; z = -h;
        }
        L.dz2[c] = dz;
        L.z2[c] = z;
    }
}

/* a child cell on or next to the child's edge: JNQ's stores (M on columns 0
 * and nx-1, rows 1..ny-1; N on rows 0 and ny-1, columns 1..nx-1), then its
 * mass with the edge fluxes it reads computed in place */
template <bool NONLIN>
__device__ __forceinline__ void mass_c_jnq_edge(const GcLayerDev &Pl, const GcLayerDev &L, int i, int j, int ir, int is,
                                             int ie, int js, int je) {
    const int nx = L.nx, ny = L.ny;
    const size_t c = (size_t)j * L.pitch + i;
    if ((i == 0 || i == nx - 1) && j >= 1) L.m1w[c] = jnq_node(Pl, L, i == 0 ? 0 : 1, j, ir, is, ie, js, je);
    if ((j == 0 || j == ny - 1) && i >= 1) L.n1w[c] = jnq_node(Pl, L, j == 0 ? 2 : 3, i, ir, is, ie, js, je);
    if (i == 0 || j == 0) {
        L.z2[c] = L.z1[c];
        return;
    }
    const float m_c = (i == nx - 1) ? jnq_node(Pl, L, 1, j, ir, is, ie, js, je) : L.m1[c];
    const float m_w = (i == 1) ? jnq_node(Pl, L, 0, j, ir, is, ie, js, je) : L.m1[c - 1];
    const float n_c = (j == ny - 1) ? jnq_node(Pl, L, 3, i, ir, is, ie, js, je) : L.n1[c];
    const float n_s = (j == 1) ? jnq_node(Pl, L, 2, i, ir, is, ie, js, je) : L.n1[c - L.pitch];
    mass_c_store<NONLIN>(L, c, L.z1[c], m_c, m_w, n_c, n_s, L.h[c]);
}

/* A child's first sub-step of JNQ and its mass (MASS_C / CONMASS) in one
 * launch, one cell per thread.  The threads on the child's edges store
 * JNQ's fluxes there (for the momentum that follows); a cell next to an
 * edge computes the edge value it reads itself, by the same arithmetic,
 * instead of waiting for the store.  Same values as k_edges then k_mass_c. */
template <bool NONLIN>
__global__ void k_mass_c_jnq(GcLayerDev Pl, GcLayerDev L, int ir, int is, int ie, int js, int je) {
    pdl_enter();
    const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    if (i >= L.nx || j >= L.ny) return;
    if (j >= 2 && j <= L.ny - 2 && i >= 2 && i <= L.nx - 2) {
        const size_t c = (size_t)j * L.pitch + i;
        mass_c_store<NONLIN>(L, c, L.z1[c], L.m1[c], L.m1[c - 1], L.n1[c], L.n1[c - L.pitch], L.h[c]);
    } else {
        mass_c_jnq_edge<NONLIN>(Pl, L, i, j, ir, is, ie, js, je);
    }
}

/* JNZ (all_grids.f90:342-421): mean of wet child surface over each r x r
 * block, summed in the Fortran order (KI outer, KJ inner). */
__global__ void k_jnz(GcLayerDev Pl, GcLayerDev C, int ir, int rel_time, int is, int ie, int js,
                      int je) {
    pdl_enter();
    int I = is + blockIdx.x * blockDim.x + threadIdx.x;
    int J = js + blockIdx.y;
    if (I > ie || J > je) return;
    const float half = (float)(ir * ir) / 2.0f;
    const bool even = (rel_time % 2) == 0;
    int i0 = (I - is) * ir; /* 0-based child index of KI = 1 is i0 */
    int j0 = (J - js) * ir;
    float sum = 0.0f, count = 0.0f;
    for (int ki = 1; ki <= ir; ki++) {
        for (int kj = 1; kj <= ir; kj++) {
            size_t c = (size_t)(j0 + kj) * C.pitch + (i0 + ki);
            float z2 = C.z2[c];
            if (C.h[c] + z2 > CC_GX) {
                if (even) sum = sum + 0.5f * (C.z1[c] + z2);
                else sum = sum + z2;
                count = count + 1.0f;
            }
        }
    }
    Pl.z2[(size_t)(J - 1) * Pl.pitch + (I - 1)] = (count > half) ? sum / count : 0.0f;
}

/* the same for a compile-time ratio R: the R x R block's surfaces and depths
 * are loaded as one batch of independent loads, then summed in the order
 * above (child I outermost) */
/* the JNZ surface of parent cell (I, J) (1-based, inside the window) for a
 * compile-time ratio R: the R x R block's surfaces and depths are loaded as
 * one batch of independent loads, then summed in the order above (child I
 * outermost) */
template <int R, bool EVEN>
__device__ __forceinline__ float jnz_value(const GcLayerDev &C, int is, int js, int I, int J) {
    const float half = (float)(R * R) / 2.0f;
    const int i0 = (I - is) * R, j0 = (J - js) * R;
    const float *__restrict__ z2p = C.z2;
    const float *__restrict__ z1p = C.z1;
    const float *__restrict__ hp = C.h;
    float z2[R][R], hh[R][R], z1[R][R];
#pragma unroll
    for (int ki = 0; ki < R; ki++)
#pragma unroll
        for (int kj = 0; kj < R; kj++) {
            const size_t c = (size_t)(j0 + 1 + kj) * C.pitch + (i0 + 1 + ki);
            z2[ki][kj] = __ldg(z2p + c);
            hh[ki][kj] = __ldg(hp + c);
            if (EVEN) z1[ki][kj] = __ldg(z1p + c);
        }
    float sum = 0.0f, count = 0.0f;
#pragma unroll
    for (int ki = 0; ki < R; ki++)
#pragma unroll
        for (int kj = 0; kj < R; kj++) {
            if (hh[ki][kj] + z2[ki][kj] > CC_GX) {
                if (EVEN) sum = sum + 0.5f * (z1[ki][kj] + z2[ki][kj]);
                else sum = sum + z2[ki][kj];
                count = count + 1.0f;
            }
        }
    return (count > half) ? sum / count : 0.0f;
}

template <int R, bool EVEN>
__global__ void k_jnz_r(GcLayerDev Pl, GcLayerDev C, int is, int ie, int js, int je) {
    pdl_enter();
    int I = is + blockIdx.x * blockDim.x + threadIdx.x;
    int J = js + blockIdx.y;
    if (I > ie || J > je) return;
    Pl.z2[(size_t)(J - 1) * Pl.pitch + (I - 1)] = jnz_value<R, EVEN>(C, is, js, I, J);
}

/* ---------------------------------------------------------------- */
/* outputs                                                           */
/* ---------------------------------------------------------------- */
__global__ void k_maxamp(GcLayerDev L) {
    pdl_enter();
    int i = blockIdx.x * BX + threadIdx.x;
    int j = blockIdx.y * BY + threadIdx.y;
    if (i >= L.nx || j >= L.ny) return;
    size_t c = (size_t)j * L.pitch + i;
    float z = L.z2[c], m = L.zmax[c];
    if (!(m >= z)) L.zmax[c] = z;
}

/* ---------------------------------------------------------------- */
/* SC_OPTION = 1 coupling (all_grids.f90:996-1425)                   */
/* ---------------------------------------------------------------- */
/* Z1+Z2+Z3+Z4 of the four weighted parent values (all_grids.f90:1030-1034) */
__device__ __forceinline__ float sc_bilin(const float *f, int pitch, int2 ps, float4 w) {
    const size_t c = (size_t)(ps.y - 1) * pitch + (ps.x - 1);
    float z1 = f[c] * w.x;
    float z2 = f[c + 1] * w.y;
    float z3 = f[c + pitch] * w.z;
    float z4 = f[c + pitch + 1] * w.w;
    return z1 + z2 + z3 + z4;
}

/* EDGE_INTERP_SC (t = 1) and the edge blend of NEWQ_SC (t >= 2,
 * all_grids.f90:1268-1362), one thread per child edge node.  The wet test
 * is at the edge node itself on the child's level-2 surface as the
 * reference holds it (zwet); EDGE_INTERP_SC's own test reads indices left
 * over from elsewhere, which no implementation can reproduce. */
__global__ void k_sc_edges(GcLayerDev P, GcLayerDev C, GcScView sv, int t, float c1, float c2, const float *zwet) {
    pdl_enter();
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int nx = C.nx, ny = C.ny;
    if (k >= 2 * ny + 2 * nx) return;
    int side, i, j;
    if (k < ny) { side = 0; i = 0; j = k; }
    else if (k < 2 * ny) { side = 1; i = nx - 1; j = k - ny; }
    else if (k < 2 * ny + nx) { side = 2; i = k - 2 * ny; j = 0; }
    else { side = 3; i = k - 2 * ny - nx; j = ny - 1; }
    const bool vert = side < 2;
    const size_t cc = (size_t)j * C.pitch + i;
    float v = 0.0f;
    if (C.h[cc] + zwet[cc] > CC_GX) {
        const int2 ps = sv.epos[k];
        const float4 w = sv.ew[k];
        const float x1 = sc_bilin(vert ? P.m1 : P.n1, P.pitch, ps, w);
        if (t == 1) {
            v = x1;
        } else {
            const float x2 = sc_bilin(vert ? P.m2 : P.n2, P.pitch, ps, w);
            /* the reference's top edge weights YN1 by C1 (all_grids.f90:1357) */
            const float w1 = (side == 3 && !sv.fix_top) ? c1 : c2;
            v = c1 * x2 + w1 * x1;
        }
    }
    if (vert) C.m1w[cc] = v;
    else C.n1w[cc] = v;
}

/* NEWQ_SC forecast of the parent fluxes at the end of its step on four
 * bands around the child (all_grids.f90:1130-1266), into the parent's
 * level 2, which its own momentum step overwrites afterwards */
__global__ void k_sc_forecast(GcLayerDev P, GcScView sv) {
    pdl_enter();
    const int b = blockIdx.z;
    const int i = sv.band[b][0] + blockIdx.x * BX + threadIdx.x;
    const int j = sv.band[b][2] + blockIdx.y * BY + threadIdx.y;
    if (i > sv.band[b][1] || j > sv.band[b][3]) return;
    const int Pp = P.pitch;
    const size_t c = (size_t)j * Pp + i;
    const float twlvth = 0.08333333333333f;
    if (b < 2) {
        const size_t cp = c + 1;
        float out = 0.0f;
        if (P.h[c] > CC_GX && P.h[cp] > CC_GX) {
            const int jm1 = j - 1 < 0 ? 0 : j - 1, jp1 = j + 1 > P.ny - 1 ? P.ny - 1 : j + 1;
            const size_t cm = (size_t)jm1 * Pp + i, cq = (size_t)jp1 * Pp + i;
            const float tot_n = P.n1[c] + P.n1[cp] + P.n1[cm] + P.n1[cm + 1];
            const float r2 = r2_at(P, i, j, c, P.h[c], P.h[cp]);
            float xm = P.m1[c] - r2 * (P.z2[cp] - P.z2[c]) + GC_ROW(P, GC_R3, j) * tot_n;
            if (sv.modscm == 0) {
                const float scm = r2 * twlvth * ((P.z2[cq + 1] - 2.0f * P.z2[cp] + P.z2[cm + 1]) -
                                                 (P.z2[cq] - 2.0f * P.z2[c] + P.z2[cm]));
                xm = xm - scm;
            }
            if (fabsf(xm) < CC_EPS) xm = 0.0f;
            out = xm;
        }
        P.m2[c] = out;
    } else {
        const size_t cq = c + Pp;
        float out = 0.0f;
        if (P.h[c] > CC_GX && P.h[cq] > CC_GX) {
            const size_t cw = (size_t)j * Pp + (i - 1 < 0 ? 0 : i - 1);
            const size_t ce = (size_t)j * Pp + (i + 1 > P.nx - 1 ? P.nx - 1 : i + 1);
            const float tot_m = P.m1[cw] + P.m1[cw + Pp] + P.m1[c] + P.m1[cq];
            const float r4 = r4_at(P, i, j, c, P.h[c], P.h[cq]);
            float xn = P.n1[c] - r4 * (P.z2[cq] - P.z2[c]) - GC_ROW(P, GC_R5, j) * tot_m;
            if (sv.modscm == 0) {
                const float scm = r4 * twlvth * ((P.z2[ce + Pp] - 2.0f * P.z2[cq] + P.z2[cw + Pp]) -
                                                 (P.z2[ce] - 2.0f * P.z2[c] + P.z2[cw]));
                xn = xn - scm;
            }
            if (fabsf(xn) < CC_EPS) xn = 0.0f;
            out = xn;
        }
        P.n2[c] = out;
    }
}

/* JNZ_SC (all_grids.f90:1367-1425) as a gather: each parent cell of the
 * window sums the wet child surfaces that fall in it, in the reference's
 * order, and takes their mean where more than half of r*r nodes
 * contributed (elsewhere it keeps its value) */
__global__ void k_sc_jnz(GcLayerDev P, GcLayerDev C, GcScView sv) {
    pdl_enter();
    const int i = sv.wi0 + blockIdx.x * BX + threadIdx.x;
    const int j = sv.wj0 + blockIdx.y * BY + threadIdx.y;
    if (i > sv.wi1 || j > sv.wj1) return;
    const int q = (j - sv.wj0) * (sv.wi1 - sv.wi0 + 1) + (i - sv.wi0);
    float sum = 0.0f, cnt = 0.0f;
    for (int k = sv.start[q]; k < sv.start[q + 1]; k++) {
        const int cc = sv.cell[k];
        if (C.h[cc] + C.z2[cc] > CC_GX) {
            sum = sum + C.z2[cc];
            cnt = cnt + 1.0f;
        }
    }
    if (cnt > sv.half) P.z2[(size_t)j * P.pitch + i] = sum / cnt;
}

/* SPONGE_LAYER (boundaries.f90:229-244) with separable coefficients,
 * COEFX(I,J) = spx[I] and COEFY(I,J) = spy[J]: where either is positive,
 * M2 += CX*DT*M1 and N2 += CY*DT*N1 */
__global__ void k_sponge(GcLayerDev L, const float *__restrict__ spx, const float *__restrict__ spy, float dt) {
    pdl_enter();
    int i = blockIdx.x * BX + threadIdx.x;
    int j = blockIdx.y * BY + threadIdx.y;
    if (i >= L.nx || j >= L.ny) return;
    const float cx = spx[i], cy = spy[j];
    if (cx > 0.0f || cy > 0.0f) {
        size_t c = (size_t)j * L.pitch + i;
        L.m2[c] = L.m2[c] + cx * dt * L.m1[c];
        L.n2[c] = L.n2[c] + cy * dt * L.n1[c];
    }
}

/* arrival at the start of tracking: step 0 on a wet cell whose surface is
 * already above the threshold, -1 (not yet) elsewhere */
__global__ void k_arrival_start(int *arrival, const float *z, const float *h, int nx, int ny, int pitch,
                                float thr) {
    pdl_enter();
    int i = blockIdx.x * BX + threadIdx.x;
    int j = blockIdx.y * BY + threadIdx.y;
    if (i >= nx || j >= ny) return;
    size_t c = (size_t)j * pitch + i;
    arrival[c] = (h[c] > CC_GX && z[c] > thr) ? 0 : -1;
}

__global__ void k_arrival(GcLayerDev L, int step, float thr) {
    pdl_enter();
    int i = blockIdx.x * BX + threadIdx.x;
    int j = blockIdx.y * BY + threadIdx.y;
    if (i >= L.nx || j >= L.ny) return;
    size_t c = (size_t)j * L.pitch + i;
    if (L.arrival[c] < 0 && L.h[c] > CC_GX && L.z2[c] > thr) L.arrival[c] = step;
}

/* gauge stencil: for each (ki,kj) 1-based, the four surface values the
 * reference's gcomcot_get_z_ returns (GPUOutput.cu:29-44) */
__global__ void k_gauges(GcLayerDev L, int ng, const int *ij, float *out) {
    pdl_enter();
    int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ng) return;
    int i = ij[2 * g] - 1, j = ij[2 * g + 1] - 1;
    size_t c = (size_t)j * L.pitch + i;
    out[4 * g + 0] = L.z2[c];
    out[4 * g + 1] = L.z2[c + 1];
    out[4 * g + 2] = L.z2[c + L.pitch];
    out[4 * g + 3] = L.z2[c + L.pitch + 1];
}

/* outputs of one finished outer step of a batched nested member: running
 * maximum and arrival step over the outer layer (L.z2 is the new surface)
 * and the step's gauge samples (GET_TS bilinear weights, output.f90:1078-1090)
 * from the outer layer or the child (cz, pitch cpitch).  The step number is
 * step_off + *step_base (step_base may be NULL), so a replayed graph numbers
 * the steps correctly; step - step0 is the member's 0-based step index. */
__global__ void k_step_outputs(GcLayerDev L, const int *step_base, int step_off, int step0, int flags,
                               float thr, int ng, const int *gij, const float *gw, const int *glayer,
                               const float *cz, int cpitch, float *ts, int ts_len, int wi0, int wj0, int wni,
                               int wnj) {
    pdl_enter();
    const int local = step_off + (step_base ? *step_base : 0) - step0;
    if (local < 0 || local >= ts_len) return;
    if (blockIdx.x == 0 && blockIdx.y == 0 && ng > 0) {
        for (int g = threadIdx.y * BX + threadIdx.x; g < ng; g += BX * BY) {
            const bool child = glayer && glayer[g] != 0;
            const float *z = child ? cz : L.z2;
            const size_t P = child ? (size_t)cpitch : (size_t)L.pitch;
            size_t c = (size_t)(gij[2 * g + 1] - 1) * P + (size_t)(gij[2 * g] - 1);
            float l1 = z[c], l2 = z[c + 1], l3 = z[c + P], l4 = z[c + P + 1];
            float cx = gw[2 * g], cy = gw[2 * g + 1];
            float a = l1 * (1.0f - cx) * (1.0f - cy);
            float b = l2 * (cx) * (1.0f - cy);
            float d = l3 * (1.0f - cx) * (cy);
            float e = l4 * (cx) * (cy);
            ts[(size_t)local * ng + g] = a + b + d + e;
        }
    }
    int i = wi0 + blockIdx.x * BX + threadIdx.x;
    int j = wj0 + blockIdx.y * BY + threadIdx.y;
    if (i >= wi0 + wni || j >= wj0 + wnj || i >= L.nx || j >= L.ny) return;
    size_t c = (size_t)j * L.pitch + i;
    float z = L.z2[c];
    if (flags & 1) {
        float m = L.zmax[c];
        if (!(m >= z)) L.zmax[c] = z;
    }
    if ((flags & 2) && L.arrival[c] < 0 && L.h[c] > CC_GX && z > thr) L.arrival[c] = local + 1;
}

/* The end of a nested outer step whose child takes one sub-step, as one
 * launch: JNZ's feedback (all_grids.f90:378-411), the outer momentum
 * recomputed where that surface changed, and the step's outputs on the
 * window.  Same values as k_jnz_r, k_momt_s over the rectangle and
 * k_step_outputs in turn.
 *
 * A block owns a 31 x 7 patch of the momentum rectangle (0-based columns
 * ri0 .. ri0+rni-1, rows rj0 .. rj0+rnj-1) and first takes the level-2
 * surface of the 32 x 8 cells from the patch's corner: JNZ's mean inside
 * the window (1-based IS..IE x JS..JE), the stored surface outside it,
 * which nothing in this launch writes.  A patch cell's M reads its east
 * neighbour and its N its north neighbour, both in that 32 x 8 block.
 * Gauges on the outer layer take a window cell's surface the same way,
 * since another block writes it. */
template <int R, bool EVEN>
__device__ __forceinline__ float feedback_z(const GcLayerDev &P, const GcLayerDev &C, int is, int ie, int js,
                                            int je, int i, int j) {
    const int I = i + 1, J = j + 1;
    if (I >= is && I <= ie && J >= js && J <= je) return jnz_value<R, EVEN>(C, is, js, I, J);
    return P.z2[(size_t)j * P.pitch + i];
}

constexpr int FB_W = BX - 1, FB_H = BY - 1; /* a block's patch of the momentum rectangle */

template <int R, bool EVEN>
__global__ void __launch_bounds__(BX * BY) k_feedback_r(GcLayerDev L, GcLayerDev C, int is, int ie, int js, int je,
                                                        int ri0, int rj0, int rni, int rnj, const int *step_base,
                                                        int step_off, int step0, int flags, float thr, int ng,
                                                        const int *gij, const float *gw, const int *glayer,
                                                        const float *cz, int cpitch, float *ts, int ts_len) {
    pdl_enter();
    __shared__ float zt[BY][BX + 1];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int i = ri0 + blockIdx.x * FB_W + tx, j = rj0 + blockIdx.y * FB_H + ty;
    const int P = L.pitch;
    float z = 0.0f;
    if (i < L.nx && j < L.ny) z = feedback_z<R, EVEN>(L, C, is, ie, js, je, i, j);
    zt[ty][tx] = z;
    __syncthreads();
    const int local = step_off + (step_base ? *step_base : 0) - step0;
    const bool outputs = local >= 0 && local < ts_len;
    if (tx < FB_W && ty < FB_H && i < ri0 + rni && j < rj0 + rnj && i < L.nx && j < L.ny) {
        const size_t c = (size_t)j * P + i;
        const int I = i + 1, J = j + 1;
        const bool win = I >= is && I <= ie && J >= js && J <= je;
        if (win) L.z2[c] = z;
        /* k_momt_s with the surface from the block's copy */
        const int lo = L.root ? 0 : 1;
        float xm = 0.0f;
        if (i >= lo && i <= L.nx - 2 && j >= lo) {
            float h = L.h[c], hp1 = L.h[c + 1];
            if (h > CC_GX && hp1 > CC_GX) {
                size_t cm = (j > 0) ? c - P : c; /* JM1 = max(J-1,1) */
                float tot_n = L.n1[c] + L.n1[c + 1] + L.n1[cm] + L.n1[cm + 1];
                xm = L.m1[c] - r2_at(L, i, j, c, h, hp1) * (zt[ty][tx + 1] - z) + GC_ROW(L, GC_R3, j) * tot_n;
                if (fabsf(xm) < CC_EPS) xm = 0.0f;
            }
        }
        L.m2[c] = xm;
        float xn = 0.0f;
        if (j >= lo && j <= L.ny - 2 && i >= lo) {
            float h = L.h[c], hq1 = L.h[c + P];
            if (h > CC_GX && hq1 > CC_GX) {
                size_t cw = (i > 0) ? c - 1 : c; /* IM1 = max(I-1,1) */
                float tot_m = L.m1[cw] + L.m1[cw + P] + L.m1[c] + L.m1[c + P];
                xn = L.n1[c] - r4_at(L, i, j, c, h, hq1) * (zt[ty + 1][tx] - z) - GC_ROW(L, GC_R5, j) * tot_m;
                if (fabsf(xn) < CC_EPS) xn = 0.0f;
            }
        }
        L.n2[c] = xn;
        /* k_step_outputs on the window */
        if (win && outputs) {
            if (flags & 1) {
                float m = L.zmax[c];
                if (!(m >= z)) L.zmax[c] = z;
            }
            if ((flags & 2) && L.arrival[c] < 0 && L.h[c] > CC_GX && z > thr) L.arrival[c] = local + 1;
        }
    }
    if (blockIdx.x == 0 && blockIdx.y == 0 && ng > 0 && outputs) {
        for (int g = ty * BX + tx; g < ng; g += BX * BY) {
            const bool child = glayer && glayer[g] != 0;
            const int gi = gij[2 * g] - 1, gj = gij[2 * g + 1] - 1;
            float l1, l2, l3, l4;
            if (child) {
                const size_t cc = (size_t)gj * cpitch + gi;
                l1 = cz[cc]; l2 = cz[cc + 1]; l3 = cz[cc + cpitch]; l4 = cz[cc + cpitch + 1];
            } else {
                l1 = feedback_z<R, EVEN>(L, C, is, ie, js, je, gi, gj);
                l2 = feedback_z<R, EVEN>(L, C, is, ie, js, je, gi + 1, gj);
                l3 = feedback_z<R, EVEN>(L, C, is, ie, js, je, gi, gj + 1);
                l4 = feedback_z<R, EVEN>(L, C, is, ie, js, je, gi + 1, gj + 1);
            }
            float cx = gw[2 * g], cy = gw[2 * g + 1];
            float a = l1 * (1.0f - cx) * (1.0f - cy);
            float b = l2 * (cx) * (1.0f - cy);
            float d = l3 * (1.0f - cx) * (cy);
            float e = l4 * (cx) * (cy);
            ts[(size_t)local * ng + g] = a + b + d + e;
        }
    }
}

thread_local bool t_pdl = false;

/* ordinary launch, or one with programmatic stream serialization */
template <typename... KArgs, typename... Args>
void launch(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args &&...args) {
    if (!t_pdl) {
        kern<<<grid, block, smem, s>>>(std::forward<Args>(args)...);
        return;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

inline dim3 grid2(const GcLayerDev &L) {
    return dim3((unsigned)((L.nx + BX - 1) / BX), (unsigned)((L.ny + BY - 1) / BY), 1);
}

} // namespace

void gc_launch_mass(const GcLayerDev &L, cudaStream_t s) {
    if (L.laygov == 2 || L.laygov == 3) {
        if (L.laycord == 0) launch(k_mass_d<true>, grid2(L), dim3(BX, BY), 0, s, L);
        else launch(k_mass_d<false>, grid2(L), dim3(BX, BY), 0, s, L);
    } else if (L.laycord == 0 && L.laygov == 1) launch(k_mass_s<true>, grid2(L), dim3(BX, BY), 0, s, L);
    else if (L.laycord == 0) launch(k_mass_s<false>, grid2(L), dim3(BX, BY), 0, s, L);
    else if (L.laygov == 1) launch(k_mass_c<true>, grid2(L), dim3(BX, BY), 0, s, L);
    else launch(k_mass_c<false>, grid2(L), dim3(BX, BY), 0, s, L);
}

/* CONMOME: the shared-memory tile form (both faces per thread) in blocks of
 * 32 x 4 cells at 64 registers, eight blocks to an SM.  A 601 x 501 child
 * takes 2.02 waves of them, the last 26 blocks short ones, against 2.7 waves
 * of 32 x 8 blocks, which the compiler gives 72 registers (three to an SM).
 * GCOMCOT_CONMOME_TILE=8 takes the 32 x 8 blocks, GCOMCOT_CONMOME_TILE=0 the
 * one-face form (x and y as two grid layers).  All compute the same bits. */
static int conmome_rows() {
    static const int rows = [] {
        const char *v = getenv("GCOMCOT_CONMOME_TILE");
        if (v && v[0] == '0') return 0;
        return (v && atoi(v) == 8) ? 8 : 4;
    }();
    return rows;
}

static void launch_conmome(const GcLayerDev &L, int upd, cudaStream_t s) {
    const bool sph = L.laycord == 0;
    const int rows = conmome_rows();
    if (rows == 4) {
        const dim3 g4((unsigned)((L.nx + BX - 1) / BX), (unsigned)((L.ny + 3) / 4), 1);
        if (sph) launch(k_conmome_tile<true, 4, 8>, g4, dim3(BX, 4), 0, s, L, upd);
        else launch(k_conmome_tile<false, 4, 8>, g4, dim3(BX, 4), 0, s, L, upd);
    } else if (rows == 8) {
        if (sph) launch(k_conmome_tile<true, 8, 1>, grid2(L), dim3(BX, 8), 0, s, L, upd);
        else launch(k_conmome_tile<false, 8, 1>, grid2(L), dim3(BX, 8), 0, s, L, upd);
    } else {
        const dim3 g2(grid2(L).x, grid2(L).y, 2);
        if (sph) launch(k_conmome<true>, g2, dim3(BX, BY), 0, s, L, upd);
        else launch(k_conmome<false>, g2, dim3(BX, BY), 0, s, L, upd);
    }
}

void gc_launch_moment(const GcLayerDev &L, cudaStream_t s) {
    if (L.laygov == 2 || L.laygov == 3) {
        if (L.laycord == 0) launch(k_momt_d<true>, grid2(L), dim3(BX, BY), 0, s, L);
        else launch(k_momt_d<false>, grid2(L), dim3(BX, BY), 0, s, L);
    } else if (L.laygov == 1) launch_conmome(L, 0, s);
    else if (L.laycord == 0) launch(k_momt_s, grid2(L), dim3(BX, BY), 0, s, L, 0, 0, L.nx, L.ny);
    else launch(k_momt_c, grid2(L), dim3(BX, BY), 0, s, L);
}

int gc_launch_moment_update(const GcLayerDev &L, cudaStream_t s) {
    if (L.laygov == 1 && !L.root && L.modscm != 0) {
        launch_conmome(L, 1, s);
        return 1;
    }
    gc_launch_moment(L, s);
    gc_launch_update_edges(L, s);
    return 2;
}

void gc_launch_momt_s_window(const GcLayerDev &L, int i0, int i1, int j0, int j1, cudaStream_t s) {
    i0 = i0 < 0 ? 0 : i0;
    j0 = j0 < 0 ? 0 : j0;
    i1 = i1 > L.nx - 1 ? L.nx - 1 : i1;
    j1 = j1 > L.ny - 1 ? L.ny - 1 : j1;
    if (i1 < i0 || j1 < j0) return;
    const int ni = i1 - i0 + 1, nj = j1 - j0 + 1;
    dim3 grid((unsigned)((ni + BX - 1) / BX), (unsigned)((nj + BY - 1) / BY), 1);
    launch(k_momt_s, grid, dim3(BX, BY), 0, s, L, i0, j0, ni, nj);
}

void gc_launch_open(const GcLayerDev &L, cudaStream_t s) {
    int n = 2 * L.nx + 2 * (L.ny - 2);
    launch(k_open, (n + 127) / 128, 128, 0, s, L);
}

void gc_launch_update_edges(const GcLayerDev &L, cudaStream_t s) {
    int n = L.ny + L.nx - 1;
    launch(k_update_edges, (n + 127) / 128, 128, 0, s, L);
}

void gc_launch_edges(const GcLayerDev &P, const GcLayerDev &C, int rel_size, int rel_time,
                     const int *corners, int t, cudaStream_t s) {
    int is = corners[0], ie = corners[1], js = corners[2], je = corners[3];
    int len = (ie - is + 5) > (je - js + 5) ? (ie - is + 5) : (je - js + 5);
    size_t smem = (size_t)len * sizeof(float);
    launch(k_edges, 4, EDGE_THREADS, smem, s, P, C, rel_size, rel_time, is, ie, js, je, t, len);
}

bool gc_launch_edges_mass(const GcLayerDev &P, const GcLayerDev &C, int rel_size, int rel_time,
                          const int *corners, int t, cudaStream_t s) {
    if (t != 1 || C.root || C.laycord != 1 || (C.laygov != 0 && C.laygov != 1)) return false;
    const int is = corners[0], ie = corners[1], js = corners[2], je = corners[3];
    (void)rel_time;
    if (C.laygov == 1) launch(k_mass_c_jnq<true>, grid2(C), dim3(BX, BY), 0, s, P, C, rel_size, is, ie, js, je);
    else launch(k_mass_c_jnq<false>, grid2(C), dim3(BX, BY), 0, s, P, C, rel_size, is, ie, js, je);
    return true;
}

void gc_launch_jnz(const GcLayerDev &P, const GcLayerDev &C, int rel_size, int rel_time,
                   const int *corners, cudaStream_t s) {
    int is = corners[0], ie = corners[1], js = corners[2], je = corners[3];
    dim3 grid((unsigned)((ie - is + 1 + 127) / 128), (unsigned)(je - js + 1), 1);
    const bool even = (rel_time % 2) == 0;
#define GC_JNZ_R(R)                                                                             \
    case R:                                                                                     \
        if (even) launch(k_jnz_r<R, true>, grid, 128, 0, s, P, C, is, ie, js, je);             \
        else launch(k_jnz_r<R, false>, grid, 128, 0, s, P, C, is, ie, js, je);                 \
        return;
    switch (rel_size) {
        GC_JNZ_R(2)
        GC_JNZ_R(3)
        GC_JNZ_R(4)
        GC_JNZ_R(5)
        default: break;
    }
#undef GC_JNZ_R
    launch(k_jnz, grid, 128, 0, s, P, C, rel_size, rel_time, is, ie, js, je);
}

void gc_launch_maxamp(const GcLayerDev &L, cudaStream_t s) {
    launch(k_maxamp, grid2(L), dim3(BX, BY), 0, s, L);
}

void gc_launch_sc_edges(const GcLayerDev &P, const GcLayerDev &C, const GcScView &sv, int t, int rel_time,
                        const float *zwet, cudaStream_t s) {
    const int n = 2 * C.ny + 2 * C.nx;
    const float c1 = ((float)t - 1.0f) / (float)rel_time;
    const float c2 = 1.0f - c1;
    launch(k_sc_edges, (n + 127) / 128, 128, 0, s, P, C, sv, t, c1, c2, zwet);
}

void gc_launch_sc_forecast(const GcLayerDev &P, const GcScView &sv, cudaStream_t s) {
    int wmax = 1, hmax = 1;
    for (int b = 0; b < 4; b++) {
        wmax = std::max(wmax, sv.band[b][1] - sv.band[b][0] + 1);
        hmax = std::max(hmax, sv.band[b][3] - sv.band[b][2] + 1);
    }
    dim3 grid((unsigned)((wmax + BX - 1) / BX), (unsigned)((hmax + BY - 1) / BY), 4);
    launch(k_sc_forecast, grid, dim3(BX, BY), 0, s, P, sv);
}

void gc_launch_sc_jnz(const GcLayerDev &P, const GcLayerDev &C, const GcScView &sv, cudaStream_t s) {
    dim3 grid((unsigned)((sv.wi1 - sv.wi0 + 1 + BX - 1) / BX), (unsigned)((sv.wj1 - sv.wj0 + 1 + BY - 1) / BY), 1);
    launch(k_sc_jnz, grid, dim3(BX, BY), 0, s, P, C, sv);
}

void gc_launch_sponge(const GcLayerDev &L, const float *spx, const float *spy, float dt, cudaStream_t s) {
    launch(k_sponge, grid2(L), dim3(BX, BY), 0, s, L, spx, spy, dt);
}

void gc_launch_arrival_start(int *arrival, const float *z, const float *h, int nx, int ny, int pitch, float thr,
                             cudaStream_t s) {
    dim3 grid((unsigned)((nx + BX - 1) / BX), (unsigned)((ny + BY - 1) / BY), 1);
    launch(k_arrival_start, grid, dim3(BX, BY), 0, s, arrival, z, h, nx, ny, pitch, thr);
}

void gc_launch_arrival(const GcLayerDev &L, int step, float thr, cudaStream_t s) {
    launch(k_arrival, grid2(L), dim3(BX, BY), 0, s, L, step, thr);
}

void gc_launch_gauges(const GcLayerDev &L, int ng, const int *d_ij, float *d_out, cudaStream_t s) {
    if (ng <= 0) return;
    launch(k_gauges, (ng + 127) / 128, 128, 0, s, L, ng, d_ij, d_out);
}

void gc_launch_step_outputs(const GcLayerDev &L, const int *step_base, int step_off, int step0, int flags,
                            float thr, int ng, const int *gij, const float *gw, const int *glayer,
                            const float *cz, int cpitch, float *ts, int ts_len, const int *win, cudaStream_t s) {
    int i0 = 0, j0 = 0, ni = L.nx, nj = L.ny;
    if (win) { i0 = win[0]; ni = win[1] - win[0] + 1; j0 = win[2]; nj = win[3] - win[2] + 1; }
    dim3 grid((unsigned)((ni + BX - 1) / BX), (unsigned)((nj + BY - 1) / BY), 1);
    launch(k_step_outputs, grid, dim3(BX, BY), 0, s, L, step_base, step_off, step0, flags, thr, ng, gij, gw, glayer,
                                                 cz, cpitch, ts, ts_len, i0, j0, ni, nj);
}

bool gc_launch_feedback(const GcLayerDev &P, const GcLayerDev &C, int rel_size, int rel_time, const int *corners,
                        const int *rect, const int *step_base, int step_off, int step0, int flags, float thr, int ng,
                        const int *gij, const float *gw, const int *glayer, const float *cz, int cpitch, float *ts,
                        int ts_len, cudaStream_t s) {
    const int is = corners[0], ie = corners[1], js = corners[2], je = corners[3];
    const int i0 = std::max(rect[0], 0), i1 = std::min(rect[1], P.nx - 1);
    const int j0 = std::max(rect[2], 0), j1 = std::min(rect[3], P.ny - 1);
    if (i1 < i0 || j1 < j0) return false;
    const int ni = i1 - i0 + 1, nj = j1 - j0 + 1;
    const dim3 grid((unsigned)((ni + FB_W - 1) / FB_W), (unsigned)((nj + FB_H - 1) / FB_H), 1);
    const bool even = (rel_time % 2) == 0;
#define GC_FB_R(R)                                                                                              \
    case R:                                                                                                     \
        if (even)                                                                                               \
            launch(k_feedback_r<R, true>, grid, dim3(BX, BY), 0, s, P, C, is, ie, js, je, i0, j0, ni, nj,       \
                   step_base, step_off, step0, flags, thr, ng, gij, gw, glayer, cz, cpitch, ts, ts_len);        \
        else                                                                                                    \
            launch(k_feedback_r<R, false>, grid, dim3(BX, BY), 0, s, P, C, is, ie, js, je, i0, j0, ni, nj,      \
                   step_base, step_off, step0, flags, thr, ng, gij, gw, glayer, cz, cpitch, ts, ts_len);        \
        return true;
    switch (rel_size) {
        GC_FB_R(2)
        GC_FB_R(3)
        GC_FB_R(4)
        GC_FB_R(5)
        default: break;
    }
#undef GC_FB_R
    return false;
}

void gc_set_pdl(bool on) { t_pdl = on; }
bool gc_pdl_on() { return t_pdl; }
