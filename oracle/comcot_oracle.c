/*
 * CPU oracle for the COMCOT time-stepping hot path -- TEST INFRASTRUCTURE.
 * Only tests/, __graft_entry__.smoke() and bench.py (cpu_baseline and the
 * --impl reference arm) load this library.  It restates, formula by formula,
 * the reference's Fortran solvers (file:line cited per routine).  Arithmetic is
 * REAL (float by default, double in the FP64 twin), evaluated left to right as
 * gfortran does, with no contraction (-ffp-contract=off).  Loop nests run with
 * J outermost for memory locality; no routine reads a value it writes in the
 * same sweep, so the nesting order does not change any result.
 *
 * Where the reference's live GPU path and its Fortran differ, this file follows
 * the Fortran, except for the maximum-amplitude recorder, whose only live code
 * is the GPU kernel (the Fortran recorder is commented out, output.f90:876-885).
 */
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#include "comcot_oracle.h"
#include "oracle_consts.h"
#include "comcot_math.h"

#define R(x) ((REAL)(x))
#define IDX(L, i, j) ((size_t)((j) - 1) * (size_t)(L)->nx + (size_t)((i) - 1))
#define MAX(a, b) ((a) > (b) ? (a) : (b))
#define MIN(a, b) ((a) < (b) ? (a) : (b))

/* elementary functions: the deterministic versions the library also uses
 * (comcot_math.h) in float, libm in the FP64 twin.  Built with -DOCL_LIBM the
 * float build calls libm's expf/powf instead, an independent check that the
 * shared functions hide no error (tests/test_oracle_libm_cpu.py). */
#ifdef OCL_LIBM
#define O_EXPF(x) expf(x)
#define O_POWF(x, y) powf((x), (y))
#else
#define O_EXPF(x) cc_expf(x)
#define O_POWF(x, y) cc_powf((x), (y))
#endif
static inline REAL o_exp(REAL x) {
    if (sizeof(REAL) == sizeof(float)) return (REAL)O_EXPF((float)x);
    return (REAL)exp((double)x);
}
static inline REAL o_pow(REAL x, REAL y) {
    if (sizeof(REAL) == sizeof(float)) return (REAL)O_POWF((float)x, (float)y);
    return (REAL)pow((double)x, (double)y);
}
static inline REAL o_sqrt(REAL x) {
    if (sizeof(REAL) == sizeof(float)) return (REAL)sqrtf((float)x);
    return (REAL)sqrt((double)x);
}
static inline REAL o_abs(REAL x) { return x < R(0) ? -x : x; }

/* ------------------------------------------------------------------ */
/* a small pthread parallel-for over J; every cell is independent.     */
/* ------------------------------------------------------------------ */
static int g_threads = 1;
void ocl_set_threads(int n) { g_threads = n < 1 ? 1 : n; }
int ocl_get_threads(void) { return g_threads; }

typedef void (*rowfn)(void *ctx, int j0, int j1);
typedef struct { rowfn fn; void *ctx; int j0, j1; } par_job;
static void *par_tramp(void *a) {
    par_job *p = (par_job *)a;
    p->fn(p->ctx, p->j0, p->j1);
    return NULL;
}
/* runs fn over [lo, hi] inclusive */
static void par_rows(rowfn fn, void *ctx, int lo, int hi) {
    int n = hi - lo + 1;
    if (n <= 0) return;
    int t = g_threads;
    if (t > n) t = n;
    if (t <= 1 || n < 64) { fn(ctx, lo, hi); return; }
    pthread_t th[256];
    par_job jobs[256];
    if (t > 256) t = 256;
    int chunk = (n + t - 1) / t;
    int used = 0;
    for (int k = 0; k < t; k++) {
        int a = lo + k * chunk, b = MIN(hi, a + chunk - 1);
        if (a > b) break;
        jobs[k].fn = fn; jobs[k].ctx = ctx; jobs[k].j0 = a; jobs[k].j1 = b;
        if (pthread_create(&th[k], NULL, par_tramp, &jobs[k]) != 0) {
            fn(ctx, a, b);
            jobs[k].fn = NULL;
        }
        used++;
    }
    for (int k = 0; k < used; k++)
        if (jobs[k].fn) pthread_join(th[k], NULL);
}

/* ------------------------------------------------------------------ */
/* MASS_S  (mass.f90:61-100) linear continuity, spherical              */
/* ------------------------------------------------------------------ */
static void mass_s_rows(void *ctx, int js, int je) {
    ocl_layer *L = (ocl_layer *)ctx;
    int is = 2, ie = (L->id == 1) ? L->nx - 1 : L->nx;
    for (int j = js; j <= je; j++) {
        int jm1 = j - 1;
        for (int i = is; i <= ie; i++) {
            size_t c = IDX(L, i, j);
            REAL h = L->h[c];
            if (h > R(CC_GX)) {
                REAL zz = L->z1[c] - L->r1[j - 1] * (L->m1[c] - L->m1[IDX(L, i - 1, j)])
                          - L->r11[j - 1] * (L->n1[c] * L->r6[j - 1]
                                             - L->n1[IDX(L, i, jm1)] * L->r6[jm1 - 1]);
                if (o_abs(zz) < R(CC_EPS)) zz = R(0);
                if ((zz + h) <= R(CC_EPS)) zz = -h;
                L->z2[c] = zz;
            } else {
                L->z2[c] = R(0);
            }
        }
    }
}

/* MASS_C (mass.f90:103-157) linear continuity, Cartesian */
static void mass_c_rows(void *ctx, int js, int je) {
    ocl_layer *L = (ocl_layer *)ctx;
    REAL rx = R(L->rx), ry = R(L->ry);
    int is = 2, ie = (L->id == 1) ? L->nx - 1 : L->nx;
    for (int j = js; j <= je; j++) {
        for (int i = is; i <= ie; i++) {
            size_t c = IDX(L, i, j);
            REAL h = L->h[c];
            if (h > R(CC_GX)) {
                REAL zz = L->z1[c] - rx * (L->m1[c] - L->m1[IDX(L, i - 1, j)])
                          - ry * (L->n1[c] - L->n1[IDX(L, i, j - 1)]);
                if (o_abs(zz) < R(CC_EPS)) zz = R(0);
                if ((zz + h) <= R(CC_EPS)) zz = -h;
                L->z2[c] = zz;
            } else {
                L->z2[c] = R(0);
            }
        }
    }
}

/* CONMASS (mass.f90:162-224) nonlinear continuity with moving shoreline */
static void conmass_rows(void *ctx, int js, int je) {
    ocl_layer *L = (ocl_layer *)ctx;
    REAL rx = R(L->rx), ry = R(L->ry);
    int is = 2, ie = (L->id == 1) ? L->nx - 1 : L->nx;
    for (int j = js; j <= je; j++) {
        for (int i = is; i <= ie; i++) {
            size_t c = IDX(L, i, j);
            REAL h = L->h[c];
            if (h > R(CC_ELMAX)) {
                REAL zzz = L->z1[c] - rx * (L->m1[c] - L->m1[IDX(L, i - 1, j)])
                           - ry * (L->n1[c] - L->n1[IDX(L, i, j - 1)]);
                if (o_abs(zzz) < R(CC_EPS)) zzz = R(0);
                REAL dd = zzz + h;
                if (dd >= R(CC_GX)) {
                    L->dz2[c] = dd;
                    L->z2[c] = zzz;
                } else {
                    L->dz2[c] = R(0);
                    L->z2[c] = -h;
                }
            } else {
                L->dz2[c] = R(0);
                L->z2[c] = -h;
            }
        }
    }
}

/* CONMASS_S (mass.f90:226-278) nonlinear continuity, spherical, moving shoreline */
static void conmass_s_rows(void *ctx, int js, int je) {
    ocl_layer *L = (ocl_layer *)ctx;
    int is = 2, ie = (L->id == 1) ? L->nx - 1 : L->nx;
    for (int j = js; j <= je; j++) {
        int jm1 = j - 1;
        for (int i = is; i <= ie; i++) {
            size_t c = IDX(L, i, j);
            REAL h = L->h[c];
            if (h >= R(CC_ELMAX)) {
                REAL zz = L->z1[c] - L->r1[j - 1] * (L->m1[c] - L->m1[IDX(L, i - 1, j)])
                          - L->r11[j - 1] * (L->n1[c] * L->r6[j - 1]
                                             - L->n1[IDX(L, i, jm1)] * L->r6[jm1 - 1]);
                if (o_abs(zz) < R(CC_EPS)) zz = R(0);
                REAL dd = zz + h;
                if (dd >= R(CC_GX)) {
                    L->dz2[c] = dd;
                    L->z2[c] = zz;
                } else {
                    L->dz2[c] = R(0);
                    L->z2[c] = -h;
                }
            } else {
                L->dz2[c] = R(0);
                L->z2[c] = -h;
            }
        }
    }
}

/* MASS_S_D / MASS_C_D (dispersion.f90:239-356, 357-543) for LAYGOV 2 and 3.
 * ALPHA (dispersion.f90:36-165) clears the whole MASK inside its cell loop
 * (:125), so MASK ends up 0 everywhere and every cell takes the
 * non-dispersive branch (:333-337, :460-462): the linear continuity with the
 * land clamp ZZ+H <= ZERO (MASS_S / MASS_C use EPS). */
static void mass_d_rows(void *ctx, int js, int je) {
    ocl_layer *L = (ocl_layer *)ctx;
    REAL rx = R(L->rx), ry = R(L->ry);
    int is = 2, ie = (L->id == 1) ? L->nx - 1 : L->nx;
    for (int j = js; j <= je; j++) {
        int jm1 = MAX(j - 1, 1);
        for (int i = is; i <= ie; i++) {
            size_t c = IDX(L, i, j);
            REAL h = L->h[c];
            int im1 = MAX(i - 1, 1);
            if (h > R(CC_GX)) {
                REAL zz;
                if (L->laycord == 0)
                    zz = L->z1[c] - L->r1[j - 1] * (L->m1[c] - L->m1[IDX(L, im1, j)])
                         - L->r11[j - 1] * (L->n1[c] * L->r6[j - 1] - L->n1[IDX(L, i, jm1)] * L->r6[jm1 - 1]);
                else
                    zz = L->z1[c] - rx * (L->m1[c] - L->m1[IDX(L, im1, j)]) - ry * (L->n1[c] - L->n1[IDX(L, i, jm1)]);
                if (o_abs(zz) < R(CC_EPS)) zz = R(0);
                if ((zz + h) <= R(0)) zz = -h;
                L->z2[c] = zz;
            } else {
                L->z2[c] = R(0);
            }
        }
    }
}

void ocl_mass(ocl_layer *L) {
    /* dispatcher: mass.f90:18-52.  Edge rows: I=2.., J=2.. (mass.f90:70-78) */
    int je = (L->id == 1) ? L->ny - 1 : L->ny;
    if (L->laygov == 2 || L->laygov == 3) {
        par_rows(mass_d_rows, L, 2, je);
    } else if (L->laycord == 0) {
        if (L->laygov == 1) par_rows(conmass_s_rows, L, 2, je);
        else par_rows(mass_s_rows, L, 2, je);
    } else if (L->laygov == 1) {
        par_rows(conmass_rows, L, 2, je);
    } else {
        par_rows(mass_c_rows, L, 2, je);
    }
}

/* ------------------------------------------------------------------ */
/* MOMT_S (moment.f90:65-149) linear momentum with Coriolis, spherical */
/* ------------------------------------------------------------------ */
static void momt_s_rows(void *ctx, int js, int je) {
    ocl_layer *L = (ocl_layer *)ctx;
    int nx = L->nx, ny = L->ny;
    int is0 = (L->id == 1) ? 1 : 2, js0 = is0;
    for (int j = js; j <= je; j++) {
        /* x-momentum: I = IS..NX-1, J = JS..NY */
        if (j >= js0) {
            int jm1 = MAX(j - 1, 1);
            for (int i = is0; i <= nx - 1; i++) {
                size_t c = IDX(L, i, j), cp = IDX(L, i + 1, j);
                if (L->h[c] > R(CC_GX) && L->h[cp] > R(CC_GX)) {
                    REAL tot_n = L->n1[c] + L->n1[cp] + L->n1[IDX(L, i, jm1)]
                                 + L->n1[IDX(L, i + 1, jm1)];
                    REAL xm = L->m1[c] - L->r2[c] * (L->z2[cp] - L->z2[c])
                              + L->r3[j - 1] * tot_n;
                    if (o_abs(xm) < R(CC_EPS)) xm = R(0);
                    L->m2[c] = xm;
                } else {
                    L->m2[c] = R(0);
                }
            }
        }
        /* y-momentum: J = JS..NY-1, I = IS..NX */
        if (j >= js0 && j <= ny - 1) {
            int jp1 = j + 1;
            for (int i = is0; i <= nx; i++) {
                size_t c = IDX(L, i, j), cq = IDX(L, i, jp1);
                if (L->h[c] > R(CC_GX) && L->h[cq] > R(CC_GX)) {
                    int im1 = MAX(i - 1, 1);
                    REAL tot_m = L->m1[IDX(L, im1, j)] + L->m1[IDX(L, im1, jp1)]
                                 + L->m1[c] + L->m1[cq];
                    REAL xn = L->n1[c] - L->r4[c] * (L->z2[cq] - L->z2[c])
                              - L->r5[j - 1] * tot_m;
                    if (o_abs(xn) < R(CC_EPS)) xn = R(0);
                    L->n2[c] = xn;
                } else {
                    L->n2[c] = R(0);
                }
            }
        }
    }
}

/* MOMT_C (moment.f90:152-277) linear momentum, Cartesian, optional friction
 * and modified scheme */
static void momt_c_rows(void *ctx, int js, int je) {
    ocl_layer *L = (ocl_layer *)ctx;
    int nx = L->nx, ny = L->ny;
    int is0 = (L->id == 1) ? 1 : 2, js0 = is0;
    REAL konst = R(0.5) * R(L->dt) * R(CC_GRAV);
    REAL fm = R(L->fric_coef);
    REAL grx = R(L->grx), gry = R(L->gry);
    for (int j = js; j <= je; j++) {
        if (j >= js0) { /* M: I = IS..NX-1, J = JS..NY */
            int jm1 = MAX(j - 1, 1), jp1 = MIN(j + 1, ny);
            for (int i = is0; i <= nx - 1; i++) {
                int ip1 = i + 1;
                size_t c = IDX(L, i, j), cp = IDX(L, ip1, j);
                REAL xm;
                if (L->h[c] > R(CC_GX) && L->h[cp] > R(CC_GX)) {
                    REAL ff = R(0);
                    REAL hm = L->hp[c] + R(0.5) * (L->z2[c] + L->z2[cp]);
                    xm = L->m1[c] - grx * hm * (L->z2[cp] - L->z2[c]);
                    if (L->fric_switch != 1) {
                        REAL xqq = R(0.25) * (L->n1[c] + L->n1[cp] + L->n1[IDX(L, i, jm1)]
                                              + L->n1[IDX(L, ip1, jm1)]);
                        if (hm >= R(1.0e-3f))
                            ff = konst * fm * fm * o_sqrt(L->m1[c] * L->m1[c] + xqq * xqq)
                                 / o_pow(hm, R(CC_MANNEXP));
                        else
                            ff = R(0);
                        xm = xm - ff * L->m1[c];
                    }
                    if (L->modscm == 0) {
                        REAL scm = grx * R(CC_TWLVTH) * hm
                                   * ((L->z2[IDX(L, ip1, jp1)] - R(2) * L->z2[cp] + L->z2[IDX(L, ip1, jm1)])
                                      - (L->z2[IDX(L, i, jp1)] - R(2) * L->z2[c] + L->z2[IDX(L, i, jm1)]));
                        xm = xm - scm;
                    }
                    if (L->fric_switch != 1) xm = xm / (R(1) + ff);
                    if (o_abs(xm) < R(CC_EPS)) xm = R(0);
                } else {
                    xm = R(0);
                }
                L->m2[c] = xm;
            }
        }
        if (j >= js0 && j <= ny - 1) { /* N: J = JS..NY-1, I = IS..NX */
            int jp1 = j + 1;
            for (int i = is0; i <= nx; i++) {
                size_t c = IDX(L, i, j), cq = IDX(L, i, jp1);
                if (L->h[c] > R(CC_GX) && L->h[cq] > R(CC_GX)) {
                    int im1 = MAX(i - 1, 1), ip1 = MIN(i + 1, nx);
                    REAL ff = R(0);
                    REAL hn = L->hq[c] + R(0.5) * (L->z2[c] + L->z2[cq]);
                    REAL xn = L->n1[c] - gry * hn * (L->z2[cq] - L->z2[c]);
                    if (L->fric_switch != 1) {
                        REAL xpp = R(0.25) * (L->m1[c] + L->m1[cq] + L->m1[IDX(L, im1, j)]
                                              + L->m1[IDX(L, im1, jp1)]);
                        if (hn >= R(1.0e-5f))
                            ff = konst * fm * fm * o_sqrt(L->n1[c] * L->n1[c] + xpp * xpp)
                                 / o_pow(hn, R(CC_MANNEXP));
                        else
                            ff = R(0);
                        xn = xn - ff * L->n1[c];
                    }
                    if (L->modscm == 0) {
                        REAL scm = gry * R(CC_TWLVTH) * hn
                                   * ((L->z2[IDX(L, ip1, jp1)] - R(2) * L->z2[cq] + L->z2[IDX(L, im1, jp1)])
                                      - (L->z2[IDX(L, ip1, j)] - R(2) * L->z2[c] + L->z2[IDX(L, im1, j)]));
                        xn = xn - scm;
                    }
                    if (L->fric_switch != 1) xn = xn / (R(1) + ff);
                    if (o_abs(xn) < R(CC_EPS)) xn = R(0);
                    L->n2[c] = xn;
                } else {
                    L->n2[c] = R(0);
                }
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* CONMOME (moment.f90:280-780) + WAVE_BREAKING (moment.f90:1272-1384) */
/* ------------------------------------------------------------------ */
typedef struct { ocl_layer *L; REAL *dp1, *dp2, *dq1, *dq2; } conmome_ctx;

/* face depths DP, DQ (moment.f90:345-366); DZ(:,:,1) is never written by the
 * reference (only mass.f90:204-216 assign DZ(:,:,2)), so it is zero here. */
static void conmome_pre_rows(void *vctx, int js, int je) {
    conmome_ctx *x = (conmome_ctx *)vctx;
    ocl_layer *L = x->L;
    int ix = L->nx, jy = L->ny;
    for (int j = js; j <= je; j++) {
        int jp1 = MIN(j + 1, jy);
        for (int i = 1; i <= ix; i++) {
            int ip1 = MIN(i + 1, ix);
            size_t c = IDX(L, i, j);
            REAL d = L->dz2[c], dpx = L->dz2[IDX(L, ip1, j)], dqy = L->dz2[IDX(L, i, jp1)];
            REAL dp1 = R(0.25) * (d + R(0) + dpx + R(0));
            REAL dp2 = R(0.50) * (d + dpx);
            REAL dq1 = R(0.25) * (d + R(0) + dqy + R(0));
            REAL dq2 = R(0.50) * (d + dqy);
            if (dp1 < R(CC_GX)) dp1 = R(0);
            if (dp2 < R(CC_GX)) dp2 = R(0);
            if (dq1 < R(CC_GX)) dq1 = R(0);
            if (dq2 < R(CC_GX)) dq2 = R(0);
            x->dp1[c] = dp1; x->dp2[c] = dp2; x->dq1[c] = dq1; x->dq2[c] = dq2;
        }
    }
}

/* WAVE_BREAKING: damps the convection terms where the surface rises faster
 * than 0.08 sqrt(g d) (moment.f90:1300-1325) */
static inline void wave_breaking(ocl_layer *L, size_t c, REAL *advx, REAL *advy) {
    REAL cc = o_sqrt(R(CC_GRAV) * L->dz2[c]);
    REAL dzdt_f = R(CC_BRK_F) * cc;
    REAL dzdt_i = R(CC_BRK_I) * cc;
    REAL dzdt = o_abs(L->z2[c] - L->z1[c]) / R(L->dt);
    if (dzdt > dzdt_f) {
        REAL ref = (dzdt - dzdt_f) / (dzdt_i - dzdt_f);
        REAL coef = o_exp(-(R(1) * ref));
        *advx = coef * *advx;
        *advy = coef * *advy;
    }
}

static void conmome_x_rows(void *vctx, int js, int je) {
    conmome_ctx *x = (conmome_ctx *)vctx;
    ocl_layer *L = x->L;
    int ix = L->nx, jy = L->ny;
    int is = 2, ie = ix - 1;
    if (L->id == 1) is = 1;
    REAL rx = R(L->rx), ry = R(L->ry), grx = R(L->grx);
    REAL konst = (L->fric_switch != 1) ? R(0.5) * R(L->dt) * R(CC_GRAV) : R(0);
    REAL fm = R(L->fric_coef);
    int ispans = CC_SPAN, ispane = ix - CC_SPAN, jspans = CC_SPAN, jspane = jy - CC_SPAN;
    const REAL *dp1 = x->dp1, *dp2 = x->dp2, *dz = L->dz2, *z = L->z2, *hz = L->h;
    const REAL *p = L->m1, *q = L->n1;
    for (int j = js; j <= je; j++) {
        int jp1 = MIN(j + 1, jy), jm1 = MAX(j - 1, 1);
        for (int i = is; i <= ie; i++) {
            int ip1 = MIN(i + 1, ix), im1 = MAX(i - 1, 1);
            size_t c = IDX(L, i, j), cp = IDX(L, ip1, j);
            REAL dd = R(0), df = R(0), ff = R(0);
            int noflux = 0;
            if (hz[c] <= R(CC_ELMAX) || L->hp[c] <= R(CC_ELMAX)) {
                noflux = 1;
            } else {
                if (dz[c] > R(CC_GX) && dz[cp] > R(CC_GX)) {
                    dd = dp2[c]; df = dp1[c];
                } else if (dz[c] > R(CC_GX) && dz[cp] <= R(CC_GX) && hz[cp] + z[c] > R(CC_GX)) {
                    dd = R(0.5) * dz[c]; df = dd;
                } else if (dz[c] <= R(CC_GX) && dz[cp] > R(CC_GX) && hz[c] + z[cp] > R(CC_GX)) {
                    dd = R(0.5) * dz[cp]; df = dd;
                } else {
                    noflux = 1;
                }
                if (!noflux && dd < R(CC_GX)) noflux = 1;
            }
            if (noflux) { L->m2[c] = R(0); continue; }
            if (df < R(CC_DFMIN)) df = R(CC_DFMIN);
            REAL xqq = R(0.25) * (q[c] + q[cp] + q[IDX(L, i, jm1)] + q[IDX(L, ip1, jm1)]);
            if (L->fric_switch != 1)
                ff = konst * fm * fm * o_sqrt(p[c] * p[c] + xqq * xqq) / o_pow(df, R(CC_MANNEXP));
            else
                ff = R(0);
            REAL xp = p[c] - grx * dd * (z[cp] - z[c]);
            if (L->modscm == 0 && j < jy) {
                REAL scm = grx * dd / R(12)
                           * ((z[IDX(L, ip1, jp1)] - R(2) * z[cp] + z[IDX(L, ip1, jm1)])
                              - (z[IDX(L, i, jp1)] - R(2) * z[c] + z[IDX(L, i, jm1)]));
                xp = xp - scm;
            }
            if (L->fric_switch != 1) xp = xp - ff * p[c];
            if (L->linchk == 1 && dp1[c] >= R(CC_GX) && i > ispans && i < ispane && j > jspans
                && j < jspane) {
                REAL advx = R(0), advy = R(0);
                if (p[c] < R(0)) {
                    if (dp1[cp] < R(CC_GX) || dz[cp] < R(CC_GX))
                        advx = rx * (-(p[c] * p[c] / dp1[c]));
                    else
                        advx = rx * (p[cp] * p[cp] / dp1[cp] - p[c] * p[c] / dp1[c]);
                } else {
                    size_t cm = IDX(L, im1, j);
                    if (dp1[cm] < R(CC_GX) || dz[c] < R(CC_GX))
                        advx = rx * (p[c] * p[c] / dp1[c]);
                    else
                        advx = rx * (p[c] * p[c] / dp1[c] - p[cm] * p[cm] / dp1[cm]);
                }
                if (xqq < R(0)) {
                    size_t cj = IDX(L, i, jp1);
                    if (dz[cj] < R(CC_GX) || dz[IDX(L, ip1, jp1)] < R(CC_GX)) {
                        advy = ry * (-(p[c] * xqq / dp1[c]));
                    } else if (dp1[cj] < R(CC_GX)) {
                        advy = ry * (-(p[c] * xqq / dp1[c]));
                    } else {
                        REAL xqe = R(0.25) * (q[cj] + q[IDX(L, ip1, jp1)] + q[c] + q[cp]);
                        advy = ry * (p[cj] * xqe / dp1[cj] - p[c] * xqq / dp1[c]);
                    }
                } else {
                    size_t cj = IDX(L, i, jm1);
                    if (dz[cj] < R(CC_GX) || dz[IDX(L, ip1, jm1)] < R(CC_GX)) {
                        advy = ry * (p[c] * xqq / dp1[c]);
                    } else if (dp1[cj] < R(CC_GX)) {
                        advy = ry * (p[c] * xqq / dp1[c]);
                    } else {
                        REAL xqe = R(0.25) * (q[cj] + q[IDX(L, ip1, jm1)] + q[IDX(L, i, j - 2)]
                                              + q[IDX(L, ip1, j - 2)]);
                        advy = ry * (p[c] * xqq / dp1[c] - p[cj] * xqe / dp1[cj]);
                    }
                }
                wave_breaking(L, c, &advx, &advy);
                xp = xp - advx - advy;
            }
            if (L->fric_switch != 1) xp = xp / (R(1) + ff);
            if (o_abs(xp) < R(CC_EPS)) xp = R(0);
            REAL lim = R(CC_VLIMIT) * dd;
            if (xp > lim) xp = lim;
            if (xp < -lim) xp = -lim;
            L->m2[c] = xp;
        }
    }
}

static void conmome_y_rows(void *vctx, int js, int je) {
    conmome_ctx *x = (conmome_ctx *)vctx;
    ocl_layer *L = x->L;
    int ix = L->nx, jy = L->ny;
    int is = 2, ie = ix;
    if (L->id == 1) { is = 1; ie = ix - 1; }
    REAL rx = R(L->rx), ry = R(L->ry), gry = R(L->gry);
    REAL konst = (L->fric_switch != 1) ? R(0.5) * R(L->dt) * R(CC_GRAV) : R(0);
    REAL fm = R(L->fric_coef);
    int ispans = CC_SPAN, ispane = ix - CC_SPAN, jspans = CC_SPAN, jspane = jy - CC_SPAN;
    const REAL *dq1 = x->dq1, *dq2 = x->dq2, *dz = L->dz2, *z = L->z2, *hz = L->h;
    const REAL *p = L->m1, *q = L->n1;
    for (int j = js; j <= je; j++) {
        int jp1 = MIN(j + 1, jy), jm1 = MAX(j - 1, 1);
        for (int i = is; i <= ie; i++) {
            int ip1 = MIN(i + 1, ix), im1 = MAX(i - 1, 1);
            size_t c = IDX(L, i, j), cq = IDX(L, i, jp1);
            REAL dd = R(0), df = R(0), ff = R(0);
            int noflux = 0;
            if (hz[c] <= R(CC_ELMAX) || L->hq[c] <= R(CC_ELMAX)) {
                noflux = 1;
            } else {
                if (dz[c] > R(CC_GX) && dz[cq] > R(CC_GX)) {
                    dd = dq2[c]; df = dq1[c];
                } else if (dz[c] > R(CC_GX) && dz[cq] <= R(CC_GX) && hz[cq] + z[c] > R(CC_GX)) {
                    dd = R(0.5) * dz[c]; df = dd;
                } else if (dz[c] <= R(CC_GX) && dz[cq] > R(CC_GX) && hz[c] + z[cq] > R(CC_GX)) {
                    dd = R(0.5) * dz[cq]; df = dd;
                } else {
                    noflux = 1;
                }
                if (!noflux && dd < R(CC_GX)) noflux = 1;
            }
            if (noflux) { L->n2[c] = R(0); continue; }
            if (df < R(CC_DFMIN)) df = R(CC_DFMIN);
            REAL xpp = R(0.25) * (p[c] + p[cq] + p[IDX(L, im1, j)] + p[IDX(L, im1, jp1)]);
            if (L->fric_switch != 1)
                ff = konst * fm * fm * o_sqrt(q[c] * q[c] + xpp * xpp) / o_pow(df, R(CC_MANNEXP));
            else
                ff = R(0);
            REAL xq = q[c] - gry * dd * (z[cq] - z[c]);
            if (L->modscm == 0 && i < ix) {
                REAL scm = gry * dd / R(12)
                           * ((z[IDX(L, ip1, jp1)] - R(2) * z[cq] + z[IDX(L, im1, jp1)])
                              - (z[IDX(L, ip1, j)] - R(2) * z[c] + z[IDX(L, im1, j)]));
                xq = xq - scm;
            }
            /* moment.f90:672 subtracts the y friction from XP, not XQ; XP is
             * not used afterwards, so XQ only sees the 1/(1+FF) division. */
            if (L->linchk == 1 && dq1[c] >= R(CC_GX) && i > ispans && i < ispane && j > jspans
                && j < jspane) {
                REAL advx = R(0), advy = R(0);
                if (q[c] < R(0)) {
                    if (dq1[cq] < R(CC_GX) || dz[cq] < R(CC_GX))
                        advy = ry * (-(q[c] * q[c] / dq1[c]));
                    else
                        advy = ry * (q[cq] * q[cq] / dq1[cq] - q[c] * q[c] / dq1[c]);
                } else {
                    size_t cm = IDX(L, i, jm1);
                    if (dq1[cm] < R(CC_GX) || dz[c] < R(CC_GX))
                        advy = ry * (q[c] * q[c] / dq1[c]);
                    else
                        advy = ry * (q[c] * q[c] / dq1[c] - q[cm] * q[cm] / dq1[cm]);
                }
                if (xpp < R(0)) {
                    size_t ci = IDX(L, ip1, j);
                    if (dz[ci] < R(CC_GX) || dz[IDX(L, ip1, jp1)] < R(CC_GX)) {
                        advx = rx * (-(q[c] * xpp / dq1[c]));
                    } else if (dq1[ci] < R(CC_GX)) {
                        advx = rx * (-(q[c] * xpp / dq1[c]));
                    } else {
                        REAL xpe = R(0.25) * (p[ci] + p[IDX(L, ip1, jp1)] + p[c] + p[cq]);
                        advx = rx * (q[ci] * xpe / dq1[ci] - q[c] * xpp / dq1[c]);
                    }
                } else {
                    size_t ci = IDX(L, im1, j);
                    if (dz[ci] < R(CC_GX) || dz[IDX(L, im1, jp1)] < R(CC_GX)) {
                        advx = rx * (q[c] * xpp / dq1[c]);
                    } else if (dq1[IDX(L, i - 1, j)] < R(CC_GX)) {
                        advx = rx * (q[c] * xpp / dq1[c]);
                    } else {
                        REAL xpe = R(0.25) * (p[ci] + p[IDX(L, im1, jp1)] + p[IDX(L, i - 2, j)]
                                              + p[IDX(L, i - 2, jp1)]);
                        advx = rx * (q[c] * xpp / dq1[c] - q[ci] * xpe / dq1[ci]);
                    }
                }
                wave_breaking(L, c, &advx, &advy);
                xq = xq - advx - advy;
            }
            if (L->fric_switch != 1) xq = xq / (R(1) + ff);
            if (o_abs(xq) < R(CC_EPS)) xq = R(0);
            REAL lim = R(CC_VLIMIT) * dd;
            if (xq > lim) xq = lim;
            if (xq < -lim) xq = -lim;
            L->n2[c] = xq;
        }
    }
}


/* CONMOME_S (moment.f90:783-1268), nonlinear momentum in spherical
 * coordinates.  As CONMOME but: the face depth on a wet/dry face is
 * HP + (Z + Z(I+1))/2 (:906-915), the pressure term uses R2 / R4 of PARA
 * (per row for LAYGOV 1), Coriolis enters as +4 R3 XQQ / -4 R5 XPP
 * (:952, :1154), the advection coefficients are R21 (= R1), R0 and R22, and
 * the y friction is applied to XQ. */
static void conmome_s_x_rows(void *vctx, int js, int je) {
    conmome_ctx *x = (conmome_ctx *)vctx;
    ocl_layer *L = x->L;
    int ix = L->nx, jy = L->ny;
    int is = 2, ie = ix - 1;
    if (L->id == 1) is = 1;
    REAL konst = (L->fric_switch != 1) ? R(0.5) * R(L->dt) * R(CC_GRAV) : R(0);
    REAL fm = R(L->fric_coef);
    int ispans = CC_SPAN, ispane = ix - CC_SPAN, jspans = CC_SPAN, jspane = jy - CC_SPAN;
    const REAL *dp1 = x->dp1, *dp2 = x->dp2, *dz = L->dz2, *z = L->z2, *hz = L->h;
    const REAL *p = L->m1, *q = L->n1;
    for (int j = js; j <= je; j++) {
        int jp1 = MIN(j + 1, jy), jm1 = MAX(j - 1, 1);
        REAL r2 = L->r2[IDX(L, 1, j)], r3 = L->r3[j - 1], r21 = L->r1[j - 1], r0 = L->r0[j - 1];
        for (int i = is; i <= ie; i++) {
            int ip1 = MIN(i + 1, ix), im1 = MAX(i - 1, 1);
            size_t c = IDX(L, i, j), cp = IDX(L, ip1, j);
            REAL dd = R(0), df = R(0), ff = R(0);
            int noflux = 0;
            if (hz[c] <= R(CC_ELMAX) || L->hp[c] <= R(CC_ELMAX)) {
                noflux = 1;
            } else {
                if (dz[c] > R(CC_GX) && dz[cp] > R(CC_GX)) {
                    dd = dp2[c]; df = dp1[c];
                } else if (dz[c] > R(CC_GX) && dz[cp] <= R(CC_GX) && hz[cp] + z[c] > R(CC_GX)) {
                    dd = L->hp[c] + R(0.5) * (z[c] + z[cp]); df = dd;
                } else if (dz[c] <= R(CC_GX) && dz[cp] > R(CC_GX) && hz[c] + z[cp] > R(CC_GX)) {
                    dd = L->hp[c] + R(0.5) * (z[c] + z[cp]); df = dd;
                } else {
                    noflux = 1;
                }
                if (!noflux && dd < R(CC_GX)) noflux = 1;
            }
            if (noflux) { L->m2[c] = R(0); continue; }
            if (df < R(CC_DFMIN)) df = R(CC_DFMIN);
            REAL xqq = R(0.25) * (q[c] + q[cp] + q[IDX(L, i, jm1)] + q[IDX(L, ip1, jm1)]);
            if (L->fric_switch != 1)
                ff = konst * fm * fm * o_sqrt(p[c] * p[c] + xqq * xqq) / o_pow(df, R(CC_MANNEXP));
            else
                ff = R(0);
            REAL xp;
            if (L->modscm == 0 && j < jy)
                xp = p[c] - r2 * dd * (z[cp] - z[c])
                     - r2 * dd / R(12)
                           * ((z[IDX(L, ip1, jp1)] - R(2) * z[cp] + z[IDX(L, ip1, jm1)])
                              - (z[IDX(L, i, jp1)] - R(2) * z[c] + z[IDX(L, i, jm1)]));
            else
                xp = p[c] - r2 * dd * (z[cp] - z[c]);
            if (L->fric_switch != 1) xp = xp - ff * p[c];
            xp = xp + R(4.0) * r3 * xqq;
            if (L->linchk == 1 && dp1[c] >= R(CC_GX) && i > ispans && i < ispane && j > jspans
                && j < jspane) {
                REAL advx = R(0), advy = R(0);
                if (p[c] < R(0)) {
                    if (dp1[cp] < R(CC_GX) || dz[cp] < R(CC_GX))
                        advx = r21 * (-(p[c] * p[c] / dp1[c]));
                    else
                        advx = r21 * (p[cp] * p[cp] / dp1[cp] - p[c] * p[c] / dp1[c]);
                } else {
                    size_t cm = IDX(L, im1, j);
                    if (dp1[cm] < R(CC_GX) || dz[c] < R(CC_GX))
                        advx = r21 * (p[c] * p[c] / dp1[c]);
                    else
                        advx = r21 * (p[c] * p[c] / dp1[c] - p[cm] * p[cm] / dp1[cm]);
                }
                if (xqq < R(0)) {
                    size_t cj = IDX(L, i, jp1);
                    if (dz[cj] < R(CC_GX) || dz[IDX(L, ip1, jp1)] < R(CC_GX)) {
                        advy = r0 * (-(p[c] * xqq / dp1[c]));
                    } else if (dp1[cj] < R(CC_GX)) {
                        advy = r0 * (-(p[c] * xqq / dp1[c]));
                    } else {
                        REAL xqe = R(0.25) * (q[cj] + q[IDX(L, ip1, jp1)] + q[c] + q[cp]);
                        advy = r0 * (p[cj] * xqe / dp1[cj] - p[c] * xqq / dp1[c]);
                    }
                } else {
                    size_t cj = IDX(L, i, jm1);
                    if (dz[cj] < R(CC_GX) || dz[IDX(L, ip1, jm1)] < R(CC_GX)) {
                        advy = r0 * (p[c] * xqq / dp1[c]);
                    } else if (dp1[cj] < R(CC_GX)) {
                        advy = r0 * (p[c] * xqq / dp1[c]);
                    } else {
                        REAL xqe = R(0.25) * (q[cj] + q[IDX(L, ip1, jm1)] + q[IDX(L, i, j - 2)]
                                              + q[IDX(L, ip1, j - 2)]);
                        advy = r0 * (p[c] * xqq / dp1[c] - p[cj] * xqe / dp1[cj]);
                    }
                }
                wave_breaking(L, c, &advx, &advy);
                xp = xp - advx - advy;
            }
            if (L->fric_switch != 1) xp = xp / (R(1) + ff);
            if (o_abs(xp) < R(CC_EPS)) xp = R(0);
            REAL lim = R(CC_VLIMIT) * dd;
            if (xp > lim) xp = lim;
            if (xp < -lim) xp = -lim;
            L->m2[c] = xp;
        }
    }
}

static void conmome_s_y_rows(void *vctx, int js, int je) {
    conmome_ctx *x = (conmome_ctx *)vctx;
    ocl_layer *L = x->L;
    int ix = L->nx, jy = L->ny;
    int is = 2, ie = ix;
    if (L->id == 1) { is = 1; ie = ix - 1; }
    REAL konst = (L->fric_switch != 1) ? R(0.5) * R(L->dt) * R(CC_GRAV) : R(0);
    REAL fm = R(L->fric_coef);
    int ispans = CC_SPAN, ispane = ix - CC_SPAN, jspans = CC_SPAN, jspane = jy - CC_SPAN;
    const REAL *dq1 = x->dq1, *dq2 = x->dq2, *dz = L->dz2, *z = L->z2, *hz = L->h;
    const REAL *p = L->m1, *q = L->n1;
    for (int j = js; j <= je; j++) {
        int jp1 = MIN(j + 1, jy), jm1 = MAX(j - 1, 1);
        REAL r4 = L->r4[IDX(L, 1, j)], r5 = L->r5[j - 1], r0 = L->r0[j - 1], r22 = L->r22[j - 1];
        for (int i = is; i <= ie; i++) {
            int ip1 = MIN(i + 1, ix), im1 = MAX(i - 1, 1);
            size_t c = IDX(L, i, j), cq = IDX(L, i, jp1);
            REAL dd = R(0), df = R(0), ff = R(0);
            int noflux = 0;
            if (hz[c] <= R(CC_ELMAX) || L->hq[c] <= R(CC_ELMAX)) {
                noflux = 1;
            } else {
                if (dz[c] > R(CC_GX) && dz[cq] > R(CC_GX)) {
                    dd = dq2[c]; df = dq1[c];
                } else if (dz[c] > R(CC_GX) && dz[cq] <= R(CC_GX) && hz[cq] + z[c] > R(CC_GX)) {
                    dd = L->hq[c] + R(0.5) * (z[c] + z[cq]); df = dd;
                } else if (dz[c] <= R(CC_GX) && dz[cq] > R(CC_GX) && hz[c] + z[cq] > R(CC_GX)) {
                    dd = L->hq[c] + R(0.5) * (z[c] + z[cq]); df = dd;
                } else {
                    noflux = 1;
                }
                if (!noflux && dd < R(CC_GX)) noflux = 1;
            }
            if (noflux) { L->n2[c] = R(0); continue; }
            if (df < R(CC_DFMIN)) df = R(CC_DFMIN);
            REAL xpp = R(0.25) * (p[c] + p[cq] + p[IDX(L, im1, j)] + p[IDX(L, im1, jp1)]);
            if (L->fric_switch != 1)
                ff = konst * fm * fm * o_sqrt(q[c] * q[c] + xpp * xpp) / o_pow(df, R(CC_MANNEXP));
            else
                ff = R(0);
            REAL xq;
            if (L->modscm == 0 && i < ix)
                xq = q[c] - r4 * dd * (z[cq] - z[c])
                     - r4 * dd / R(12)
                           * ((z[IDX(L, ip1, jp1)] - R(2) * z[cq] + z[IDX(L, im1, jp1)])
                              - (z[IDX(L, ip1, j)] - R(2) * z[c] + z[IDX(L, im1, j)]));
            else
                xq = q[c] - r4 * dd * (z[cq] - z[c]);
            if (L->fric_switch != 1) xq = xq - ff * q[c];
            xq = xq - R(4.0) * r5 * xpp;
            if (L->linchk == 1 && dq1[c] >= R(CC_GX) && i > ispans && i < ispane && j > jspans
                && j < jspane) {
                REAL advx = R(0), advy = R(0);
                if (q[c] < R(0)) {
                    if (dq1[cq] < R(CC_GX) || dz[cq] < R(CC_GX))
                        advy = r0 * (-(q[c] * q[c] / dq1[c]));
                    else
                        advy = r0 * (q[cq] * q[cq] / dq1[cq] - q[c] * q[c] / dq1[c]);
                } else {
                    size_t cm = IDX(L, i, jm1);
                    if (dq1[cm] < R(CC_GX) || dz[c] < R(CC_GX))
                        advy = r0 * (q[c] * q[c] / dq1[c]);
                    else
                        advy = r0 * (q[c] * q[c] / dq1[c] - q[cm] * q[cm] / dq1[cm]);
                }
                if (xpp < R(0)) {
                    size_t ci = IDX(L, ip1, j);
                    if (dz[ci] < R(CC_GX) || dz[IDX(L, ip1, jp1)] < R(CC_GX)) {
                        advx = r22 * (-(q[c] * xpp / dq1[c]));
                    } else if (dq1[ci] < R(CC_GX)) {
                        advx = r22 * (-(q[c] * xpp / dq1[c]));
                    } else {
                        REAL xpe = R(0.25) * (p[ci] + p[IDX(L, ip1, jp1)] + p[c] + p[cq]);
                        advx = r22 * (q[ci] * xpe / dq1[ci] - q[c] * xpp / dq1[c]);
                    }
                } else {
                    size_t ci = IDX(L, im1, j);
                    if (dz[ci] < R(CC_GX) || dz[IDX(L, im1, jp1)] < R(CC_GX)) {
                        advx = r22 * (q[c] * xpp / dq1[c]);
                    } else if (dq1[IDX(L, i - 1, j)] < R(CC_GX)) {
                        advx = r22 * (q[c] * xpp / dq1[c]);
                    } else {
                        REAL xpe = R(0.25) * (p[ci] + p[IDX(L, im1, jp1)] + p[IDX(L, i - 2, j)]
                                              + p[IDX(L, i - 2, jp1)]);
                        advx = r22 * (q[c] * xpp / dq1[c] - q[ci] * xpe / dq1[ci]);
                    }
                }
                wave_breaking(L, c, &advx, &advy);
                xq = xq - advx - advy;
            }
            if (L->fric_switch != 1) xq = xq / (R(1) + ff);
            if (o_abs(xq) < R(CC_EPS)) xq = R(0);
            REAL lim = R(CC_VLIMIT) * dd;
            if (xq > lim) xq = lim;
            if (xq < -lim) xq = -lim;
            L->n2[c] = xq;
        }
    }
}

static void conmome(ocl_layer *L) {
    size_t n = (size_t)L->nx * L->ny;
    conmome_ctx x;
    x.L = L;
    x.dp1 = (REAL *)malloc(4 * n * sizeof(REAL));
    x.dp2 = x.dp1 + n; x.dq1 = x.dp2 + n; x.dq2 = x.dq1 + n;
    par_rows(conmome_pre_rows, &x, 1, L->ny);
    /* x: children I=2..NX-1, J=2..NY; root I=1..NX-1, J=1..NY-1 (moment.f90:376-389,
     * the same ranges in CONMOME_S, :867-878,1052-1063) */
    rowfn gx = L->laycord == 0 ? conmome_s_x_rows : conmome_x_rows;
    if (L->id == 1) par_rows(gx, &x, 1, L->ny - 1);
    else par_rows(gx, &x, 2, L->ny);
    /* y: children I=2..NX, J=2..NY-1; root I=1..NX-1, J=1..NY-1 (moment.f90:586-599) */
    rowfn fy = L->laycord == 0 ? conmome_s_y_rows : conmome_y_rows;
    if (L->id == 1) par_rows(fy, &x, 1, L->ny - 1);
    else par_rows(fy, &x, 2, L->ny - 1);
    free(x.dp1);
}

/* MOMT_S_D (dispersion.f90:544-838) with MASK = 0: MOMT_S plus the
 * modified-scheme term when MODSCM = 0 (:686-692, :817-823), and the y wet
 * test against ZERO (:706) */
static void momt_s_d_rows(void *ctx, int js, int je) {
    ocl_layer *L = (ocl_layer *)ctx;
    int nx = L->nx, ny = L->ny;
    int is0 = (L->id == 1) ? 1 : 2, js0 = is0;
    const REAL twlvth = R(0.08333333333333);
    for (int j = js; j <= je; j++) {
        if (j >= js0) {
            int jm1 = MAX(j - 1, 1), jp1 = MIN(j + 1, ny);
            for (int i = is0; i <= nx - 1; i++) {
                int ip1 = i + 1;
                size_t c = IDX(L, i, j), cp = IDX(L, ip1, j);
                if (L->h[c] > R(CC_GX) && L->h[cp] > R(CC_GX)) {
                    REAL tot_n = L->n1[c] + L->n1[cp] + L->n1[IDX(L, i, jm1)] + L->n1[IDX(L, ip1, jm1)];
                    REAL xm = L->m1[c] - L->r2[c] * (L->z2[cp] - L->z2[c]) + L->r3[j - 1] * tot_n;
                    if (L->modscm == 0) {
                        REAL scm = L->r2[c] * twlvth *
                                   ((L->z2[IDX(L, ip1, jp1)] - R(2) * L->z2[cp] + L->z2[IDX(L, ip1, jm1)]) -
                                    (L->z2[IDX(L, i, jp1)] - R(2) * L->z2[c] + L->z2[IDX(L, i, jm1)]));
                        xm = xm - scm;
                    }
                    if (o_abs(xm) < R(CC_EPS)) xm = R(0);
                    L->m2[c] = xm;
                } else {
                    L->m2[c] = R(0);
                }
            }
        }
        if (j >= js0 && j <= ny - 1) {
            int jp1 = j + 1;
            for (int i = is0; i <= nx; i++) {
                size_t c = IDX(L, i, j), cq = IDX(L, i, jp1);
                if (L->h[c] > R(0) && L->h[cq] > R(0)) {
                    int im1 = MAX(i - 1, 1), ip1 = MIN(i + 1, nx);
                    REAL tot_m = L->m1[IDX(L, im1, j)] + L->m1[IDX(L, im1, jp1)] + L->m1[c] + L->m1[cq];
                    REAL xn = L->n1[c] - L->r4[c] * (L->z2[cq] - L->z2[c]) - L->r5[j - 1] * tot_m;
                    if (L->modscm == 0) {
                        REAL scm = L->r4[c] * twlvth *
                                   ((L->z2[IDX(L, ip1, jp1)] - R(2) * L->z2[cq] + L->z2[IDX(L, im1, jp1)]) -
                                    (L->z2[IDX(L, ip1, j)] - R(2) * L->z2[c] + L->z2[IDX(L, im1, j)]));
                        xn = xn - scm;
                    }
                    if (o_abs(xn) < R(CC_EPS)) xn = R(0);
                    L->n2[c] = xn;
                } else {
                    L->n2[c] = R(0);
                }
            }
        }
    }
}

/* MOMT_C_D (dispersion.f90:839-1692) with MASK = 0 (:1225-1233, :1560-1568): total face depth
 * HM = HP + (Z + Z(I+1))/2 (x) and HN = (H + H(J+1) + Z + Z(J+1))/2 (y),
 * Manning friction, the modified-scheme term when MODSCM = 0; the convection
 * terms of LAYGOV 3 sit inside the MASK branch and never apply.  A dry face
 * is not written (the IFs at :922 and :1255 have no ELSE), so it keeps its
 * level-2 value, which after CHANGE / UPDATE equals level 1. */
static void momt_c_d_rows(void *ctx, int js, int je) {
    ocl_layer *L = (ocl_layer *)ctx;
    int nx = L->nx, ny = L->ny;
    int is0 = (L->id == 1) ? 1 : 2, js0 = is0;
    const REAL twlvth = R(0.08333333333333);
    const REAL konst = R(0.5) * R(L->dt) * R(CC_GRAV);
    const REAL fm = R(L->fric_coef), grx = R(L->grx), gry = R(L->gry);
    const REAL mexp = R(CC_MANNEXP);
    for (int j = js; j <= je; j++) {
        if (j >= js0) {
            int jm1 = MAX(j - 1, 1), jp1 = MIN(j + 1, ny);
            for (int i = is0; i <= nx - 1; i++) {
                int ip1 = i + 1;
                size_t c = IDX(L, i, j), cp = IDX(L, ip1, j);
                if (!(L->h[c] > R(CC_GX) && L->h[cp] > R(CC_GX))) continue;
                REAL hm = L->hp[c] + R(0.5) * (L->z2[c] + L->z2[cp]);
                REAL ff = R(0);
                if (L->fric_switch != 1) {
                    REAL xqq = R(0.25) * (L->n1[c] + L->n1[cp] + L->n1[IDX(L, i, jm1)] + L->n1[IDX(L, ip1, jm1)]);
                    if (hm >= R(1.0e-3))
                        ff = konst * fm * fm * o_sqrt(L->m1[c] * L->m1[c] + xqq * xqq) / o_pow(hm, mexp);
                }
                REAL xm = (R(1) - ff) * L->m1[c] - grx * hm * (L->z2[cp] - L->z2[c]);
                if (L->modscm == 0) {
                    REAL scm = grx * twlvth * hm *
                               ((L->z2[IDX(L, ip1, jp1)] - R(2) * L->z2[cp] + L->z2[IDX(L, ip1, jm1)]) -
                                (L->z2[IDX(L, i, jp1)] - R(2) * L->z2[c] + L->z2[IDX(L, i, jm1)]));
                    xm = xm - scm;
                }
                if (L->fric_switch != 1) xm = xm / (R(1) + ff);
                if (o_abs(xm) < R(CC_EPS)) xm = R(0);
                L->m2[c] = xm;
            }
        }
        if (j >= js0 && j <= ny - 1) {
            int jp1 = j + 1;
            for (int i = is0; i <= nx; i++) {
                size_t c = IDX(L, i, j), cq = IDX(L, i, jp1);
                if (!(L->h[c] > R(CC_GX) && L->h[cq] > R(CC_GX))) continue;
                int im1 = MAX(i - 1, 1), ip1 = MIN(i + 1, nx);
                REAL hn = R(0.5) * (L->h[c] + L->h[cq] + L->z2[c] + L->z2[cq]);
                REAL ff = R(0);
                if (L->fric_switch != 1) {
                    REAL xpp = R(0.25) * (L->m1[c] + L->m1[cq] + L->m1[IDX(L, im1, j)] + L->m1[IDX(L, im1, jp1)]);
                    if (hn >= R(1.0e-5))
                        ff = konst * fm * fm * o_sqrt(L->n1[c] * L->n1[c] + xpp * xpp) / o_pow(hn, mexp);
                }
                REAL xn = (R(1) - ff) * L->n1[c] - gry * hn * (L->z2[cq] - L->z2[c]);
                if (L->modscm == 0) {
                    REAL scm = gry * twlvth * hn *
                               ((L->z2[IDX(L, ip1, jp1)] - R(2) * L->z2[cq] + L->z2[IDX(L, im1, jp1)]) -
                                (L->z2[IDX(L, ip1, j)] - R(2) * L->z2[c] + L->z2[IDX(L, im1, j)]));
                    xn = xn - scm;
                }
                if (L->fric_switch != 1) xn = xn / (R(1) + ff);
                if (o_abs(xn) < R(CC_EPS)) xn = R(0);
                L->n2[c] = xn;
            }
        }
    }
}

void ocl_moment(ocl_layer *L) {
    /* dispatcher moment.f90:21-54 */
    int js = (L->id == 1) ? 1 : 2;
    if (L->laygov == 2 || L->laygov == 3) {
        par_rows(L->laycord == 0 ? momt_s_d_rows : momt_c_d_rows, L, js, L->ny);
        return;
    }
    if (L->laycord == 0 && L->laygov == 1) conmome(L);
    else if (L->laycord == 0) par_rows(momt_s_rows, L, js, L->ny);
    else if (L->laygov == 1) conmome(L);
    else par_rows(momt_c_rows, L, js, L->ny);
}

/* ------------------------------------------------------------------ */
/* OPEN (boundaries.f90:22-202) radiation boundary on the outer layer  */
/* ------------------------------------------------------------------ */
void ocl_open(ocl_layer *L) {
    int nx = L->nx, ny = L->ny;
    const REAL *m = L->m1, *n = L->n1, *h = L->h;  /* M(:,:,2) == M(:,:,1) at call time */
    REAL *z = L->z2;
    const REAL grav = R(CC_GRAV), gx = R(CC_GX), ub = R(CC_UB);
    for (int i = 2; i <= nx - 1; i++) { /* J = 1 */
        size_t c = IDX(L, i, 1);
        if (h[c] > gx) {
            REAL cc = o_sqrt(grav * h[c]);
            REAL uh = R(0.5) * (m[c] + m[IDX(L, i - 1, 1)]);
            REAL uu = o_sqrt(uh * uh + n[c] * n[c]);
            REAL zz = uu / cc;
            if (n[c] > R(0)) zz = -zz;
            if (o_abs(zz) > ub) zz = R(0);
            z[c] = zz;
        } else z[c] = R(0);
    }
    for (int i = 2; i <= nx - 1; i++) { /* J = NY */
        size_t c = IDX(L, i, ny), cs = IDX(L, i, ny - 1);
        if (h[c] > gx) {
            REAL cc = o_sqrt(grav * h[c]);
            REAL uh = R(0.5) * (m[c] + m[IDX(L, i - 1, ny)]);
            REAL uu = o_sqrt(uh * uh + n[cs] * n[cs]);
            REAL zz = uu / cc;
            if (n[cs] < R(0)) zz = -zz;
            if (o_abs(zz) > ub) zz = R(0);
            z[c] = zz;
        } else z[c] = R(0);
    }
    for (int j = 2; j <= ny - 1; j++) { /* I = 1 */
        size_t c = IDX(L, 1, j), cs = IDX(L, 1, j - 1);
        if (h[c] > gx) {
            REAL cc = o_sqrt(grav * h[c]);
            REAL uh;
            if (h[cs] > gx) uh = R(0.5) * (n[c] + n[cs]);
            else uh = n[c];
            REAL uu = o_sqrt(uh * uh + m[c] * m[c]);
            REAL zz = uu / cc;
            if (m[c] > R(0)) zz = -zz;
            if (o_abs(zz) > ub) zz = R(0);
            z[c] = zz;
        } else z[c] = R(0);
    }
    for (int j = 2; j <= ny - 1; j++) { /* I = NX */
        size_t c = IDX(L, nx, j), cw = IDX(L, nx - 1, j);
        if (h[c] > gx) {
            REAL cc = o_sqrt(grav * h[c]);
            REAL uh = R(0.5) * (n[c] + n[IDX(L, nx, j - 1)]);
            REAL uu = o_sqrt(uh * uh + m[cw] * m[cw]);
            REAL zz = uu / cc;
            if (m[cw] < R(0)) zz = -zz;
            if (o_abs(zz) > ub) zz = R(0);
            z[c] = zz;
        } else z[c] = R(0);
    }
    { /* corner (1,1) */
        size_t c = IDX(L, 1, 1);
        if (h[c] > gx) {
            REAL qx = m[c], qy = n[c];
            REAL cc = o_sqrt(grav * h[c]);
            REAL uh = o_sqrt(qx * qx + qy * qy);
            REAL zz = uh / cc;
            if (qx > R(0) || qy > R(0)) zz = -zz;
            if (o_abs(zz) > ub) zz = R(0);
            z[c] = zz;
        } else z[c] = R(0);
    }
    { /* corner (NX,1) */
        size_t c = IDX(L, nx, 1);
        if (h[c] > gx) {
            REAL qx = m[IDX(L, nx - 1, 1)], qy = n[c];
            REAL cc = o_sqrt(grav * h[c]);
            REAL uh = o_sqrt(qx * qx + qy * qy);
            REAL zz = uh / cc;
            if (qx < R(0) || qy > R(0)) zz = -zz;
            if (o_abs(zz) > ub) zz = R(0);
            z[c] = zz;
        } else z[c] = R(0);
    }
    { /* corner (1,NY) */
        size_t c = IDX(L, 1, ny);
        if (h[c] > gx) {
            REAL qx = m[c], qy = n[IDX(L, 1, ny - 1)];
            REAL cc = o_sqrt(grav * h[c]);
            REAL uh = o_sqrt(qx * qx + qy * qy);
            REAL zz = uh / cc;
            if (qx > R(0) || qy < R(0)) zz = -zz;
            if (o_abs(zz) > ub) zz = R(0);
            z[c] = zz;
        } else z[c] = R(0);
    }
    { /* corner (NX,NY) */
        size_t c = IDX(L, nx, ny);
        if (h[c] > gx) {
            REAL qx = m[IDX(L, nx - 1, ny)], qy = n[IDX(L, nx, ny - 1)];
            REAL cc = o_sqrt(grav * h[c]);
            REAL uh = o_sqrt(qx * qx + qy * qy);
            REAL zz = uh / cc;
            if (qx < R(0) || qy < R(0)) zz = -zz;
            z[c] = zz;
            if (o_abs(z[c]) > ub) z[c] = R(0);
        } else z[c] = R(0);
    }
}

/* ------------------------------------------------------------------ */
/* time-level rotation                                                 */
/* ------------------------------------------------------------------ */
void ocl_change(ocl_layer *L) {
    /* CHANGE (comcot.f90:475-512): Z, M, N (:,:,2) -> (:,:,1) */
    size_t n = (size_t)L->nx * L->ny;
    memcpy(L->z1, L->z2, n * sizeof(REAL));
    memcpy(L->m1, L->m2, n * sizeof(REAL));
    memcpy(L->n1, L->n2, n * sizeof(REAL));
}

void ocl_update(ocl_layer *L) {
    /* UPDATE (all_grids.f90:316-339): edge copy of Z(:,:,2), then rotation */
    int nx = L->nx, ny = L->ny;
    for (int j = 1; j <= ny; j++) L->z2[IDX(L, 1, j)] = L->z2[IDX(L, 2, j)];
    for (int i = 1; i <= nx; i++) L->z2[IDX(L, i, 1)] = L->z2[IDX(L, i, 2)];
    ocl_change(L);
}

/* ------------------------------------------------------------------ */
/* JNQ / EDGEINTERP / NEWQ  (all_grids.f90:452-801)                    */
/* ------------------------------------------------------------------ */
/* EDGEINTERP_VERT (all_grids.f90:502-550): child M on column II from the
 * parent flux profile flux[J], J = YS..YE */
static void edgeinterp_vert(const REAL *flux, ocl_layer *C, int side) {
    int nn = 2 * C->rel_size, ir = C->rel_size;
    int ys = C->corners[2], ye = C->corners[3];
    int j_shift = -ys * ir + 1;
    int ii = (side == 0) ? 1 : C->nx;
    for (int j = ys; j <= ye; j++) {
        REAL flux_s = R(0.5) * (flux[j - 2] + flux[j - 1]);
        REAL flux_e = R(0.5) * (flux[j] + flux[j - 1]);
        REAL c1 = (REAL)((double)(flux_e - flux_s) / (double)nn);
        REAL c2 = -c1 + flux_s;
        int js = j * ir + j_shift;
        for (int k = 1; k <= ir; k++) {
            int jj = js + k;
            size_t c = IDX(C, ii, jj);
            C->m1[c] = R(2) * R(k) * c1 + c2;
            if (C->h[c] + C->z1[c] <= R(CC_GX)) C->m1[c] = R(0);
        }
    }
}

/* EDGEINTERP_HORI (all_grids.f90:553-604): child N on row JJ */
static void edgeinterp_hori(const REAL *flux, ocl_layer *C, int side) {
    int nn = 2 * C->rel_size, ir = C->rel_size;
    int xs = C->corners[0], xe = C->corners[1];
    int i_shift = -xs * ir + 1;
    int jj = (side == 0) ? 1 : C->ny;
    for (int i = xs; i <= xe; i++) {
        REAL flux_s = R(0.5) * (flux[i - 2] + flux[i - 1]);
        REAL flux_e = R(0.5) * (flux[i] + flux[i - 1]);
        REAL c1 = (REAL)((double)(flux_e - flux_s) / (double)nn);
        REAL c2 = -c1 + flux_s;
        int is = i * ir + i_shift;
        for (int k = 1; k <= ir; k++) {
            int ii = is + k;
            size_t c = IDX(C, ii, jj);
            C->n1[c] = R(2) * R(k) * c1 + c2;
            if (C->h[c] + C->z1[c] <= R(CC_GX)) C->n1[c] = R(0);
        }
    }
}

void ocl_jnq(ocl_layer *P, ocl_layer *C) {
    /* JNQ (all_grids.f90:452-498), SC_OPTION = 0 */
    int is = C->corners[0], ie = C->corners[1], js = C->corners[2], je = C->corners[3];
    REAL *col = (REAL *)malloc((size_t)(P->ny > P->nx ? P->ny : P->nx) * sizeof(REAL));
    for (int j = 1; j <= P->ny; j++) col[j - 1] = P->m1[IDX(P, is - 1, j)];
    edgeinterp_vert(col, C, 0);
    for (int j = 1; j <= P->ny; j++) col[j - 1] = P->m1[IDX(P, ie, j)];
    edgeinterp_vert(col, C, 1);
    for (int i = 1; i <= P->nx; i++) col[i - 1] = P->n1[IDX(P, i, js - 1)];
    edgeinterp_hori(col, C, 0);
    for (int i = 1; i <= P->nx; i++) col[i - 1] = P->n1[IDX(P, i, je)];
    edgeinterp_hori(col, C, 1);
    free(col);
}

/* NEWQ_VERT (all_grids.f90:608-724) */
static void newq_vert(ocl_layer *P, ocl_layer *C, int t, int side) {
    int is = C->corners[0], ie = C->corners[1], js = C->corners[2], je = C->corners[3];
    int i = (side == 0) ? is - 1 : ie;
    REAL c1 = (R(t) - R(1)) / R(C->rel_time);
    REAL c2 = R(1) - c1;
    REAL *yflux = (REAL *)calloc((size_t)P->ny, sizeof(REAL));
    int ip1 = i + 1;
    REAL grx = R(P->grx);
    for (int j = js - 2; j <= je + 2; j++) {
        size_t c = IDX(P, i, j), cp = IDX(P, ip1, j);
        if ((P->h[c] + P->z2[c] > R(CC_GX)) && (P->h[cp] + P->z2[cp] > R(CC_GX))) {
            if (t == 2) {
                REAL xm;
                if (P->laycord == 0) {
                    int jm1 = j - 1;
                    REAL tot_n = P->n1[c] + P->n1[cp] + P->n1[IDX(P, i, jm1)] + P->n1[IDX(P, ip1, jm1)];
                    xm = P->m1[c] - P->r2[c] * (P->z2[cp] - P->z2[c]) + P->r3[j - 1] * tot_n;
                } else {
                    REAL hm = P->hp[c] + R(0.5) * (P->z2[c] + P->z2[cp]);
                    xm = P->m1[c] - grx * hm * (P->z2[cp] - P->z2[c]);
                }
                if (o_abs(xm) < R(CC_EPS)) xm = R(0);
                P->yflux[(size_t)side * P->ny + (j - 1)] = xm;
            }
            yflux[j - 1] = c1 * P->yflux[(size_t)side * P->ny + (j - 1)] + c2 * P->m1[c];
        }
    }
    edgeinterp_vert(yflux, C, side);
    free(yflux);
}

/* NEWQ_HORI (all_grids.f90:728-801) */
static void newq_hori(ocl_layer *P, ocl_layer *C, int t, int side) {
    int is = C->corners[0], ie = C->corners[1], js = C->corners[2], je = C->corners[3];
    int j = (side == 0) ? js - 1 : je;
    REAL c1 = (R(t) - R(1)) / R(C->rel_time);
    REAL c2 = R(1) - c1;
    REAL *xflux = (REAL *)calloc((size_t)P->nx, sizeof(REAL));
    int jp1 = j + 1;
    REAL gry = R(P->gry);
    for (int i = is - 2; i <= ie + 2; i++) {
        size_t c = IDX(P, i, j), cq = IDX(P, i, jp1);
        if ((P->h[c] + P->z2[c] > R(CC_GX)) && (P->h[cq] + P->z2[cq] > R(CC_GX))) {
            if (t == 2) {
                int im1 = i - 1;
                REAL xn;
                if (P->laycord == 0) {
                    REAL tot_m = P->m1[IDX(P, im1, j)] + P->m1[IDX(P, im1, jp1)] + P->m1[c] + P->m1[cq];
                    xn = P->n1[c] - P->r4[c] * (P->z2[cq] - P->z2[c]) - P->r5[j - 1] * tot_m;
                } else {
                    REAL hn = P->hq[c] + R(0.5) * (P->z2[c] + P->z2[cq]);
                    xn = P->n1[c] - gry * hn * (P->z2[cq] - P->z2[c]);
                }
                if (o_abs(xn) < R(CC_EPS)) xn = R(0);
                P->xflux[(size_t)side * P->nx + (i - 1)] = xn;
            }
            xflux[i - 1] = c1 * P->xflux[(size_t)side * P->nx + (i - 1)] + c2 * P->n1[c];
        }
    }
    edgeinterp_hori(xflux, C, side);
    free(xflux);
}

void ocl_newq(ocl_layer *P, ocl_layer *C, int t) {
    /* NEWQ (all_grids.f90:608-660), SC_OPTION = 0 */
    newq_vert(P, C, t, 0);
    newq_vert(P, C, t, 1);
    newq_hori(P, C, t, 0);
    newq_hori(P, C, t, 1);
}

/* JNZ (all_grids.f90:342-421), SC_OPTION = 0: child -> parent surface */
typedef struct { ocl_layer *P, *C; } jnz_ctx;
static void jnz_rows(void *vctx, int js, int je) {
    jnz_ctx *x = (jnz_ctx *)vctx;
    ocl_layer *P = x->P, *C = x->C;
    int ir = C->rel_size;
    REAL half = R((C->rel_size * C->rel_size)) / R(2);
    int is = C->corners[0], ie = C->corners[1], jsc = C->corners[2];
    int i_shift = -is * ir + 1, j_shift = -jsc * ir + 1;
    int even = (C->rel_time % 2) == 0;
    for (int j = js; j <= je; j++) {
        for (int i = is; i <= ie; i++) {
            REAL sum = R(0), count = R(0);
            int i0 = i * ir + i_shift, j0 = j * ir + j_shift;
            for (int ki = 1; ki <= ir; ki++) {
                for (int kj = 1; kj <= ir; kj++) {
                    size_t c = IDX(C, i0 + ki, j0 + kj);
                    if (C->h[c] + C->z2[c] > R(CC_GX)) {
                        if (even) sum = sum + R(0.5) * (C->z1[c] + C->z2[c]);
                        else sum = sum + C->z2[c];
                        count = count + R(1);
                    }
                }
            }
            if (count > half) P->z2[IDX(P, i, j)] = sum / count;
            else P->z2[IDX(P, i, j)] = R(0);
        }
    }
}

void ocl_jnz(ocl_layer *P, ocl_layer *C) {
    jnz_ctx x = {P, C};
    par_rows(jnz_rows, &x, C->corners[2], C->corners[3]);
}

/* ------------------------------------------------------------------ */
/* SC_OPTION = 1: Cartesian child of a spherical parent, coupled through */
/* the child nodes' positions POS and bilinear weights CXY in the parent */
/* ------------------------------------------------------------------ */
static inline const int *sc_pos(ocl_layer *C, int i, int j) { return C->pos + 2 * IDX(C, i, j); }
static inline const REAL *sc_w(ocl_layer *C, int i, int j) { return C->cxy + 4 * IDX(C, i, j); }

/* Z1+Z2+Z3+Z4 of the four weighted parent values (all_grids.f90:1030-1034) */
static REAL sc_bilin(const REAL *f, ocl_layer *P, const int *ps, const REAL *w) {
    int ki = ps[0], kj = ps[1];
    REAL z1 = f[IDX(P, ki, kj)] * w[0];
    REAL z2 = f[IDX(P, ki + 1, kj)] * w[1];
    REAL z3 = f[IDX(P, ki, kj + 1)] * w[2];
    REAL z4 = f[IDX(P, ki + 1, kj + 1)] * w[3];
    return z1 + z2 + z3 + z4;
}

/* EDGE_INTERP_SC (all_grids.f90:996-1087).  The reference tests wetness at
 * LA%H(I,J)+LA%Z(I,J,2) with I (left/right edges) and J (bottom/top edges)
 * left over from elsewhere: an undefined value on entry and NY+1 after the
 * J loops, outside the array.  That read cannot be reproduced; the test
 * here is at the edge node itself, as NEWQ_SC (:1268-1362) makes it. */
void ocl_edge_sc(ocl_layer *P, ocl_layer *C) {
    for (int j = 1; j <= C->ny; j++)
        for (int s = 0; s < 2; s++) {
            int i = s == 0 ? 1 : C->nx;
            size_t c = IDX(C, i, j);
            C->m1[c] = (C->h[c] + C->z2[c] > R(CC_GX)) ? sc_bilin(P->m1, P, sc_pos(C, i, j), sc_w(C, i, j)) : R(0);
        }
    for (int i = 1; i <= C->nx; i++)
        for (int s = 0; s < 2; s++) {
            int j = s == 0 ? 1 : C->ny;
            size_t c = IDX(C, i, j);
            C->n1[c] = (C->h[c] + C->z2[c] > R(CC_GX)) ? sc_bilin(P->n1, P, sc_pos(C, i, j), sc_w(C, i, j)) : R(0);
        }
}

/* NEWQ_SC forecast of the parent X flux on one band (all_grids.f90:1130-1163) */
static void sc_forecast_m(ocl_layer *P, int is, int ie, int js, int je) {
    const REAL twlvth = R(0.08333333333333);
    for (int i = is; i <= ie; i++) {
        int ip1 = i + 1;
        for (int j = js; j <= je; j++) {
            size_t c = IDX(P, i, j), cp = IDX(P, ip1, j);
            if (P->h[c] > R(CC_GX) && P->h[cp] > R(CC_GX)) {
                int jm1 = MAX(j - 1, 1), jp1 = MIN(j + 1, P->ny);
                REAL tot_n = P->n1[c] + P->n1[cp] + P->n1[IDX(P, i, jm1)] + P->n1[IDX(P, ip1, jm1)];
                REAL xm = P->m1[c] - P->r2[c] * (P->z2[cp] - P->z2[c]) + P->r3[j - 1] * tot_n;
                if (P->modscm == 0) {
                    REAL scm = P->r2[c] * twlvth *
                               ((P->z2[IDX(P, ip1, jp1)] - R(2) * P->z2[cp] + P->z2[IDX(P, ip1, jm1)]) -
                                (P->z2[IDX(P, i, jp1)] - R(2) * P->z2[c] + P->z2[IDX(P, i, jm1)]));
                    xm = xm - scm;
                }
                if (o_abs(xm) < R(CC_EPS)) xm = R(0);
                P->m2[c] = xm;
            } else {
                P->m2[c] = R(0);
            }
        }
    }
}

/* the Y flux on one band (all_grids.f90:1198-1231) */
static void sc_forecast_n(ocl_layer *P, int is, int ie, int js, int je) {
    const REAL twlvth = R(0.08333333333333);
    for (int j = js; j <= je; j++) {
        int jp1 = j + 1;
        for (int i = is; i <= ie; i++) {
            size_t c = IDX(P, i, j), cq = IDX(P, i, jp1);
            if (P->h[c] > R(CC_GX) && P->h[cq] > R(CC_GX)) {
                int im1 = MAX(i - 1, 1), ip1 = MIN(i + 1, P->nx);
                REAL tot_m = P->m1[IDX(P, im1, j)] + P->m1[IDX(P, im1, jp1)] + P->m1[c] + P->m1[cq];
                REAL xn = P->n1[c] - P->r4[c] * (P->z2[cq] - P->z2[c]) - P->r5[j - 1] * tot_m;
                if (P->modscm == 0) {
                    REAL scm = P->r4[c] * twlvth *
                               ((P->z2[IDX(P, ip1, jp1)] - R(2) * P->z2[cq] + P->z2[IDX(P, im1, jp1)]) -
                                (P->z2[IDX(P, ip1, j)] - R(2) * P->z2[c] + P->z2[IDX(P, im1, j)]));
                    xn = xn - scm;
                }
                if (o_abs(xn) < R(CC_EPS)) xn = R(0);
                P->n2[c] = xn;
            } else {
                P->n2[c] = R(0);
            }
        }
    }
}

void ocl_newq_sc(ocl_layer *P, ocl_layer *C, int t) {
    /* NEWQ_SC (all_grids.f90:1090-1364): forecast the parent fluxes at the
     * end of its step on four bands around the child's edges, written into
     * the parent's level 2 (its momentum step overwrites them later), then
     * blend the two levels at the edge nodes */
    const int nx = C->nx, ny = C->ny;
    int a = sc_pos(C, 1, 1)[0], b = sc_pos(C, 1, ny)[0];
    sc_forecast_m(P, MIN(a, b) - 2, MAX(a, b) + 2, C->corners[2] - 2, C->corners[3] + 2);
    a = sc_pos(C, nx, 1)[0]; b = sc_pos(C, nx, ny)[0];
    sc_forecast_m(P, MIN(a, b) - 2, MAX(a, b) + 2, C->corners[2] - 2, C->corners[3] + 2);
    a = sc_pos(C, 1, ny)[1]; b = sc_pos(C, nx, ny)[1];
    sc_forecast_n(P, C->corners[0] - 2, C->corners[1] + 2, MIN(a, b) - 2, MAX(a, b) + 2);
    a = sc_pos(C, 1, 1)[1]; b = sc_pos(C, nx, 1)[1];
    sc_forecast_n(P, C->corners[0] - 2, C->corners[1] + 2, MIN(a, b) - 2, MAX(a, b) + 2);
    const REAL c1 = (R(t) - R(1)) / R(C->rel_time);
    const REAL c2 = R(1) - c1;
    for (int j = 1; j <= ny; j++)
        for (int s = 0; s < 2; s++) {
            int i = s == 0 ? 1 : nx;
            size_t c = IDX(C, i, j);
            if (C->h[c] + C->z2[c] > R(CC_GX)) {
                REAL x1 = sc_bilin(P->m1, P, sc_pos(C, i, j), sc_w(C, i, j));
                REAL x2 = sc_bilin(P->m2, P, sc_pos(C, i, j), sc_w(C, i, j));
                C->m1[c] = c1 * x2 + c2 * x1;
            } else {
                C->m1[c] = R(0);
            }
        }
    for (int i = 1; i <= nx; i++)
        for (int s = 0; s < 2; s++) {
            int j = s == 0 ? 1 : ny;
            size_t c = IDX(C, i, j);
            if (C->h[c] + C->z2[c] > R(CC_GX)) {
                REAL y1 = sc_bilin(P->n1, P, sc_pos(C, i, j), sc_w(C, i, j));
                REAL y2 = sc_bilin(P->n2, P, sc_pos(C, i, j), sc_w(C, i, j));
                /* the reference's top edge weights YN1 by C1 (all_grids.f90:1357) */
                REAL w1 = (s == 1 && !C->sc_fix_top) ? c1 : c2;
                C->n1[c] = c1 * y2 + w1 * y1;
            } else {
                C->n1[c] = R(0);
            }
        }
}

void ocl_jnz_sc(ocl_layer *P, ocl_layer *C) {
    /* JNZ_SC (all_grids.f90:1367-1425): sum of the wet child surfaces that
     * fall in each parent cell, in the reference's loop order (child I
     * outermost); the parent surface takes their mean where more than half
     * of r*r nodes contributed and is left as it is elsewhere.  Child nodes
     * outside the parent interior (KI or KJ = 0) are skipped: the reference
     * would index its sums at 0 there. */
    size_t np = (size_t)P->nx * P->ny;
    REAL *zs = (REAL *)calloc(np, sizeof(REAL));
    REAL *cs = (REAL *)calloc(np, sizeof(REAL));
    const REAL half = R(C->rel_size * C->rel_size) / R(2);
    for (int i = 1; i <= C->nx; i++)
        for (int j = 1; j <= C->ny; j++) {
            size_t c = IDX(C, i, j);
            if (C->h[c] + C->z2[c] > R(CC_GX)) {
                const int *ps = sc_pos(C, i, j);
                if (ps[0] < 1 || ps[1] < 1) continue;
                size_t q = IDX(P, ps[0], ps[1]);
                zs[q] = zs[q] + C->z2[c];
                cs[q] = cs[q] + R(1);
            }
        }
    for (int i = C->corners[0]; i <= C->corners[1]; i++)
        for (int j = C->corners[2]; j <= C->corners[3]; j++) {
            size_t q = IDX(P, i, j);
            if (cs[q] > half) P->z2[q] = zs[q] / cs[q];
        }
    free(zs);
    free(cs);
}

/* ------------------------------------------------------------------ */
/* outputs: running maximum, arrival step, gauges                      */
/* ------------------------------------------------------------------ */
void ocl_maxamp(ocl_layer *L) {
    /* maximum_recorder_kernel (GPUOutput.cu:46-53): Zmax = max(Zmax, Z2),
     * Zmax starts from the initial Z (GPUcomcot.cu:79) */
    size_t n = (size_t)L->nx * L->ny;
    for (size_t c = 0; c < n; c++)
        if (!(L->zmax[c] >= L->z2[c])) L->zmax[c] = L->z2[c];
}

void ocl_arrival_start(ocl_layer *L, double thr) {
    /* arrival at the start of tracking: step 0 for a wet cell (H > GX) whose
     * surface is already above thr, -1 (not yet) elsewhere */
    size_t n = (size_t)L->nx * L->ny;
    REAL t = R(thr);
    for (size_t c = 0; c < n; c++) L->arrival[c] = (L->h[c] > R(CC_GX) && L->z1[c] > t) ? 0 : -1;
}

void ocl_arrival(ocl_layer *L, int step, double thr) {
    /* arrival step: the first outer step after which a wet cell (H > GX)
     * has Z2 > thr; 0 where the surface was above thr when tracking began
     * (ocl_arrival_start), -1 until then.  The reference has no arrival-time
     * product; this definition is shared with the CUDA kernels. */
    size_t n = (size_t)L->nx * L->ny;
    REAL t = R(thr);
    for (size_t c = 0; c < n; c++)
        if (L->arrival[c] < 0 && L->h[c] > R(CC_GX) && L->z2[c] > t) L->arrival[c] = step;
}

double ocl_gauge(ocl_layer *L, int ki, int kj, double cx, double cy) {
    /* GET_TS bilinear weights (output.f90:1078-1090) on Z(:,:,2) */
    REAL l1 = L->z2[IDX(L, ki, kj)], l2 = L->z2[IDX(L, ki + 1, kj)];
    REAL l3 = L->z2[IDX(L, ki, kj + 1)], l4 = L->z2[IDX(L, ki + 1, kj + 1)];
    REAL x = R(cx), y = R(cy);
    REAL z1 = l1 * (R(1) - x) * (R(1) - y);
    REAL z2 = l2 * (x) * (R(1) - y);
    REAL z3 = l3 * (R(1) - x) * (y);
    REAL z4 = l4 * (x) * (y);
    return (double)(z1 + z2 + z3 + z4);
}

/* ------------------------------------------------------------------ */
/* ALL_GRID (all_grids.f90:4-312): recursive sub-cycling of the tree   */
/* ------------------------------------------------------------------ */
static void all_grid_rec(ocl_layer *layers, int n, int parent_idx) {
    ocl_layer *P = &layers[parent_idx];
    for (int c = 0; c < n; c++) {
        ocl_layer *C = &layers[c];
        if (c == parent_idx || C->parent != P->id) continue;
        int nhalf = C->rel_time / 2 + 1;
        for (int k = 1; k <= C->rel_time; k++) {
            if (C->sc_option == 1) {
                if (k == 1) ocl_edge_sc(P, C);
                else ocl_newq_sc(P, C, k);
            } else {
                if (k == 1) ocl_jnq(P, C);
                else ocl_newq(P, C, k);
            }
            ocl_mass(C);
            all_grid_rec(layers, n, c);
            ocl_moment(C);
            if (k == nhalf) {
                if (C->sc_option == 1) ocl_jnz_sc(P, C);
                else ocl_jnz(P, C);
            }
            ocl_update(C);
        }
    }
}

void ocl_all_grid(ocl_layer *layers, int n) { all_grid_rec(layers, n, 0); }

void ocl_sponge(ocl_layer *L) {
    /* SPONGE_LAYER (boundaries.f90:229-244): where either coefficient is
     * positive, M2 += CX*DT*M1 and N2 += CY*DT*N1 */
    const REAL dt = R(L->dt);
    for (int j = 1; j <= L->ny; j++)
        for (int i = 1; i <= L->nx; i++) {
            size_t c = IDX(L, i, j);
            REAL cx = L->spx[c], cy = L->spy[c];
            if (cx > R(0) || cy > R(0)) {
                L->m2[c] = L->m2[c] + cx * dt * L->m1[c];
                L->n2[c] = L->n2[c] + cy * dt * L->n1[c];
            }
        }
}

void ocl_sponge_coef(int nx, int ny, int laycord, const REAL *x, const REAL *y, const REAL *h, REAL *coefx,
                     REAL *coefy) {
    /* H_CALC (boundaries.f90:351-385): mean wet depth, summed with I
     * outermost as the Fortran loops run */
    REAL hsum = R(0);
    int k = 0;
    for (int i = 1; i <= nx; i++)
        for (int j = 1; j <= ny; j++) {
            REAL hv = h[(size_t)(j - 1) * nx + (i - 1)];
            if (hv > R(CC_GX)) {
                hsum = hsum + hv;
                k = k + 1;
            }
        }
    REAL depth = k > 0 ? hsum / (REAL)k : R(0);
    if (depth <= R(CC_GX)) depth = R(CC_GX);
    /* SPONGE_COEF (boundaries.f90:271-345) */
    const REAL pi = R(CC_PI), grav = R(CC_GRAV);
    const REAL wavelength = R(20.0) * depth;
    const REAL width = R(2.0) * wavelength;
    const REAL alpha_c = R(10.0);
    const REAL t = wavelength / o_sqrt(grav * depth);
    const REAL omega = R(2.0) * pi / t;
    const REAL sw = laycord == 0 ? width / R(CC_R_EARTH) * R(180.0) / pi : width;
    const REAL r_max = width;
    const REAL xs = x[0] + sw, ys = y[0] + sw, xe = x[nx - 1] - sw, ye = y[ny - 1] - sw;
    const REAL em1 = o_exp(R(1.0)) - R(1.0);
    for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++) {
            const REAL x0 = x[i - 1], y0 = y[j - 1];
            REAL rx = x0 <= xs ? -(x0 - xs) : (x0 >= xe ? x0 - xe : R(0));
            REAL ry = y0 <= ys ? -(y0 - ys) : (y0 >= ye ? y0 - ye : R(0));
            REAL xr = rx, yr = ry;
            if (xr <= R(0)) xr = R(0);
            if (yr <= R(0)) yr = R(0);
            if (xr >= r_max) xr = r_max;
            if (yr >= r_max) yr = r_max;
            const REAL ax = xr / r_max, ay = yr / r_max;
            REAL cx = alpha_c * omega * (o_exp(ax * ax) - R(1.0)) / em1;
            REAL cy = alpha_c * omega * (o_exp(ay * ay) - R(1.0)) / em1;
            if (cx <= R(CC_EPS)) cx = R(0);
            if (cy <= R(CC_EPS)) cy = R(0);
            coefx[(size_t)(j - 1) * nx + (i - 1)] = cx;
            coefy[(size_t)(j - 1) * nx + (i - 1)] = cy;
        }
}

void ocl_step(ocl_layer *layers, int n, int step, double arrival_thr) {
    /* one outer step in the GPU driver's order (comcot.f90:359-439) */
    ocl_layer *L = &layers[0];
    ocl_mass(L);
    ocl_open(L);
    ocl_all_grid(layers, n);
    ocl_moment(L);
    if (L->spx && L->spy) ocl_sponge(L);
    if (L->zmax) ocl_maxamp(L);
    if (L->arrival) ocl_arrival(L, step, arrival_thr);
}

static ocl_layer *find_layer(ocl_layer *layers, int n, int id) {
    for (int k = 0; k < n; k++)
        if (layers[k].id == id) return &layers[k];
    return NULL;
}

/* outer steps first .. first + nsteps - 1 (1-based: the arrival step a
 * cell records is the outer step's number, so a run may continue where an
 * earlier one stopped); gauge samples go to ts[0 .. nsteps-1] */
int ocl_run_from(ocl_layer *layers, int n, int first, int nsteps, double arrival_thr, int ngauges,
                 const int *g_layer, const int *g_ki, const int *g_kj, const double *g_cx,
                 const double *g_cy, REAL *ts) {
    for (int k = 1; k <= nsteps; k++) {
        ocl_step(layers, n, first + k - 1, arrival_thr);
        for (int g = 0; g < ngauges; g++) {
            ocl_layer *G = find_layer(layers, n, g_layer[g]);
            if (!G) return -1;
            ts[(size_t)(k - 1) * ngauges + g] = (REAL)ocl_gauge(G, g_ki[g], g_kj[g], g_cx[g], g_cy[g]);
        }
        ocl_change(&layers[0]);
    }
    return 0;
}

int ocl_run(ocl_layer *layers, int n, int nsteps, double arrival_thr, int ngauges,
            const int *g_layer, const int *g_ki, const int *g_kj, const double *g_cx,
            const double *g_cy, REAL *ts) {
    return ocl_run_from(layers, n, 1, nsteps, arrival_thr, ngauges, g_layer, g_ki, g_kj, g_cx, g_cy, ts);
}

/* ------------------------------------------------------------------ */
/* set-up restatements                                                 */
/* ------------------------------------------------------------------ */
void ocl_pq_depth(int nx, int ny, const REAL *h, REAL *hp, REAL *hq) {
    /* PQ_DEPTH (initialization.f90:2501-2526); cells with H <= GX keep 0 */
    for (int j = 1; j <= ny; j++) {
        int jp1 = MIN(j + 1, ny);
        for (int i = 1; i <= nx; i++) {
            int ip1 = MIN(i + 1, nx);
            size_t c = (size_t)(j - 1) * nx + (i - 1);
            if (h[c] > R(CC_GX)) {
                hp[c] = R(0.5) * (h[c] + h[(size_t)(j - 1) * nx + (ip1 - 1)]);
                hq[c] = R(0.5) * (h[c] + h[(size_t)(jp1 - 1) * nx + (i - 1)]);
            } else {
                hp[c] = R(0);
                hq[c] = R(0);
            }
        }
    }
}

void ocl_para(int nx, int ny, int laygov, double dt, double dx_min, const double *lat,
              const double *del_y_min, const REAL *hp, const REAL *hq, REAL *r1, REAL *r11,
              REAL *r2, REAL *r3, REAL *r4, REAL *r5, REAL *r6) {
    /* PARA (comcot.f90:694-752), LAYGOV 0/1, in REAL arithmetic */
    REAL rr = R(dt) / R(CC_R_EARTH);
    REAL rs = R(CC_GRAV) * rr;
    REAL rt = R(0.5) * R(dt) * R(CC_CORI_W);
    REAL osixty = R(0.016666666667);
    REAL rad_deg = R(CC_RAD_DEG), rad_min = R(CC_RAD_MIN);
    for (int j = 1; j <= ny; j++) {
        REAL y = R(lat[j - 1]), dely = R(del_y_min[j - 1]);
        REAL ang_m = y * rad_deg;
        REAL ang_n = (y + R(0.5) * dely * osixty) * rad_deg;
        REAL cos_m, cos_n, sin_m, sin_n;
        if (sizeof(REAL) == sizeof(float)) {
            cos_m = (REAL)cosf((float)ang_m); cos_n = (REAL)cosf((float)ang_n);
            sin_m = (REAL)sinf((float)ang_m); sin_n = (REAL)sinf((float)ang_n);
        } else {
            cos_m = (REAL)cos((double)ang_m); cos_n = (REAL)cos((double)ang_n);
            sin_m = (REAL)sin((double)ang_m); sin_n = (REAL)sin((double)ang_n);
        }
        r1[j - 1] = rr / cos_m / (R(dx_min) * rad_min);
        r11[j - 1] = rr / cos_m / (dely * rad_min);
        r3[j - 1] = rt * sin_m;
        r5[j - 1] = rt * sin_n;
        r6[j - 1] = cos_n;
        for (int i = 1; i <= nx; i++) {
            size_t c = (size_t)(j - 1) * nx + (i - 1);
            if (laygov == 0) {
                r2[c] = rs / cos_m / (R(dx_min) * rad_min) * MAX(hp[c], R(0));
                r4[c] = rs / (dely * rad_min) * MAX(hq[c], R(0));
            } else {
                r2[c] = rs / cos_m / (R(dx_min) * rad_min);
                r4[c] = rs / (dely * rad_min);
            }
        }
    }
}

void ocl_para_nl(int ny, double dt, double dx_min, const double *lat, const double *del_y_min, REAL *r0,
                 REAL *r22) {
    /* R0 = RR/(DEL_Y*RAD_MIN), R22 = RR/COS_N/(DX*RAD_MIN) (comcot.f90:727,733) */
    REAL rr = R(dt) / R(CC_R_EARTH);
    REAL osixty = R(0.016666666667);
    REAL rad_deg = R(CC_RAD_DEG), rad_min = R(CC_RAD_MIN);
    for (int j = 1; j <= ny; j++) {
        REAL y = R(lat[j - 1]), dely = R(del_y_min[j - 1]);
        REAL ang_n = (y + R(0.5) * dely * osixty) * rad_deg;
        REAL cos_n = sizeof(REAL) == sizeof(float) ? (REAL)cosf((float)ang_n) : (REAL)cos((double)ang_n);
        r0[j - 1] = rr / (dely * rad_min);
        r22[j - 1] = rr / cos_n / (R(dx_min) * rad_min);
    }
}

int ocl_rel_time(double dt_parent, double dx_m, double dy_m, double hmax, int nonlinear,
                 double *dt_child) {
    /* CR_CHECK sub-level rule (initialization.f90:1210-1237) */
    REAL h_max = MAX(R(hmax), R(CC_GX));
    REAL cr_limit = nonlinear ? R(0.35) : R(0.5);
    REAL del_x = MIN(R(dx_m), R(dy_m));
    REAL dt = cr_limit * del_x / o_sqrt(R(CC_GRAV) * h_max);
    REAL dtp = R(dt_parent);
    if (dt >= dtp) {
        *dt_child = (double)dtp;
        return 1;
    }
    int ir = (int)floor((double)(dtp / dt)) + 1;
    *dt_child = (double)(dtp / R(ir));
    return ir;
}

void ocl_corners(int nx_p, const double *xp, int ny_p, const double *yp, double xs, double xe,
                 double ys, double ye, int *corners) {
    /* SUBGRID_MATCHING corner search (initialization.f90:913-936) */
    for (int k = 2; k <= nx_p - 1; k++) {
        REAL lo = (R(xp[k - 2]) + R(xp[k - 1])) / R(2), hi = (R(xp[k - 1]) + R(xp[k])) / R(2);
        if (R(xs) >= lo && R(xs) < hi) corners[0] = k + 1;
        if (R(xe) >= lo && R(xe) < hi) corners[1] = k - 1;
    }
    for (int k = 2; k <= ny_p - 1; k++) {
        REAL lo = (R(yp[k - 2]) + R(yp[k - 1])) / R(2), hi = (R(yp[k - 1]) + R(yp[k])) / R(2);
        if (R(ys) >= lo && R(ys) < hi) corners[2] = k + 1;
        if (R(ye) >= lo && R(ye) < hi) corners[3] = k - 1;
    }
}


/* ------------------------------------------------------------------ */
/* Okada (1985) seafloor deformation (deform.f90:74-240, 494-586)      */
/* ------------------------------------------------------------------ */
static inline REAL r_sin(REAL x) { return sizeof(REAL) == sizeof(float) ? (REAL)sinf((float)x) : (REAL)sin((double)x); }
static inline REAL r_cos(REAL x) { return sizeof(REAL) == sizeof(float) ? (REAL)cosf((float)x) : (REAL)cos((double)x); }
static inline REAL r_log(REAL x) { return sizeof(REAL) == sizeof(float) ? (REAL)logf((float)x) : (REAL)log((double)x); }
static inline REAL r_atan(REAL x) { return sizeof(REAL) == sizeof(float) ? (REAL)atanf((float)x) : (REAL)atan((double)x); }
static inline REAL r_asin(REAL x) { return sizeof(REAL) == sizeof(float) ? (REAL)asinf((float)x) : (REAL)asin((double)x); }
static inline REAL r_powr(REAL x, REAL y) {
    return sizeof(REAL) == sizeof(float) ? (REAL)powf((float)x, (float)y) : (REAL)pow((double)x, (double)y);
}
static inline int r_isnan(REAL x) { return x != x; }
static inline int r_isbig(REAL x) {
    REAL a = o_abs(x);
    return sizeof(REAL) == sizeof(float) ? (float)a >= 3.40282347e38f : (double)a >= 1.7976931348623157e308;
}

/* oblique stereographic projection on the WGS84 ellipsoid (Snyder 1987),
 * metres east / north of (lon0, lat0) */
void ocl_stereo(REAL lonin, REAL latin, REAL lon0, REAL lat0, REAL *xo, REAL *yo) {
    const REAL rad = R(CC_RAD_DEG);
    const REAL pole = R(CC_PI) / R(2.0) - R(CC_EPS);
    REAL lat = latin * rad, lon = lonin * rad, lt0 = lat0 * rad, ln0 = lon0 * rad;
    if (lat > pole) lat = pole;
    if (lat < -pole) lat = -pole;
    if (lt0 > pole) lt0 = pole;
    if (lt0 < -pole) lt0 = -pole;
    const REAL cs = r_cos(lat), sn = r_sin(lat), cs0 = r_cos(lt0), sn0 = r_sin(lt0);
    const REAL a = R(6378137.0), e = R(0.08181919092891), f2 = R(0.00669438000426), k0 = R(0.9996);
    const REAL tmp0 = o_sqrt(R(1.0) - f2 * (sn0 * sn0));
    (void)cs;
    const REAL rho0 = a * (R(1.0) - f2) / (tmp0 * tmp0 * tmp0);
    /* NU0 is not declared REAL in the reference (deform.f90:515-518, no
     * IMPLICIT NONE), so Fortran's implicit typing makes it an INTEGER and
     * the assignment truncates */
    const REAL nu0 = (REAL)(int)(a / tmp0);
    const REAL rr = o_sqrt(rho0 * nu0);
    const REAL c04 = (cs0 * cs0) * (cs0 * cs0);
    const REAL n = o_sqrt(R(1.0) + f2 * c04 / (R(1.0) - f2));
    const REAL s1 = (R(1.0) + sn0) / (R(1.0) - sn0);
    const REAL s2 = (R(1.0) - e * sn0) / (R(1.0) + e * sn0);
    const REAL w1 = r_powr(s1 * r_powr(s2, e), n);
    const REAL sn_xi0 = (w1 - R(1.0)) / (w1 + R(1.0));
    const REAL c = (n + sn0) * (R(1.0) - sn_xi0) / (n - sn0) / (R(1.0) + sn_xi0);
    const REAL w2 = c * w1;
    const REAL sa = (R(1.0) + sn) / (R(1.0) - sn);
    const REAL sb = (R(1.0) - e * sn) / (R(1.0) + e * sn);
    const REAL w = c * r_powr(sa * r_powr(sb, e), n);
    const REAL xi0 = r_asin((w2 - R(1.0)) / (w2 + R(1.0)));
    const REAL lm0 = ln0;
    const REAL lm = n * (lon - lm0) + lm0;
    const REAL xi = r_asin((w - R(1.0)) / (w + R(1.0)));
    const REAL beta = R(1.0) + r_sin(xi) * r_sin(xi0) + r_cos(xi) * r_cos(xi0) * r_cos(lm - lm0);
    *yo = R(0.0) + R(2.0) * rr * k0 * (r_sin(xi) * r_cos(xi0) - r_cos(xi) * r_sin(xi0) * r_cos(lm - lm0)) / beta;
    *xo = R(0.0) + R(2.0) * rr * k0 * r_cos(xi) * r_sin(lm - lm0) / beta;
}

/* STRIKE_SLIP (deform.f90:190-215) */
static REAL okada_ss(REAL y1, REAL y2, REAL q_x2, REAL dp, REAL dd) {
    const REAL sn = r_sin(dp), cs = r_cos(dp);
    const REAL q = q_x2 * sn - dd * cs;
    const REAL d_bar = y2 * sn - q * cs;
    const REAL r = o_sqrt(y1 * y1 + y2 * y2 + q * q);
    REAL t1 = r + d_bar, t2 = r + y2;
    if (t1 <= R(CC_EPS)) t1 = R(CC_EPS);
    if (t2 <= R(CC_EPS)) t2 = R(CC_EPS);
    const REAL a4 = R(0.5) / cs * (r_log(t1) - sn * r_log(t2));
    return -(d_bar * q / r / (r + y2) + q * sn / (r + y2) + a4 * sn) / R(2.0) / R(3.14159);
}

/* DIP_SLIP (deform.f90:218-236) */
static REAL okada_ds(REAL y1, REAL y2, REAL q_x2, REAL dp, REAL dd) {
    const REAL sn = r_sin(dp), cs = r_cos(dp);
    const REAL q = q_x2 * sn - dd * cs;
    const REAL d_bar = y2 * sn - q * cs;
    const REAL r = o_sqrt(y1 * y1 + y2 * y2 + q * q);
    const REAL xx = o_sqrt(y1 * y1 + q * q);
    const REAL a5 = R(1.0) / cs * r_atan((y2 * (xx + q * cs) + xx * (r + xx) * sn) / y1 / (r + xx) / cs);
    return -(d_bar * q / r / (r + y1) + sn * r_atan(y1 * y2 / q / r) - a5 * sn * cs) / R(2.0) / R(3.14159);
}

void ocl_okada(const ocl_fault *f, int laycord, int nx, int ny, const double *x, const double *y, double dx,
               double dy, REAL *deform) {
    const REAL rad = R(CC_RAD_DEG);
    const REAL ang_l = rad * R(f->dl), ang_r = rad * R(f->rd), ang_t = rad * R(f->th);
    const REAL halfl = R(0.5) * R(f->l), w = R(f->w);
    REAL hh = R(f->hh) + R(0.5) * w * r_sin(ang_l);
    REAL del_x = R(0.5) * w * r_cos(ang_l) * r_cos(ang_t);
    REAL del_y = R(0.5) * w * r_cos(ang_l) * r_sin(ang_t);
    if (f->sw == 9) {
        hh = R(f->hh) + w * r_sin(ang_l);
        del_x = w * r_cos(ang_l) * r_cos(ang_t);
        del_y = w * r_cos(ang_l) * r_sin(ang_t);
    }
    const REAL ds = R(f->d) * r_cos(ang_r), dd = R(f->d) * r_sin(ang_r);
    const REAL sn = r_sin(ang_l), cs = r_cos(ang_l);
    const REAL st = r_sin(ang_t), ct = r_cos(ang_t);
    REAL xl = 0, yl = 0;
    if (laycord != 0) ocl_stereo(R(f->xo), R(f->yo), R(f->x0), R(f->y0), &xl, &yl);
    for (int i = 1; i <= nx; i++) {
        for (int j = 1; j <= ny; j++) {
            REAL xs, ys;
            if (laycord == 0) {
                ocl_stereo(R(x[i - 1]), R(y[j - 1]), R(f->x0), R(f->y0), &xs, &ys);
                xs = xs - del_x;
                ys = ys + del_y;
            } else {
                /* deform.f90:150-154 as written: X = DX*(I-1) - XL, where XL is the
                 * layer origin's projected offset from the epicentre */
                const REAL yy = R(dy) * (R(j) - R(1.0)), xx = R(dx) * (R(i) - R(1.0));
                xs = xx - xl - del_x;
                ys = yy - yl + del_y;
            }
            const REAL x1 = xs * st + ys * ct;
            REAL x2 = xs * ct - ys * st;
            x2 = -x2;
            const REAL p = x2 * cs + hh * sn;
            const REAL f1 = okada_ss(x1 + halfl, p, x2, ang_l, hh);
            const REAL f2 = okada_ss(x1 + halfl, p - w, x2, ang_l, hh);
            const REAL f3 = okada_ss(x1 - halfl, p, x2, ang_l, hh);
            const REAL f4 = okada_ss(x1 - halfl, p - w, x2, ang_l, hh);
            const REAL g1 = okada_ds(x1 + halfl, p, x2, ang_l, hh);
            const REAL g2 = okada_ds(x1 + halfl, p - w, x2, ang_l, hh);
            const REAL g3 = okada_ds(x1 - halfl, p, x2, ang_l, hh);
            const REAL g4 = okada_ds(x1 - halfl, p - w, x2, ang_l, hh);
            REAL us = (f1 - f2 - f3 + f4) * ds;
            REAL ud = (g1 - g2 - g3 + g4) * dd;
            if (r_isbig(us)) us = 0;
            if (r_isbig(ud)) ud = 0;
            if (r_isnan(us)) us = 0;
            if (r_isnan(ud)) ud = 0;
            if (o_abs(us) <= R(CC_GX)) us = 0;
            if (o_abs(ud) <= R(CC_GX)) ud = 0;
            deform[(size_t)(j - 1) * nx + (i - 1)] = us + ud;
        }
    }
}

void ocl_okada_apply(const ocl_fault *f, int nf, int laycord, int nx, int ny, const double *x, const double *y,
                     double dx, double dy, REAL *z, REAL *h) {
    size_t n = (size_t)nx * ny;
    REAL *d = (REAL *)malloc(n * sizeof(REAL));
    if (!d) return;
    for (int k = 0; k < nf; k++) {
        ocl_okada(&f[k], laycord, nx, ny, x, y, dx, dy, d);
        for (size_t c = 0; c < n; c++) {
            z[c] = z[c] + d[c];
            h[c] = h[c] - d[c];
        }
    }
    free(d);
}

/* the shared deterministic elementary functions, exposed for their tests */
float ocl_expf(float x) { return cc_expf(x); }
float ocl_powf(float x, float y) { return cc_powf(x, y); }
