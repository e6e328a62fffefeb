/*
 * Fused linear-spherical time step for sm_100a.
 *
 * One pass over the grid performs, per cell, what the reference runs as
 * separate synchronised launches: MASS_S (mass.f90:61-100), the OPEN
 * radiation boundary on the outermost layer (boundaries.f90:22-202),
 * MOMT_S (moment.f90:65-149), the maximum-amplitude recorder
 * (GPUOutput.cu:46-53), the arrival-step record, and the gauge sampling of
 * the previous step (GET_TS, output.f90:1078-1090).
 *
 * Work decomposition: a CTA owns a TX x TY tile (I x J).  Its TX threads
 * march up the tile's rows; at row r they stage row r of M1, N1, H in a
 * four-row shared-memory ring, compute the new surface Z2 of row r (with a
 * one-column halo on the right), then the momentum of row r-1, which needs
 * Z2 of rows r-1 and r.  The halo row/column of Z2 is recomputed from the
 * same inputs by both neighbouring tiles, bit-identically.  Per cell the
 * kernel streams Z1, M1, N1, H in and Z2, M2, N2 out (28 bytes) plus the
 * 8-byte max-amplitude read/write; R2 and R4 are rebuilt from H and the
 * per-row factors instead of being streamed.
 *
 * Arithmetic is evaluated in the Fortran order with separately rounded
 * float operations (the library is built with -fmad=false).
 */
#include "fused.h"

namespace {

template <int TX>
struct FusedSmem {
    float m[4][TX + 2]; /* column c+1 <-> I = i0 + c; column 0 is i0-1 */
    float n[4][TX + 1];
    float h[4][TX + 1];
    float z[4][TX + 1];
};

__device__ __forceinline__ float fabs_(float x) { return x < 0.0f ? -x : x; }

__device__ __forceinline__ float ld_row(const float *__restrict__ a, int i, int nx, size_t roff) {
    return (i < nx) ? __ldg(a + roff + i) : 0.0f;
}

/* OPEN on a perimeter cell, from the staged rows (boundaries.f90:42-200) */
__device__ __forceinline__ float open_from_smem(int i, int j, int nx, int ny, float h, float hs,
                                                float m, float mw, float n, float ns) {
    if (!(h > CC_GX)) return 0.0f;
    float cc = sqrtf(CC_GRAV * h);
    float zz;
    bool corner = (i == 0 || i == nx - 1) && (j == 0 || j == ny - 1);
    if (!corner) {
        if (j == 0) {
            float uh = 0.5f * (m + mw);
            float uu = sqrtf(uh * uh + n * n);
            zz = uu / cc;
            if (n > 0.0f) zz = -zz;
        } else if (j == ny - 1) {
            float uh = 0.5f * (m + mw);
            float uu = sqrtf(uh * uh + ns * ns);
            zz = uu / cc;
            if (ns < 0.0f) zz = -zz;
        } else if (i == 0) {
            float uh = (hs > CC_GX) ? 0.5f * (n + ns) : n;
            float uu = sqrtf(uh * uh + m * m);
            zz = uu / cc;
            if (m > 0.0f) zz = -zz;
        } else {
            float uh = 0.5f * (n + ns);
            float uu = sqrtf(uh * uh + mw * mw);
            zz = uu / cc;
            if (mw < 0.0f) zz = -zz;
        }
    } else {
        float qx = (i == 0) ? m : mw;
        float qy = (j == 0) ? n : ns;
        float uh = sqrtf(qx * qx + qy * qy);
        zz = uh / cc;
        bool neg;
        if (i == 0 && j == 0) neg = (qx > 0.0f || qy > 0.0f);
        else if (j == 0) neg = (qx < 0.0f || qy > 0.0f);
        else if (i == 0) neg = (qx > 0.0f || qy < 0.0f);
        else neg = (qx < 0.0f || qy < 0.0f);
        if (neg) zz = -zz;
    }
    if (fabs_(zz) > CC_UB) zz = 0.0f;
    return zz;
}

template <int TX, int TY>
__device__ __forceinline__ void fused_tile(const GcFusedGrid &G, int lt, int step,
                                           FusedSmem<TX> &S) {
    const int t = threadIdx.x;
    const int nx = G.nx, ny = G.ny;
    const size_t P = (size_t)G.pitch;
    const int tx = lt % G.tiles_x, ty = lt / G.tiles_x;
    const int i0 = tx * TX, j0 = ty * TY;
    const int local = step - G.step0; /* 0-based index of the step being computed */
    if (local < 0 || local > G.nsteps) return;
    const int cur = G.cur0 ^ (local & 1);
    const float *__restrict__ z1 = G.z[cur];
    const float *__restrict__ m1 = G.m[cur];
    const float *__restrict__ n1 = G.n[cur];
    float *__restrict__ z2 = G.z[cur ^ 1];
    float *__restrict__ m2 = G.m[cur ^ 1];
    float *__restrict__ n2 = G.n[cur ^ 1];
    const float *__restrict__ hh = G.h;
    const float *__restrict__ rows = G.rows;
    const bool root = G.root != 0;
    const int i = i0 + t;

    /* gauges: sample the surface the previous step left (its Z2 is our Z1) */
    if (lt == 0 && G.ng > 0) {
        int prev = local - 1;
        if (prev >= 0 && prev < G.ts_len) {
            for (int g = t; g < G.ng; g += TX) {
                int ki = G.gij[2 * g] - 1, kj = G.gij[2 * g + 1] - 1;
                size_t c = (size_t)kj * P + ki;
                float l1 = z1[c], l2 = z1[c + 1], l3 = z1[c + P], l4 = z1[c + P + 1];
                float cx = G.gw[2 * g], cy = G.gw[2 * g + 1];
                float a = l1 * (1.0f - cx) * (1.0f - cy);
                float b = l2 * (cx) * (1.0f - cy);
                float d = l3 * (1.0f - cx) * (cy);
                float e = l4 * (cx) * (cy);
                G.ts[(size_t)prev * G.ng + g] = a + b + d + e;
            }
        }
    }

    if (local >= G.nsteps) return; /* finished: only the last gauge sample */

    /* prologue: row max(j0-1,0) of N and H */
    {
        const int jr = j0 > 0 ? j0 - 1 : 0;
        const int s = (j0 - 1) & 3;
        const size_t ro = (size_t)jr * P;
        S.n[s][t] = ld_row(n1, i, nx, ro);
        S.h[s][t] = ld_row(hh, i, nx, ro);
        if (t == 0) {
            S.n[s][TX] = ld_row(n1, i0 + TX, nx, ro);
            S.h[s][TX] = ld_row(hh, i0 + TX, nx, ro);
        }
    }

    /* prefetch row j0 into registers */
    float pm = 0.f, pn = 0.f, ph = 0.f, pz = 0.f, pmw = 0.f, pme = 0.f, pne = 0.f, phe = 0.f, pze = 0.f;
#define GC_FETCH(R_)                                                   \
    if ((R_) < ny) {                                                   \
        const size_t ro_ = (size_t)(R_) * P;                           \
        pm = ld_row(m1, i, nx, ro_);                                   \
        pn = ld_row(n1, i, nx, ro_);                                   \
        ph = ld_row(hh, i, nx, ro_);                                   \
        pz = ld_row(z1, i, nx, ro_);                                   \
        if (t == 0) {                                                  \
            pmw = ld_row(m1, i0 > 0 ? i0 - 1 : 0, nx, ro_);            \
            pme = ld_row(m1, i0 + TX, nx, ro_);                        \
            pne = ld_row(n1, i0 + TX, nx, ro_);                        \
            phe = ld_row(hh, i0 + TX, nx, ro_);                        \
            pze = ld_row(z1, i0 + TX, nx, ro_);                        \
        }                                                              \
    }
    GC_FETCH(j0)

    for (int r = j0; r <= j0 + TY; r++) {
        const bool rv = r < ny;
        const int s = r & 3, sp = (r - 1) & 3;
        float zc = pz, zce = pze;
        if (rv) {
            S.m[s][t + 1] = pm;
            S.n[s][t] = pn;
            S.h[s][t] = ph;
            if (t == 0) {
                S.m[s][0] = pmw;
                S.m[s][TX + 1] = pme;
                S.n[s][TX] = pne;
                S.h[s][TX] = phe;
            }
        }
        GC_FETCH(r + 1) /* next row's loads overlap this row's compute */
        __syncthreads();
        if (rv) {
            /* new surface of row r: TX owned columns + one halo column */
            const float r1 = rows[GC_R1 * (size_t)ny + r];
            const float r11 = rows[GC_R11 * (size_t)ny + r];
            const float r6 = rows[GC_R6 * (size_t)ny + r];
            const float r6m = r > 0 ? rows[GC_R6 * (size_t)ny + r - 1] : 0.0f;
            for (int k = 0; k < (t == 0 ? 2 : 1); k++) {
                const int c = (k == 0) ? t : TX;
                const int ic = i0 + c;
                if (ic >= nx) continue;
                const float z1v = (k == 0) ? zc : zce;
                const float h = S.h[s][c];
                float zn;
                if (root && (ic == 0 || ic == nx - 1 || r == 0 || r == ny - 1)) {
                    zn = open_from_smem(ic, r, nx, ny, h, S.h[sp][c], S.m[s][c + 1], S.m[s][c],
                                        S.n[s][c], S.n[sp][c]);
                } else if (!root && (ic == 0 || r == 0)) {
                    zn = z1v;
                } else if (h > CC_GX) {
                    float zz = z1v - r1 * (S.m[s][c + 1] - S.m[s][c])
                               - r11 * (S.n[s][c] * r6 - S.n[sp][c] * r6m);
                    if (fabs_(zz) < CC_EPS) zz = 0.0f;
                    if ((zz + h) <= CC_EPS) zz = -h;
                    zn = zz;
                } else {
                    zn = 0.0f;
                }
                S.z[s][c] = zn;
                if (k == 0 && r < j0 + TY) {
                    const size_t cell = (size_t)r * P + ic;
                    z2[cell] = zn;
                    if (G.flags & GC_F_MAXAMP) {
                        float zm = G.zmax[cell];
                        if (!(zm >= zn)) G.zmax[cell] = zn;
                    }
                    if ((G.flags & GC_F_ARRIVAL) && zn > G.thr && h > CC_GX) {
                        if (G.arrival[cell] < 0) G.arrival[cell] = local + 1;
                    }
                }
            }
        }
        __syncthreads();
        /* momentum of row j = r-1 */
        const int j = r - 1;
        if (j >= j0 && j < ny && i < nx) {
            const int a = j & 3, b = (j + 1) & 3, cm = j > 0 ? ((j - 1) & 3) : a;
            const size_t cell = (size_t)j * P + i;
            const int c = t;
            float xm = 0.0f;
            const bool mdom = root ? (i <= nx - 2) : (i >= 1 && i <= nx - 2 && j >= 1);
            if (mdom) {
                float h = S.h[a][c], hp1 = S.h[a][c + 1];
                if (h > CC_GX && hp1 > CC_GX) {
                    float tot_n = S.n[a][c] + S.n[a][c + 1] + S.n[cm][c] + S.n[cm][c + 1];
                    float r2 = G.explicit_r24 ? G.r2[cell]
                                              : rows[GC_CX * (size_t)ny + j] * (0.5f * (h + hp1));
                    xm = S.m[a][c + 1] - r2 * (S.z[a][c + 1] - S.z[a][c])
                         + rows[GC_R3 * (size_t)ny + j] * tot_n;
                    if (fabs_(xm) < CC_EPS) xm = 0.0f;
                }
            }
            m2[cell] = xm;
            float xn = 0.0f;
            const bool ndom = root ? (j <= ny - 2) : (i >= 1 && j >= 1 && j <= ny - 2);
            if (ndom) {
                float h = S.h[a][c], hq1 = S.h[b][c];
                if (h > CC_GX && hq1 > CC_GX) {
                    float tot_m = S.m[a][c] + S.m[b][c] + S.m[a][c + 1] + S.m[b][c + 1];
                    float r4 = G.explicit_r24 ? G.r4[cell]
                                              : rows[GC_CY * (size_t)ny + j] * (0.5f * (h + hq1));
                    xn = S.n[a][c] - r4 * (S.z[b][c] - S.z[a][c])
                         - rows[GC_R5 * (size_t)ny + j] * tot_m;
                    if (fabs_(xn) < CC_EPS) xn = 0.0f;
                }
            }
            n2[cell] = xn;
        }
    }
    __syncthreads(); /* the next tile reuses the ring */
#undef GC_FETCH
}

template <int TX, int TY, bool MULTI>
__global__ void __launch_bounds__(TX) k_fused(GcFusedGrid one, const GcFusedGrid *__restrict__ grids,
                                              const int2 *__restrict__ tiles, int ntiles,
                                              const int *__restrict__ step_base, int step_off) {
    __shared__ FusedSmem<TX> S;
    const int step = step_off + (step_base ? *step_base : 0);
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        if (MULTI) {
            const int2 w = tiles[tile];
            fused_tile<TX, TY>(grids[w.x], w.y, step, S);
        } else {
            fused_tile<TX, TY>(one, tile, step, S);
        }
    }
}

struct Variant {
    int tx, ty;
    void (*one)(GcFusedGrid, const GcFusedGrid *, const int2 *, int, const int *, int);
    void (*multi)(GcFusedGrid, const GcFusedGrid *, const int2 *, int, const int *, int);
};

#define GC_VARIANT(TX, TY) {TX, TY, k_fused<TX, TY, false>, k_fused<TX, TY, true>}
const Variant kVariants[] = {
    GC_VARIANT(128, 16), GC_VARIANT(128, 32), GC_VARIANT(128, 64),
    GC_VARIANT(256, 16), GC_VARIANT(256, 32), GC_VARIANT(64, 32),
};
#undef GC_VARIANT
constexpr int kNumVariants = sizeof(kVariants) / sizeof(kVariants[0]);

} // namespace

int gc_fused_num_variants() { return kNumVariants; }

GcTileCfg gc_fused_variant(int v) {
    if (v < 0 || v >= kNumVariants) v = 0;
    return GcTileCfg{kVariants[v].tx, kVariants[v].ty};
}

int gc_fused_tiles(int variant, int nx, int ny, int *tiles_x) {
    GcTileCfg c = gc_fused_variant(variant);
    int tx = (nx + c.tx - 1) / c.tx, ty = (ny + c.ty - 1) / c.ty;
    if (tiles_x) *tiles_x = tx;
    return tx * ty;
}

cudaError_t gc_fused_launch_one(int variant, const GcFusedGrid &g, int step, cudaStream_t s) {
    if (variant < 0 || variant >= kNumVariants) variant = 0;
    const Variant &v = kVariants[variant];
    int ntiles = gc_fused_tiles(variant, g.nx, g.ny, nullptr);
    v.one<<<ntiles, v.tx, 0, s>>>(g, nullptr, nullptr, ntiles, nullptr, step);
    return cudaGetLastError();
}

int gc_fused_max_ctas(int variant) {
    if (variant < 0 || variant >= kNumVariants) variant = 0;
    const Variant &v = kVariants[variant];
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, v.multi, v.tx, 0);
    return sms * (per > 0 ? per : 1);
}

cudaError_t gc_fused_launch_multi(int variant, const GcFusedGrid *d_grids, const int2 *d_tiles,
                                  int ntiles, const int *d_step_base, int step_off, int nctas,
                                  cudaStream_t s) {
    if (variant < 0 || variant >= kNumVariants) variant = 0;
    const Variant &v = kVariants[variant];
    if (ntiles <= 0) return cudaSuccess;
    if (nctas <= 0 || nctas > ntiles) nctas = ntiles;
    GcFusedGrid dummy;
    memset(&dummy, 0, sizeof dummy);
    v.multi<<<nctas, v.tx, 0, s>>>(dummy, d_grids, d_tiles, ntiles, d_step_base, step_off);
    return cudaGetLastError();
}
