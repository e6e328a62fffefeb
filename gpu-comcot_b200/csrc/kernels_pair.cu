/*
 * Two linear-spherical time steps per pass over HBM, for sm_100a.
 *
 * One launch advances every grid of a work list by two outer steps: MASS_S
 * (mass.f90:61-100), the OPEN radiation boundary of the outermost layer
 * (boundaries.f90:22-202) and MOMT_S (moment.f90:65-149) at step A, then the
 * same again at step B on step A's results, with the maximum-amplitude
 * recorder (GPUOutput.cu:46-53) and the arrival record after each of them and
 * the gauge samples (GET_TS, output.f90:1078-1090) of both surfaces.  Step A's
 * surface and fluxes never leave the chip, so a step moves half the bytes of
 * the one-step kernel (kernels_fused.cu): per cell and launch Z1, M1, N1, H
 * and max-eta are read and Z3, M3, N3 and max-eta written, 36 bytes for two
 * steps.
 *
 * Work decomposition: a warp computes a strip of 128 columns (lane l owns
 * the four columns s+4l .. s+4l+3, as a float4) and marches down its rows.
 * Every stencil neighbour along I is a warp shuffle of the adjacent lane's
 * float4, so each lane reads only its own 16 bytes of a row: no halo loads,
 * no shared-memory bank conflicts.  A step's results are exact only where all
 * their inputs were, which loses at most two columns at each side of the
 * strip per step; tiles therefore overlap, and a tile stores only its middle
 * 120 columns (lanes 1..30).  At the grid's west and east edges no halo is
 * needed (the perimeter cells use OPEN and the IM1 clamp, which read nothing
 * beyond the edge), so the first tile stores 124 columns from column 0 and
 * the last one runs to the grid's last column.  Along J, step B at output row
 * j needs step A at rows j-1 .. j+2, and step A at row j needs the inputs of
 * rows j-1 .. j+1: a tile of TY output rows reads rows j0-2 .. j0+TY+1.
 *
 * Each row's Z1, M1, N1, H, max-eta and 32-byte coefficient record arrive by
 * 1-D bulk copies (cp.async.bulk, completing on an mbarrier) into an S-stage
 * shared-memory ring private to the warp; a stage is read into registers as
 * soon as it lands and refilled with the row S ahead.  What later rows need
 * of earlier ones (step A's surface and fluxes of the two previous rows, step
 * B's of the previous one) is carried in registers.
 *
 * Ping-pong: the engine keeps three time levels per member, level L in
 * buffer L % 3, so a launch reading level L writes level L + 2 to a buffer no
 * tile reads (the one-step kernel writes L + 1 the same way).  Level L + 1 is
 * never stored.
 *
 * Every pipeline wait is bounded by the `wait_limit` launch parameter; a wait
 * that gives up sets g_pair_error and the warp leaves once its copies in
 * flight have landed (or a second bounded wait expired).  `stall` != 0 makes
 * the first warp of the launch expect 16 bytes that no copy delivers on its
 * first row (nothing is issued for that row), so a test can watch the bound
 * work without any copy left in flight.
 *
 * Arithmetic follows the Fortran order with separately rounded float
 * operations (the library is built with -fmad=false); both steps give the
 * bits of two launches of the one-step kernel.
 */
#include "bulk_pipe.cuh"
#include "fused.h"
#include "open_bd.cuh"

namespace {

using namespace gcpipe;

constexpr unsigned FULL = 0xffffffffu;
constexpr int kPairOut = 120; /* columns an interior tile stores */

__device__ int g_pair_error; /* set when a pipeline wait gave up */

/* one stage holds one row of a warp strip (byte offsets) */
struct PStage {
    static constexpr int Z = 0, M = 512, N = 1024, H = 1536, X = 2048, C = 2560;
    static constexpr int BYTES = 2688; /* 2592 rounded up to 128 */
};

template <int S>
__host__ __device__ constexpr int pair_warp_bytes() {
    return (S * PStage::BYTES + S * 8 + 127) / 128 * 128;
}

__device__ __forceinline__ float shw(float v) { return __shfl_up_sync(FULL, v, 1); }   /* lane - 1 */
__device__ __forceinline__ float she(float v) { return __shfl_down_sync(FULL, v, 1); } /* lane + 1 */
__device__ __forceinline__ float comp(const float4 &v, int q) {
    return q == 0 ? v.x : (q == 1 ? v.y : (q == 2 ? v.z : v.w));
}
__device__ __forceinline__ float4 lds4(const char *p) { return *reinterpret_cast<const float4 *>(p); }

/* OPEN on a perimeter cell of the outermost layer (open_bd.cuh) */
using gcopen::open_cell;

/* MASS_S at one cell (mass.f90:82-95) */
__device__ __forceinline__ float mass1(float z1, float m, float mw, float n, float ns, float h, float r1, float r11,
                                       float r6, float r6m) {
    float zz = z1 - r1 * (m - mw) - r11 * (n * r6 - ns * r6m);
    zz = (fabsf(zz) < CC_EPS) ? 0.0f : zz;
    zz = ((zz + h) <= CC_EPS) ? -h : zz;
    return (h > CC_GX) ? zz : 0.0f;
}

/* the new surface of a lane's four cells at row r: OPEN on the perimeter
 * (EDGE), MASS_S elsewhere.  mw: M at the column left of the first cell;
 * ns, hs: N and H of row r-1 */
template <bool EDGE>
__device__ __forceinline__ float4 surface4(const float4 &z1, const float4 &m, float mw, const float4 &n,
                                           const float4 &ns, const float4 &h, const float4 &hs, float r1, float r11,
                                           float r6, float r6m, int ib, int r, int nx, int ny) {
    const float mv[4] = {m.x, m.y, m.z, m.w}, nv[4] = {n.x, n.y, n.z, n.w}, nsv[4] = {ns.x, ns.y, ns.z, ns.w};
    const float hv[4] = {h.x, h.y, h.z, h.w}, hsv[4] = {hs.x, hs.y, hs.z, hs.w}, zv[4] = {z1.x, z1.y, z1.z, z1.w};
    float o[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const float w = q == 0 ? mw : mv[q - 1];
        if constexpr (EDGE) {
            const int i = ib + q;
            if (i == 0 || i == nx - 1 || r == 0 || r == ny - 1)
                o[q] = open_cell(i, r, nx, ny, hv[q], hsv[q], mv[q], w, nv[q], nsv[q]);
            else
                o[q] = mass1(zv[q], mv[q], w, nv[q], nsv[q], hv[q], r1, r11, r6, r6m);
        } else {
            o[q] = mass1(zv[q], mv[q], w, nv[q], nsv[q], hv[q], r1, r11, r6, r6m);
        }
    }
    return make_float4(o[0], o[1], o[2], o[3]);
}

/* MOMT_S, x direction, at row j (moment.f90:86-115): M' from M, the surface
 * of row j and its east neighbour ze, N of rows j (nb) and j-1 (nc) with
 * their east neighbours, H of row j with its east neighbour.  mdom: the
 * domain test of the outer layer (I <= NX-1). */
template <bool EDGE>
__device__ __forceinline__ float4 flux_m4(const float4 &m, const float4 &z, float ze, const float4 &nb, float nbe,
                                          const float4 &nc, float nce, const float4 &h, float he, float cx, float r3,
                                          int ib, int nx) {
    const float mv[4] = {m.x, m.y, m.z, m.w};
    const float zv[5] = {z.x, z.y, z.z, z.w, ze}, nbv[5] = {nb.x, nb.y, nb.z, nb.w, nbe};
    const float ncv[5] = {nc.x, nc.y, nc.z, nc.w, nce}, hv[5] = {h.x, h.y, h.z, h.w, he};
    float o[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const float h0 = hv[q], hp1 = hv[q + 1];
        const float tot_n = nbv[q] + nbv[q + 1] + ncv[q] + ncv[q + 1];
        const float r2 = cx * (0.5f * (h0 + hp1));
        float vm = mv[q] - r2 * (zv[q + 1] - zv[q]) + r3 * tot_n;
        vm = (fabsf(vm) < CC_EPS) ? 0.0f : vm;
        bool dom = true;
        if constexpr (EDGE) dom = ib + q <= nx - 2;
        o[q] = (dom && h0 > CC_GX && hp1 > CC_GX) ? vm : 0.0f;
    }
    return make_float4(o[0], o[1], o[2], o[3]);
}

/* MOMT_S, y direction, at row j (moment.f90:117-145): N' from N of row j, the
 * surfaces of rows j+1 (za) and j (zb), M of rows j (mb) and j+1 (ma) with
 * their west neighbours, H of rows j and j+1.  ndom: J <= NY-1 and I <= NX. */
template <bool EDGE>
__device__ __forceinline__ float4 flux_n4(const float4 &n, const float4 &za, const float4 &zb, const float4 &mb,
                                          float mbw, const float4 &ma, float maw, const float4 &h, const float4 &ha,
                                          float cy, float r5, int ib, int j, int nx, int ny) {
    const float nv[4] = {n.x, n.y, n.z, n.w}, zav[4] = {za.x, za.y, za.z, za.w}, zbv[4] = {zb.x, zb.y, zb.z, zb.w};
    const float mbv[5] = {mbw, mb.x, mb.y, mb.z, mb.w}, mav[5] = {maw, ma.x, ma.y, ma.z, ma.w};
    const float hv[4] = {h.x, h.y, h.z, h.w}, hav[4] = {ha.x, ha.y, ha.z, ha.w};
    float o[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const float tot_m = mbv[q] + mav[q] + mbv[q + 1] + mav[q + 1];
        const float r4 = cy * (0.5f * (hv[q] + hav[q]));
        float vn = nv[q] - r4 * (zav[q] - zbv[q]) - r5 * tot_m;
        vn = (fabsf(vn) < CC_EPS) ? 0.0f : vn;
        bool dom = true;
        if constexpr (EDGE) dom = j <= ny - 2 && ib + q < nx;
        o[q] = (dom && hv[q] > CC_GX && hav[q] > CC_GX) ? vn : 0.0f;
    }
    return make_float4(o[0], o[1], o[2], o[3]);
}

/* max-eta: keeps the old value unless the new surface is above it */
__device__ __forceinline__ float4 max4(const float4 &x, const float4 &z) {
    return make_float4(x.x >= z.x ? x.x : z.x, x.y >= z.y ? x.y : z.y, x.z >= z.z ? x.z : z.z,
                       x.w >= z.w ? x.w : z.w);
}

/* arrival by max-eta: a wet cell above the threshold whose maximum before
 * this step was not arrives at `step` */
__device__ __forceinline__ void arrive4(int *row, int ib, int lo, int hi, const float4 &z, const float4 &xo,
                                        const float4 &h, float thr, int step) {
    const float zv[4] = {z.x, z.y, z.z, z.w}, xv[4] = {xo.x, xo.y, xo.z, xo.w}, hv[4] = {h.x, h.y, h.z, h.w};
#pragma unroll
    for (int q = 0; q < 4; q++)
        if (ib + q >= lo && ib + q <= hi && zv[q] > thr && hv[q] > CC_GX && xv[q] <= thr) row[ib + q] = step;
}

/* whether any of a lane's four cells can arrive at this step: a surface
 * above the threshold, and a maximum before the step at or below it (a cell
 * whose maximum already exceeds the threshold arrived before).  A lane this
 * returns false for would store nothing in arrive4. */
__device__ __forceinline__ bool may_arrive(const float4 &z, const float4 &xo, float thr) {
    return fmaxf(fmaxf(z.x, z.y), fmaxf(z.z, z.w)) > thr && fminf(fminf(xo.x, xo.y), fminf(xo.z, xo.w)) <= thr;
}

/* store of a lane's four cells, masked to columns [lo, hi] */
__device__ __forceinline__ void st4m(float *row, int ib, int lo, int hi, const float4 &v) {
    if (ib >= lo && ib + 3 <= hi) {
        *reinterpret_cast<float4 *>(row + ib) = v;
    } else if (ib + 3 >= lo && ib <= hi) {
        const float vv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int q = 0; q < 4; q++)
            if (ib + q >= lo && ib + q <= hi) row[ib + q] = vv[q];
    }
}

/* the 2x2 surface stencil at column ki (0-based) of a strip starting at s,
 * from two rows held as float4 per lane (every lane takes part) */
__device__ __forceinline__ void gauge_stencil(const float4 &lo_row, const float4 &hi_row, int ki, int s, float &l1,
                                              float &l2, float &l3, float &l4) {
    const int c0 = ki - s, c1 = ki + 1 - s;
    l1 = __shfl_sync(FULL, comp(lo_row, c0 & 3), c0 >> 2);
    l2 = __shfl_sync(FULL, comp(lo_row, c1 & 3), c1 >> 2);
    l3 = __shfl_sync(FULL, comp(hi_row, c0 & 3), c0 >> 2);
    l4 = __shfl_sync(FULL, comp(hi_row, c1 & 3), c1 >> 2);
}

/* one gauge sample from two rows held as float4 per lane (GET_TS weights) */
__device__ __forceinline__ float gauge_sample(const float4 &lo_row, const float4 &hi_row, int ki, int s, float cx,
                                              float cy) {
    float l1, l2, l3, l4;
    gauge_stencil(lo_row, hi_row, ki, s, l1, l2, l3, l4);
    const float a = l1 * (1.0f - cx) * (1.0f - cy);
    const float b = l2 * (cx) * (1.0f - cy);
    const float d = l3 * (1.0f - cx) * (cy);
    const float e = l4 * (cx) * (cy);
    return a + b + d + e;
}

/* tile geometry along I: tile t computes columns [s, s+127] and stores
 * [lo, hi] (0-based, clipped to the grid) */
__host__ __device__ __forceinline__ void pair_cols(int t, int nx, int &s, int &lo, int &hi) {
    s = t == 0 ? 0 : kPairOut * t;
    lo = t == 0 ? 0 : s + 4;
    hi = s + 123;
    if (hi + 4 >= nx - 1) hi = nx - 1; /* the last tile runs to the grid's edge */
    if (hi > nx - 1) hi = nx - 1;
}

/* Tile layout of one grid.  Strips are 128 columns (pair_cols).  With
 * te == 0 every tile is ty rows, in row-major order.  With te > 0 the tiles
 * that carry the boundary (OPEN, the IM1/JM1 clamps) and so cost more per
 * row are shorter: the west strip's tiles and the other strips' first and
 * last tile rows take te rows, the east strip's tee = 5/6 te rows (its OPEN
 * column sits at a cell chosen at run time, a few selects dearer).  The edge
 * strips' tiles come first in the order.  Grids of at most two strips, or
 * too few rows, use te == 0. */
struct PairLayout {
    int tiles_x, ty, te, tee;
    int n_w, n_e; /* tiles of the west and east strips */
    int n_mid;    /* ty-row tiles of another strip */
    int count;
};
__host__ __device__ __forceinline__ PairLayout pair_layout(int nx, int ny, int ty, int te) {
    PairLayout L;
    L.tiles_x = nx <= 128 ? 1 : 1 + (nx - 128 + kPairOut - 1) / kPairOut;
    L.ty = ty;
    L.te = (te > 0 && te < ty && L.tiles_x > 2 && ny >= 2 * te + ty) ? te : 0;
    L.tee = L.te > 0 ? max(1, (5 * L.te + 3) / 6) : 0;
    if (L.te == 0) {
        L.n_w = L.n_e = 0;
        L.n_mid = (ny + ty - 1) / ty;
        L.count = L.tiles_x * L.n_mid;
    } else {
        L.n_w = (ny + L.te - 1) / L.te;
        L.n_e = (ny + L.tee - 1) / L.tee;
        L.n_mid = (ny - 2 * L.te + ty - 1) / ty;
        L.count = L.n_w + L.n_e + (L.tiles_x - 2) * (L.n_mid + 2);
    }
    return L;
}
/* tile lt of a layout: strip tx, first output row j0, rows h (the body
 * clips the last tile of a strip to the grid) */
__host__ __device__ __forceinline__ void pair_tile_at(const PairLayout &L, int ny, int lt, int &tx, int &j0, int &h) {
    if (L.te == 0) {
        tx = lt % L.tiles_x;
        j0 = (lt / L.tiles_x) * L.ty;
        h = L.ty;
        return;
    }
    if (lt < L.n_w) {
        tx = 0;
        j0 = lt * L.te;
        h = L.te;
        return;
    }
    if (lt < L.n_w + L.n_e) {
        tx = L.tiles_x - 1;
        j0 = (lt - L.n_w) * L.tee;
        h = L.tee;
        return;
    }
    const int k = lt - L.n_w - L.n_e;
    tx = 1 + k % (L.tiles_x - 2);
    const int b = k / (L.tiles_x - 2);
    if (b == 0) {
        j0 = 0;
        h = L.te;
    } else if (b <= L.n_mid) {
        j0 = L.te + (b - 1) * L.ty;
        h = min(L.ty, ny - L.te - j0);
    } else {
        j0 = ny - L.te;
        h = L.te;
    }
}

/* what one warp needs to run its ring of S stages over a tile's rows */
struct PairRing {
    char *wsm;      /* the warp's stages (generic address) */
    uint32_t wbase; /* the same in the shared window */
    uint32_t bars;  /* the stages' mbarriers */
    int seq0;       /* ring position of the tile's first row */
};

/* copies of input row r of a strip (columns s .. s + cb/4 - 1) into the stage
 * at sb: Z, M, N of the level read, H, max-eta on output rows (out), and the
 * row's coefficient record.  `fake`: announce 16 bytes no copy delivers. */
template <class Desc>
__device__ __forceinline__ void pair_issue(const Desc &G, int l0, int r, int s, uint32_t cb, bool out,
                                           uint32_t sb, uint32_t bar, bool fake) {
    fence_proxy_async(); /* the warp's reads of this stage come first */
    if (fake) {
        mbar_expect_tx(bar, 16u);
        return;
    }
    mbar_expect_tx(bar, (out ? 5u : 4u) * cb + 32u);
    const size_t ro = (size_t)r * (size_t)G.pitch + s;
    bulk_g2s(sb + PStage::Z, G.z[l0] + ro, cb, bar);
    bulk_g2s(sb + PStage::M, G.m[l0] + ro, cb, bar);
    bulk_g2s(sb + PStage::N, G.n[l0] + ro, cb, bar);
    bulk_g2s(sb + PStage::H, G.h + ro, cb, bar);
    if (out) bulk_g2s(sb + PStage::X, G.zmax + ro, cb, bar);
    bulk_g2s(sb + PStage::C, G.rows + (size_t)r * GC_ROWW, 32u, bar);
}

/* the first min(S, K) rows of a tile (rows rs ..), issued by lane 0 */
template <int S, class Desc>
__device__ __forceinline__ void pair_prologue(const Desc &G, const PairRing &R, int l0, int rs, int K,
                                              int j0, int jl, int s, uint32_t cb, bool stall) {
    __syncwarp();
    if ((threadIdx.x & 31) == 0) {
        const int kk = min(S, K);
        for (int k = 0; k < kk; k++) {
            const int st = (R.seq0 + k) % S, r = rs + k;
            pair_issue(G, l0, r, s, cb, r >= j0 && r <= jl, R.wbase + st * PStage::BYTES, R.bars + 8 * st,
                       stall && k == 0);
        }
    }
}

/* gauges whose base cell (KI, KJ) lies in the tile's stored block: bit g of
 * (gm1:gm0).  Also writes the sample of the surface the previous launch left
 * (level L, step local - 1), which no tile of that launch could take. */
template <class Desc>
__device__ __forceinline__ void pair_gauge_setup(const Desc &G, int l0, int local, int lo, int hi, int j0,
                                                 int jl, unsigned &gm0, unsigned &gm1) {
    const int lane = threadIdx.x & 31;
    const int ng = G.ng;
    gm0 = gm1 = 0;
    if (ng <= 0) return;
    const size_t P = (size_t)G.pitch;
    const float *z1g = G.z[l0];
    bool in0 = false, in1 = false;
    for (int h = 0; h < 2; h++) {
        const int g = lane + 32 * h;
        bool in = false;
        if (g < ng) {
            const int ki = G.gij[2 * g] - 1, kj = G.gij[2 * g + 1] - 1;
            in = ki >= lo && ki <= hi && kj >= j0 && kj <= jl;
            if (in && local > 0) {
                const size_t c = (size_t)kj * P + ki;
                const float l1 = z1g[c], l2v = z1g[c + 1], l3 = z1g[c + P], l4 = z1g[c + P + 1];
                if (G.flags & GC_F_STENCIL) {
                    float *o = G.ts + ((size_t)(local - 1) * ng + g) * 4;
                    o[0] = l1; o[1] = l2v; o[2] = l3; o[3] = l4;
                } else {
                    const float cx = G.gw[2 * g], cy = G.gw[2 * g + 1];
                    const float a = l1 * (1.0f - cx) * (1.0f - cy);
                    const float b = l2v * (cx) * (1.0f - cy);
                    const float d = l3 * (1.0f - cx) * (cy);
                    const float e = l4 * (cx) * (cy);
                    G.ts[(size_t)(local - 1) * ng + g] = a + b + d + e;
                }
            }
        }
        if (h == 0) in0 = in;
        else in1 = in;
    }
    gm0 = __ballot_sync(FULL, in0);
    gm1 = __ballot_sync(FULL, in1);
}

/* step A's gauge samples whose base row is `row`: surface rows row (lo_row)
 * and row + 1 (hi_row) */
template <class Desc>
__device__ __forceinline__ void pair_gauge_row(const Desc &G, unsigned gm0, unsigned gm1, int row,
                                               const float4 &lo_row, const float4 &hi_row, int s, int local) {
    for (int h2 = 0; h2 < 2; h2++) {
        unsigned bits = h2 == 0 ? gm0 : gm1;
        while (bits) {
            const int g = __ffs(bits) - 1 + 32 * h2;
            bits &= bits - 1;
            if (G.gij[2 * g + 1] - 1 != row) continue;
            if (G.flags & GC_F_STENCIL) {
                float l1, l2, l3, l4;
                gauge_stencil(lo_row, hi_row, G.gij[2 * g] - 1, s, l1, l2, l3, l4);
                if ((threadIdx.x & 31) == 0) {
                    float *o = G.ts + ((size_t)local * G.ng + g) * 4;
                    o[0] = l1; o[1] = l2; o[2] = l3; o[3] = l4;
                }
            } else {
                const float v = gauge_sample(lo_row, hi_row, G.gij[2 * g] - 1, s, G.gw[2 * g], G.gw[2 * g + 1]);
                if ((threadIdx.x & 31) == 0) G.ts[(size_t)local * G.ng + g] = v;
            }
        }
    }
}

/* after a wait gave up: record it, then give the copies still in flight
 * (ring positions k .. issued-1 of the tile) a bounded chance to land */
template <int S>
__device__ __forceinline__ void pair_drain(const PairRing &R, int k, int issued) {
    if ((threadIdx.x & 31) == 0) atomicExch(&g_pair_error, 1);
    for (int q = k; q < issued; q++) {
        const int n = R.seq0 + q;
        mbar_wait(R.bars + 8 * (n % S), (uint32_t)((n / S) & 1), 1 << 12);
    }
}

/* ring stages of rows r (sc), r-1 (sp) and r-2 (spp), and the phase of sc.
 * Before the tile's second and third rows exist, sp and spp name the first
 * row's stage (JM1 = max(J-1, 1) at the grid's first row; elsewhere what is
 * read there feeds only values no output uses). */
template <int S>
struct PairStages {
    int sc, sp, spp;
    uint32_t ph;
    __device__ __forceinline__ explicit PairStages(int seq0) {
        sc = seq0 % S;
        sp = spp = sc;
        ph = (uint32_t)((seq0 / S) & 1);
    }
    __device__ __forceinline__ void advance() {
        spp = sp;
        sp = sc;
        if (++sc == S) {
            sc = 0;
            ph ^= 1u;
        }
    }
};

/* the new surface of a lane's four cells on a tile that touches the grid's
 * perimeter: MASS_S everywhere, then OPEN over it on the perimeter.  On a
 * perimeter row (warp-uniform) every cell takes OPEN.  Elsewhere OPEN takes
 * the west column (lane 0's first cell, when the strip starts at column 0)
 * and the east column (cell qe of lane le): every lane evaluates OPEN on its
 * own cell at that position, so the warp does not diverge, and the lane that
 * holds the column keeps it.  mw: M west of the lane's first cell (the IM1
 * clamp already applied); ns, hs: N and H of row r-1. */
__device__ __forceinline__ float4 surface4_edge(const float4 &z1, const float4 &m, float mw, const float4 &n,
                                                const float4 &ns, const float4 &h, const float4 &hs, float r1,
                                                float r11, float r6, float r6m, int ib, int r, int nx, int ny,
                                                bool west, bool east, bool hold_e, int qe) {
    if (r == 0 || r == ny - 1) return surface4<true>(z1, m, mw, n, ns, h, hs, r1, r11, r6, r6m, ib, r, nx, ny);
    float4 o = surface4<false>(z1, m, mw, n, ns, h, hs, r1, r11, r6, r6m, ib, r, nx, ny);
    if (west) {
        const float ow = open_cell(0, r, nx, ny, h.x, hs.x, m.x, mw, n.x, ns.x);
        if ((threadIdx.x & 31) == 0) o.x = ow;
    }
    if (east) {
        const float mwq = qe == 0 ? mw : comp(m, qe - 1);
        const float oe = open_cell(nx - 1, r, nx, ny, comp(h, qe), comp(hs, qe), comp(m, qe), mwq, comp(n, qe),
                                   comp(ns, qe));
        if (hold_e) {
            o.x = qe == 0 ? oe : o.x;
            o.y = qe == 1 ? oe : o.y;
            o.z = qe == 2 ? oe : o.z;
            o.w = qe == 3 ? oe : o.w;
        }
    }
    return o;
}

/* The body for tiles touching the grid's perimeter or running past its last
 * row.  Same shape as the interior body (every quantity computed on every
 * iteration, stores guarded), with the boundary applied over it: OPEN on the
 * perimeter (surface4_edge), the IM1 clamp on the west column, the flux
 * domains (M to column nx-2, N to row ny-2 and column nx-1: the last row's N
 * stays 0), the JM1 clamp of M on row 0, and zero inputs on rows past the
 * grid (the bottom tile iterates two rows beyond it to finish step B).  Rows
 * above j0-1 and rows past the grid compute values that nothing stored reads. */
template <int S, class Desc>
__device__ __forceinline__ bool pair_rows_edge(const Desc &G, int s, int lo, int hi, int j0, int ty, int local,
                                               char *wsm, int &seq, int wait_limit, bool stall) {
    static_assert(S >= 4, "rows r-2 .. r stay staged, at least one more in flight");
    const int lane = threadIdx.x & 31;
    const int nx = G.nx, ny = G.ny;
    const size_t P = (size_t)G.pitch;
    const int l0 = local % 3, l2 = l0 == 0 ? 2 : l0 - 1; /* buffers of levels L and L + 2 */
    const bool do_arr = (G.flags & GC_F_ARRIVAL) != 0;
    const float thr = G.thr;

    /* rows: inputs rs .. rr (real rows), iterations rs .. re */
    const int jl = min(j0 + ty - 1, ny - 1); /* last output row */
    const int rs = max(j0 - 2, 0), rr = min(j0 + ty + 1, ny - 1), re = min(j0 + ty + 1, ny + 1);
    const int K = rr - rs + 1;
    PairRing R;
    R.wsm = wsm;
    R.wbase = smem_u32(wsm);
    R.bars = R.wbase + S * PStage::BYTES;
    R.seq0 = seq;
    /* copies of one row: columns [s, c1) of the strip */
    const int c1 = min(s + 128, G.pitch);
    const uint32_t cb = 4u * (uint32_t)(c1 - s);
    pair_prologue<S>(G, R, l0, rs, K, j0, jl, s, cb, stall);
    int issued = min(S, K);
    unsigned gm0, gm1;
    pair_gauge_setup(G, l0, local, lo, hi, j0, jl, gm0, gm1);

    const int ib = s + 4 * lane;
    const bool west = s == 0, east = s + 127 >= nx - 1;
    const int le = (nx - 1 - s) >> 2, qe = (nx - 1 - s) & 3; /* lane and cell of column nx-1 */
    const bool hold_e = east && lane == le;
    const bool w0 = west && lane == 0; /* IM1 = max(I-1,1) on column 0 */
    const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
    float4 z2p = zero4, m2p = zero4, m2pp = zero4, n2p = zero4, z3p = zero4;
    float m2ppw = 0.f, n2pe = 0.f;
    bool ok = true;
    int k = 0; /* real rows consumed */
    PairStages<S> st(R.seq0);
    int r = rs;
    if (j0 >= 2) {
        /* the first row (j0-2) is read only as row r-1 and r-2 of later
         * iterations: wait for it and iterate from the row after it */
        ok = __all_sync(FULL, mbar_wait(R.bars + 8 * st.sc, st.ph, wait_limit)) != 0;
        if (ok) {
            k = 1;
            st.advance();
        }
        r = ok ? rs + 1 : re + 1;
    }
    for (; r <= re; r++) {
        const bool real = r <= ny - 1;
        float4 z1 = zero4, m1 = zero4, n1 = zero4, h = zero4, ca = zero4, cc = zero4;
        if (real) {
            const bool got = mbar_wait(R.bars + 8 * st.sc, st.ph, wait_limit);
            ok = __all_sync(FULL, got) != 0;
            if (!ok) break;
            const char *pc = wsm + st.sc * PStage::BYTES;
            z1 = lds4(pc + PStage::Z + 16 * lane);
            m1 = lds4(pc + PStage::M + 16 * lane);
            n1 = lds4(pc + PStage::N + 16 * lane);
            h = lds4(pc + PStage::H + 16 * lane);
            ca = lds4(pc + PStage::C);
            cc = lds4(pc + PStage::C + 16);
            k++;
        }
        /* rows r-1 and r-2, still staged (JM1 = max(J-1,1): row "-1" is row 0) */
        const char *pp = wsm + st.sp * PStage::BYTES;
        const char *ppp = wsm + st.spp * PStage::BYTES;
        const float4 n1p = lds4(pp + PStage::N + 16 * lane), m1p = lds4(pp + PStage::M + 16 * lane);
        const float4 hp = lds4(pp + PStage::H + 16 * lane);
        const float4 cap = lds4(pp + PStage::C), ccp = lds4(pp + PStage::C + 16);
        const float4 hpp = lds4(ppp + PStage::H + 16 * lane);
        const float4 capp = lds4(ppp + PStage::C), ccpp = lds4(ppp + PStage::C + 16);
        /* record: r1 r11 r6 r3 | r5 cx cy - */
        /* every lane takes part in every shuffle (full mask); the IM1 clamp
         * selects after it */
        const float m1w_s = shw(m1.w), m1pw_s = shw(m1p.w);
        const float m1w = w0 ? m1.x : m1w_s, m1pw = w0 ? m1p.x : m1pw_s;
        const float n1e = she(n1.x), he = she(h.x), n1pe = she(n1p.x), hpe = she(hp.x);

        /* step A: surface of row r, M of row r, N of row r-1 (0 on the last
         * row and past it: J <= NY-1 fails) */
        float4 z2 = surface4_edge(z1, m1, m1w, n1, n1p, h, hp, ca.x, ca.y, ca.z, cap.z, ib, r, nx, ny, west, east,
                                  hold_e, qe);
        if (!real) z2 = zero4;
        const float4 m2 = flux_m4<true>(m1, z2, she(z2.x), n1, n1e, n1p, n1pe, h, he, cc.y, ca.w, ib, nx);
        const float4 n2 = flux_n4<true>(n1p, z2, z2p, m1p, m1pw, m1, m1w, hp, h, ccp.z, ccp.x, ib, r - 1, nx, ny);
        if ((gm0 | gm1) && r - 1 >= j0 && r - 1 <= jl) pair_gauge_row(G, gm0, gm1, r - 1, z2p, z2, s, local);

        /* step B: surface and M of row r-1, N of row r-2 */
        const int rb = r - 1;
        const float n2e = she(n2.x);
        const float m2w_s = shw(m2p.w);
        const float m2w = w0 ? m2p.x : m2w_s;
        const float4 z3 = surface4_edge(z2p, m2p, m2w, n2, n2p, hp, hpp, cap.x, cap.y, cap.z, capp.z, ib, rb, nx, ny,
                                        west, east, hold_e, qe);
        if (rb >= j0 && rb <= jl) {
            /* M of row rb: N of rows rb and JM1(rb) */
            const float4 ncb = rb == 0 ? n2 : n2p;
            const float nce = rb == 0 ? n2e : n2pe;
            const float4 m3 = flux_m4<true>(m2p, z3, she(z3.x), n2, n2e, ncb, nce, hp, hpe, ccp.y, cap.w, ib, nx);
            /* max-eta and arrival after step A, then after step B */
            const float4 xp = lds4(pp + PStage::X + 16 * lane);
            const float4 xa = max4(xp, z2p), xb = max4(xa, z3);
            const size_t ro = (size_t)rb * P;
            st4m(G.z[l2] + ro, ib, lo, hi, z3);
            st4m(G.zmax + ro, ib, lo, hi, xb);
            st4m(G.m[l2] + ro, ib, lo, hi, m3);
            if (do_arr) {
                if (may_arrive(z2p, xp, thr)) arrive4(G.arrival + ro, ib, lo, hi, z2p, xp, hp, thr, local + 1);
                if (may_arrive(z3, xa, thr)) arrive4(G.arrival + ro, ib, lo, hi, z3, xa, hp, thr, local + 2);
            }
        }
        if (rb - 1 >= j0 && rb - 1 <= jl) {
            const float4 n3 =
                flux_n4<true>(n2p, z3, z3p, m2pp, m2ppw, m2p, m2w, hpp, hp, ccpp.z, ccpp.x, ib, rb - 1, nx, ny);
            st4m(G.n[l2] + (size_t)(rb - 1) * P, ib, lo, hi, n3);
        }

        z2p = z2;
        m2pp = m2p; m2ppw = m2w; m2p = m2;
        n2p = n2; n2pe = n2e;
        z3p = z3;
        /* row r-2 is no longer needed: refill its stage S rows ahead */
        __syncwarp();
        const int kpp = r - 2 - rs;
        if (kpp >= 0 && kpp + S < K) {
            if (lane == 0) {
                const int rn = rs + kpp + S;
                pair_issue(G, l0, rn, s, cb, rn >= j0 && rn <= jl, R.wbase + st.spp * PStage::BYTES,
                           R.bars + 8 * st.spp, false);
            }
            issued = kpp + S + 1;
        }
        st.advance();
    }
    seq = R.seq0 + K;
    if (!ok) {
        pair_drain<S>(R, k, issued);
        return false;
    }
    __syncwarp();
    return true;
}

/* The body for a tile none of whose computed cells (halo rows and columns
 * included) lies on the grid's perimeter: every row is real, there is no
 * boundary logic, and each iteration computes every quantity.  On the first
 * four iterations some of them come from rows the tile does not hold exactly
 * (a step-A surface is exact from row j0-1, step-A fluxes from row j0, step
 * B from row j0 + 1 on the iteration index), and nothing stored or carried
 * into an exact value reads them: stores are the only guarded operations.
 * Such a tile stores columns s+4 .. s+123, lanes 1 .. 30 in full.  Its
 * first row, j0-2, only feeds the N flux of row j0-2 and the surface and
 * fluxes of row j0-1 through the next iterations' reads of the stage it
 * stays in, so it gets no iteration of its own. */
template <int S, class Desc>
__device__ __forceinline__ bool pair_rows_int(const Desc &G, int s, int j0, int ty, int local, char *wsm,
                                           int &seq, int wait_limit, bool stall) {
    static_assert(S >= 4, "rows r-2 .. r stay staged, at least one more in flight");
    const int lane = threadIdx.x & 31;
    const size_t P = (size_t)G.pitch;
    const int l0 = local % 3, l2 = l0 == 0 ? 2 : l0 - 1; /* buffers of levels L and L + 2 */
    const bool do_arr = (G.flags & GC_F_ARRIVAL) != 0;
    const float thr = G.thr;
    const int jl = j0 + ty - 1, rs = j0 - 2, K = ty + 4;
    PairRing R;
    R.wsm = wsm;
    R.wbase = smem_u32(wsm);
    R.bars = R.wbase + S * PStage::BYTES;
    R.seq0 = seq;
    pair_prologue<S>(G, R, l0, rs, K, j0, jl, s, 512u, stall);
    int issued = min(S, K);
    unsigned gm0, gm1;
    pair_gauge_setup(G, l0, local, s + 4, s + kPairOut + 3, j0, jl, gm0, gm1);

    const int ib = s + 4 * lane;
    const bool own = lane >= 1 && lane <= 30;
    const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
    float4 z2p = zero4, m2p = zero4, m2pp = zero4, n2p = zero4, z3p = zero4;
    float m2ppw = 0.f, n2pe = 0.f;
    bool ok = true;
    int k = 0;
    PairStages<S> st(R.seq0);
    /* the tile's first row (j0-2) is read only as row r-1 and r-2 of later
     * iterations (nothing of its own step-A results is used): wait for it,
     * and iterate from the row after it */
    ok = __all_sync(FULL, mbar_wait(R.bars + 8 * st.sc, st.ph, wait_limit)) != 0;
    if (ok) {
        k = 1;
        st.advance();
    }
    for (int r = ok ? rs + 1 : rs + K; r < rs + K; r++) {
        const bool got = mbar_wait(R.bars + 8 * st.sc, st.ph, wait_limit);
        if (!__all_sync(FULL, got)) {
            ok = false;
            break;
        }
        k++;
        const char *pc = wsm + st.sc * PStage::BYTES;
        const char *pp = wsm + st.sp * PStage::BYTES;
        const char *ppp = wsm + st.spp * PStage::BYTES;
        const float4 z1 = lds4(pc + PStage::Z + 16 * lane), m1 = lds4(pc + PStage::M + 16 * lane);
        const float4 n1 = lds4(pc + PStage::N + 16 * lane), h = lds4(pc + PStage::H + 16 * lane);
        const float4 ca = lds4(pc + PStage::C), cc = lds4(pc + PStage::C + 16);
        const float4 n1p = lds4(pp + PStage::N + 16 * lane), m1p = lds4(pp + PStage::M + 16 * lane);
        const float4 hp = lds4(pp + PStage::H + 16 * lane);
        const float4 cap = lds4(pp + PStage::C), ccp = lds4(pp + PStage::C + 16);
        const float4 hpp = lds4(ppp + PStage::H + 16 * lane);
        const float4 capp = lds4(ppp + PStage::C), ccpp = lds4(ppp + PStage::C + 16);
        /* record: r1 r11 r6 r3 | r5 cx cy - */
        const float m1w = shw(m1.w), m1pw = shw(m1p.w);
        const float n1e = she(n1.x), he = she(h.x), n1pe = she(n1p.x), hpe = she(hp.x);

        /* step A: surface of row r, M of row r, N of row r-1 */
        const float4 z2 = surface4<false>(z1, m1, m1w, n1, n1p, h, hp, ca.x, ca.y, ca.z, cap.z, ib, r, 0, 0);
        const float4 m2 = flux_m4<false>(m1, z2, she(z2.x), n1, n1e, n1p, n1pe, h, he, cc.y, ca.w, ib, 0);
        const float4 n2 = flux_n4<false>(n1p, z2, z2p, m1p, m1pw, m1, m1w, hp, h, ccp.z, ccp.x, ib, r - 1, 0, 0);
        if ((gm0 | gm1) && r - 1 >= j0 && r - 1 <= jl) pair_gauge_row(G, gm0, gm1, r - 1, z2p, z2, s, local);

        /* step B: surface and M of row r-1, N of row r-2 */
        const int rb = r - 1;
        const float n2e = she(n2.x), m2w = shw(m2p.w);
        const float4 z3 = surface4<false>(z2p, m2p, m2w, n2, n2p, hp, hpp, cap.x, cap.y, cap.z, capp.z, ib, rb, 0, 0);
        if (rb >= j0 && rb <= jl) {
            const float4 m3 = flux_m4<false>(m2p, z3, she(z3.x), n2, n2e, n2p, n2pe, hp, hpe, ccp.y, cap.w, ib, 0);
            const float4 xp = lds4(pp + PStage::X + 16 * lane);
            const float4 xa = max4(xp, z2p), xb = max4(xa, z3);
            const size_t ro = (size_t)rb * P + ib;
            if (own) {
                *reinterpret_cast<float4 *>(G.z[l2] + ro) = z3;
                *reinterpret_cast<float4 *>(G.zmax + ro) = xb;
                *reinterpret_cast<float4 *>(G.m[l2] + ro) = m3;
                if (do_arr) {
                    if (may_arrive(z2p, xp, thr))
                        arrive4(G.arrival + ro - ib, ib, ib, ib + 3, z2p, xp, hp, thr, local + 1);
                    if (may_arrive(z3, xa, thr))
                        arrive4(G.arrival + ro - ib, ib, ib, ib + 3, z3, xa, hp, thr, local + 2);
                }
            }
        }
        if (rb - 1 >= j0 && rb - 1 <= jl) {
            const float4 n3 =
                flux_n4<false>(n2p, z3, z3p, m2pp, m2ppw, m2p, m2w, hpp, hp, ccpp.z, ccpp.x, ib, rb - 1, 0, 0);
            if (own) *reinterpret_cast<float4 *>(G.n[l2] + (size_t)(rb - 1) * P + ib) = n3;
        }

        z2p = z2;
        m2pp = m2p; m2ppw = m2w; m2p = m2;
        n2p = n2; n2pe = n2e;
        z3p = z3;
        __syncwarp();
        const int kpp = r - 2 - rs;
        if (kpp >= 0 && kpp + S < K) {
            if (lane == 0) {
                const int rn = rs + kpp + S;
                pair_issue(G, l0, rn, s, 512u, rn >= j0 && rn <= jl, R.wbase + st.spp * PStage::BYTES,
                           R.bars + 8 * st.spp, false);
            }
            issued = kpp + S + 1;
        }
        st.advance();
    }
    seq = R.seq0 + K;
    if (!ok) {
        pair_drain<S>(R, k, issued);
        return false;
    }
    __syncwarp();
    return true;
}

template <int S, class Desc>
__device__ __forceinline__ bool pair_tile(const Desc &G, int lt, int step, char *wsm, int &seq,
                                          int wait_limit, bool stall) {
    const int local = step - G.step0; /* step A's 0-based index */
    /* both steps must lie in the window, and three time levels exist */
    if (local < 0 || local + 1 >= G.nsteps || G.nbuf != 3) return true;
    int tx, j0, ty;
    pair_tile_at(pair_layout(G.nx, G.ny, G.pty, G.pte), G.ny, lt, tx, j0, ty);
    int s, lo, hi;
    pair_cols(tx, G.nx, s, lo, hi);
    /* a tile none of whose computed cells (halo rows and columns included)
     * lies on the grid's perimeter or beyond it runs the body compiled
     * without boundary logic */
    const bool edge = !(s >= 1 && s + 127 <= G.nx - 2 && j0 - 2 >= 1 && j0 + ty + 1 <= G.ny - 2);
    return edge ? pair_rows_edge<S>(G, s, lo, hi, j0, ty, local, wsm, seq, wait_limit, stall)
                : pair_rows_int<S>(G, s, j0, ty, local, wsm, seq, wait_limit, stall);
}
/* A class launch's view of one member: the fields the two-step bodies read,
 * as references into the parameter bank (the class geometry and the
 * member's record), so each is read where it is used, as the single-grid
 * form reads its descriptor, instead of being copied into registers. */
struct PairClassDesc {
    const int &nx, &ny, &pitch, &pty, &pte, &nbuf;
    const float *const &rows;
    float *const (&z)[3];
    float *const (&m)[3];
    float *const (&n)[3];
    float *const &zmax;
    int *const &arrival;
    const float *const &h;
    const int *const &gij;
    const float *const &gw;
    float *const &ts;
    const int &step0, &nsteps, &flags, &ng;
    const float &thr;
    __device__ __forceinline__ PairClassDesc(const GcFusedGrid &p, const GcPairMember &q)
        : nx(p.nx), ny(p.ny), pitch(p.pitch), pty(p.pty), pte(p.pte), nbuf(p.nbuf), rows(p.rows), z(q.z), m(q.m),
          n(q.n), zmax(q.zmax), arrival(q.arrival), h(q.h), gij(q.gij), gw(q.gw), ts(q.ts), step0(q.step0),
          nsteps(q.nsteps), flags(q.flags), ng(q.ng), thr(q.thr) {}
};

/* where a launch's tiles come from: one grid by value, a work list of
 * {grid, tile} over descriptors in memory, or a class launch's member table
 * in the parameter bank */
enum class PairSrc { One, List, Class };

template <int W, int S, PairSrc SRC>
__device__ __forceinline__ void pair_kernel_src(const GcFusedGrid &one, const GcFusedGrid *__restrict__ grids,
                                                const int2 *__restrict__ tiles, int ntiles, const GcPairClass *cls,
                                                const int *__restrict__ step_base, int step_off, int wait_limit,
                                                int stall) {
    extern __shared__ __align__(128) char smem[];
    /* programmatic dependent launch: the previous kernel in the stream has
     * finished and its writes are visible past this point */
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    const int step = step_off + (step_base ? *step_base : 0);
    /* with one warp per CTA the tile index, and with it every address of the
     * ring and the copies, is uniform across the warp */
    const int warp = W == 1 ? 0 : (int)(threadIdx.x >> 5), lane = threadIdx.x & 31;
    char *wsm = smem + warp * pair_warp_bytes<S>();
    const uint32_t bars = smem_u32(wsm) + S * PStage::BYTES;
    if (lane == 0) {
        for (int q = 0; q < S; q++) mbar_init(bars + 8 * q, 1);
        fence_mbar_init();
    }
    __syncwarp();
    int seq = 0;
    bool first = stall != 0 && blockIdx.x == 0 && warp == 0;
    for (int tile = blockIdx.x * W + warp; tile < ntiles; tile += gridDim.x * W) {
        bool ok;
        if constexpr (SRC == PairSrc::List) {
            const int2 w = tiles[tile];
            ok = pair_tile<S>(grids[w.x], w.y, step, wsm, seq, wait_limit, first);
        } else if constexpr (SRC == PairSrc::Class) {
            const int mi = tile % cls->nm, lt = tile / cls->nm;
            const PairClassDesc G(cls->proto, cls->m[mi]);
            ok = pair_tile<S>(G, lt, step, wsm, seq, wait_limit, first);
        } else {
            ok = pair_tile<S>(one, tile, step, wsm, seq, wait_limit, first);
        }
        first = false;
        if (!ok) return;
    }
}

template <int W, int S, bool MULTI>
__device__ __forceinline__ void pair_kernel(const GcFusedGrid &one, const GcFusedGrid *__restrict__ grids,
                                            const int2 *__restrict__ tiles, int ntiles,
                                            const int *__restrict__ step_base, int step_off, int wait_limit,
                                            int stall) {
    pair_kernel_src<W, S, MULTI ? PairSrc::List : PairSrc::One>(one, grids, tiles, ntiles, nullptr, step_base,
                                                                step_off, wait_limit, stall);
}

/* the single-grid form, held to 128 registers so that 16 warps fit an SM
 * (it needs no spill for that) */
template <int W, int S>
__global__ void __launch_bounds__(32 * W, 16 / W) k_pair_one(GcFusedGrid one, const GcFusedGrid *__restrict__ grids,
                                                              const int2 *__restrict__ tiles, int ntiles,
                                                              const int *__restrict__ step_base, int step_off,
                                                              int wait_limit, int stall) {
    pair_kernel<W, S, false>(one, grids, tiles, ntiles, step_base, step_off, wait_limit, stall);
}

/* the work-list form: each tile's descriptor is loaded from the list */
template <int W, int S>
__global__ void __launch_bounds__(32 * W) k_pair_list(GcFusedGrid one, const GcFusedGrid *__restrict__ grids,
                                                       const int2 *__restrict__ tiles, int ntiles,
                                                       const int *__restrict__ step_base, int step_off,
                                                       int wait_limit, int stall) {
    pair_kernel<W, S, true>(one, grids, tiles, ntiles, step_base, step_off, wait_limit, stall);
}

/* the work-list form with its registers capped so that 16 warps fit an SM
 * (the autotuner weighs that occupancy against the spills it costs) */
template <int W, int S>
__global__ void __launch_bounds__(32 * W, 16 / W) k_pair_capped(GcFusedGrid one, const GcFusedGrid *__restrict__ grids,
                                                                const int2 *__restrict__ tiles, int ntiles,
                                                                const int *__restrict__ step_base, int step_off,
                                                                int wait_limit, int stall) {
    pair_kernel<W, S, true>(one, grids, tiles, ntiles, step_base, step_off, wait_limit, stall);
}

/* the class form: member table in the parameter bank, held to the single-grid
 * form's register budget */
template <int W, int S>
__global__ void __launch_bounds__(32 * W, 16 / W) k_pair_class(const __grid_constant__ GcPairClass c,
                                                                const int *__restrict__ step_base, int step_off,
                                                                int wait_limit, int stall) {
    GcFusedGrid none;
    pair_kernel_src<W, S, PairSrc::Class>(none, nullptr, nullptr, c.nm * c.ntiles, &c, step_base, step_off,
                                          wait_limit, stall);
}

struct PairVariant {
    int w, s;
    void (*one)(GcFusedGrid, const GcFusedGrid *, const int2 *, int, const int *, int, int, int);
    void (*multi)(GcFusedGrid, const GcFusedGrid *, const int2 *, int, const int *, int, int, int);
    void (*cls)(const GcPairClass, const int *, int, int, int);
};

#define GC_PVARIANT(W, S) {W, S, k_pair_one<W, S>, k_pair_list<W, S>, k_pair_class<W, S>}
#define GC_PVARIANT_CAPPED(W, S) {W, S, k_pair_one<W, S>, k_pair_capped<W, S>, k_pair_class<W, S>}
const PairVariant kPairVariants[] = {
    GC_PVARIANT(4, 5), GC_PVARIANT(4, 4), GC_PVARIANT(2, 5), GC_PVARIANT(4, 6),
    GC_PVARIANT_CAPPED(4, 5), GC_PVARIANT_CAPPED(4, 4), GC_PVARIANT(1, 4), GC_PVARIANT(1, 5),
};
#undef GC_PVARIANT
#undef GC_PVARIANT_CAPPED
constexpr int kNumPairVariants = sizeof(kPairVariants) / sizeof(kPairVariants[0]);

int pair_smem(const PairVariant &v) {
    switch (v.s) {
    case 4: return v.w * pair_warp_bytes<4>();
    case 5: return v.w * pair_warp_bytes<5>();
    default: return v.w * pair_warp_bytes<6>();
    }
}

int g_wait_limit = 1 << 22; /* polls before a pipeline wait gives up */
int g_stall_next = 0;       /* the next launch injects one stalled row */

void prepare_pair(const PairVariant &v) {
    static bool done[64][16];
    static_assert(kNumPairVariants <= 16, "one flag per variant");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) dev = 0;
    const int idx = (int)(&v - kPairVariants);
    if (done[dev][idx]) return;
    cudaFuncSetAttribute(v.one, cudaFuncAttributeMaxDynamicSharedMemorySize, pair_smem(v));
    cudaFuncSetAttribute(v.multi, cudaFuncAttributeMaxDynamicSharedMemorySize, pair_smem(v));
    cudaFuncSetAttribute(v.cls, cudaFuncAttributeMaxDynamicSharedMemorySize, pair_smem(v));
    done[dev][idx] = true;
}

cudaError_t launch_pair(void (*kern)(GcFusedGrid, const GcFusedGrid *, const int2 *, int, const int *, int, int, int),
                        int ctas, int threads, int smem, cudaStream_t s, const GcFusedGrid &g,
                        const GcFusedGrid *grids, const int2 *tiles, int ntiles, const int *step_base,
                        int step_off) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)ctas);
    cfg.blockDim = dim3((unsigned)threads);
    cfg.dynamicSmemBytes = (size_t)smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = gc_pdl_on() ? 1 : 0;
    const int stall = g_stall_next;
    g_stall_next = 0;
    return cudaLaunchKernelEx(&cfg, kern, g, grids, tiles, ntiles, step_base, step_off, g_wait_limit, stall);
}

} // namespace

int gc_pair_num_variants() { return kNumPairVariants; }

GcTileCfg gc_pair_variant(int v) {
    if (v < 0 || v >= kNumPairVariants) v = 0;
    return GcTileCfg{kPairVariants[v].w, kPairVariants[v].s};
}

int gc_pair_tiles(int nx, int ny, int ty, int te, int *tiles_x) {
    const PairLayout L = pair_layout(nx, ny, ty, te);
    if (tiles_x) *tiles_x = L.tiles_x;
    return L.count;
}

/* rule 2's short tiles: about 60% of ty (a perimeter tile's row costs about
 * 1.5 interior rows) */
int gc_pair_short_ty(int rule, int ty) { return (rule == 2 && ty > 6) ? (3 * ty + 2) / 5 : 0; }

extern "C" int gc_pair_layout_tile(int nx, int ny, int ty, int rule, int lt, int *out5) {
    if (nx < 1 || ny < 1 || ty < 1) return -1;
    const PairLayout L = pair_layout(nx, ny, ty, gc_pair_short_ty(rule, ty));
    if (out5 && lt >= 0 && lt < L.count) {
        int tx, j0, h, s, lo, hi;
        pair_tile_at(L, ny, lt, tx, j0, h);
        pair_cols(tx, nx, s, lo, hi);
        out5[0] = s;
        out5[1] = lo;
        out5[2] = hi;
        out5[3] = j0;
        out5[4] = h;
    }
    return L.count;
}

int gc_pair_max_ctas(int variant, bool multi) {
    if (variant < 0 || variant >= kNumPairVariants) variant = 0;
    const PairVariant &v = kPairVariants[variant];
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    prepare_pair(v);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, multi ? v.multi : v.one, 32 * v.w, pair_smem(v));
    return sms * (per > 0 ? per : 1);
}

int gc_pair_pick_ty(int variant, int ngrids, const int *nx, const int *ny, int rule, bool multi) {
    const int slots = gc_pair_max_ctas(variant, multi) * gc_pair_variant(variant).warps;
    auto tiles = [&](int ty) {
        long long t = 0;
        for (int g = 0; g < ngrids; g++) t += gc_pair_tiles(nx[g], ny[g], ty, gc_pair_short_ty(rule, ty), nullptr);
        return t;
    };
    /* a warp's time is about (rows + 4 halo rows) per tile; a launch lasts
     * waves x that.  Rules 0 and 2: the height minimising it; rule 1: the
     * same among heights of at least 24 rows (less halo per row when many
     * waves) */
    const int tmin = rule == 1 ? 24 : 8;
    int best = 32;
    long long best_cost = -1, best_waves = 0;
    for (int ty = tmin; ty <= 256; ty++) {
        const long long waves = (tiles(ty) + slots - 1) / slots;
        const long long cost = waves * (ty + 4);
        if (best_cost < 0 || cost < best_cost || (cost == best_cost && waves < best_waves)) {
            best = ty;
            best_cost = cost;
            best_waves = waves;
        }
    }
    return best;
}

cudaError_t gc_pair_launch_one_at(int variant, const GcFusedGrid &g, const int *d_step_base, int step_off,
                                  cudaStream_t s) {
    if (variant < 0 || variant >= kNumPairVariants) variant = 0;
    const PairVariant &v = kPairVariants[variant];
    const int ntiles = gc_pair_tiles(g.nx, g.ny, g.pty, g.pte, nullptr);
    prepare_pair(v);
    return launch_pair(v.one, (ntiles + v.w - 1) / v.w, 32 * v.w, pair_smem(v), s, g, nullptr, nullptr, ntiles,
                       d_step_base, step_off);
}

cudaError_t gc_pair_launch_multi(int variant, const GcFusedGrid *d_grids, const int2 *d_tiles, int ntiles,
                                 const int *d_step_base, int step_off, cudaStream_t s) {
    if (variant < 0 || variant >= kNumPairVariants) variant = 0;
    const PairVariant &v = kPairVariants[variant];
    if (ntiles <= 0) return cudaSuccess;
    GcFusedGrid dummy;
    memset(&dummy, 0, sizeof dummy);
    prepare_pair(v);
    return launch_pair(v.multi, (ntiles + v.w - 1) / v.w, 32 * v.w, pair_smem(v), s, dummy, d_grids, d_tiles,
                       ntiles, d_step_base, step_off);
}

cudaError_t gc_pair_launch_class(int variant, const GcPairClass &c, const int *d_step_base, int step_off,
                                 cudaStream_t s) {
    if (variant < 0 || variant >= kNumPairVariants) variant = 0;
    const PairVariant &v = kPairVariants[variant];
    if (c.nm <= 0 || c.nm > GC_PAIR_CLASS_MAX || c.ntiles <= 0) return cudaErrorInvalidValue;
    prepare_pair(v);
    const int ntiles = c.nm * c.ntiles;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)((ntiles + v.w - 1) / v.w));
    cfg.blockDim = dim3((unsigned)(32 * v.w));
    cfg.dynamicSmemBytes = (size_t)pair_smem(v);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = gc_pdl_on() ? 1 : 0;
    const int stall = g_stall_next;
    g_stall_next = 0;
    return cudaLaunchKernelEx(&cfg, v.cls, c, d_step_base, step_off, g_wait_limit, stall);
}

int gc_pair_take_error() {
    int v = 0, z = 0;
    cudaMemcpyFromSymbol(&v, g_pair_error, sizeof v);
    if (v) cudaMemcpyToSymbol(g_pair_error, &z, sizeof z);
    return v;
}

void gc_pair_set_wait_limit(int polls) { g_wait_limit = polls > 0 ? polls : (1 << 22); }
void gc_pair_stall_next() { g_stall_next = 1; }
