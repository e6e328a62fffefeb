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
 * Work decomposition: a warp owns a 128 x TY tile (I x J); lane l owns the
 * four consecutive cells I = i0+4l .. i0+4l+3 and moves them as float4.  The
 * warp marches down the tile's rows.  Each row's M (with a west halo), N, H
 * and per-row coefficient record arrive by 1-D bulk copies
 * (cp.async.bulk, completing on an mbarrier) into an S-stage shared-memory
 * ring private to the warp; Z1 and max-eta are either staged the same way or
 * loaded straight into registers one row ahead (variant flag FL_ZD).  At row
 * r the warp computes the new surface Z2 of row r (plus the east halo
 * column, kept in a two-row shared ring), then the momentum of row r-1,
 * which needs Z2 of rows r-1 and r; the copies for row r+S-2 are issued as
 * soon as row r-2's stage is free (flag FL_NC: the momentum's N of row r-2
 * rides in registers, so row r-1's stage is refilled, with row r+S-1, right
 * after row r; three stages then keep a row in flight, and the smaller ring
 * lets 20 warps share an SM).  There is no block barrier: warps of a
 * CTA work on independent tiles.  The halo row/column of Z2 is recomputed by
 * both neighbouring tiles from the same inputs, bit-identically.
 *
 * Per cell the kernel streams Z1, M1, N1, H in and Z2, M2, N2 out (28 bytes)
 * plus the 8-byte max-amplitude read/write; R2 and R4 are rebuilt from H and
 * the per-row factors instead of being streamed.  Every pipeline wait is
 * bounded: a wait that gives up sets g_pipe_error and the warp leaves after
 * its copies in flight have landed (or a second bounded wait expired).
 *
 * Arithmetic is evaluated in the Fortran order with separately rounded
 * float operations (the library is built with -fmad=false).
 */
#include <atomic>
#include <mutex>
#include <type_traits>

#include "fused.h"
#include "open_bd.cuh"

namespace {

constexpr int TXW = 128; /* columns per warp tile: 32 lanes x 4 cells */


/* OPEN on a perimeter cell of the outermost layer (open_bd.cuh) */
using gcopen::open_cell;

/* new surface of one cell: OPEN on the outer layer's perimeter, carried
 * level-1 value on a child's I=1 / J=1 edges, MASS_S elsewhere */
__device__ __forceinline__ float z2_cell(bool root, int i, int r, int nx, int ny, float z1, float h,
                                         float hs, float m, float mw, float n, float ns, float r1,
                                         float r11, float r6, float r6m) {
    if (root && (i == 0 || i == nx - 1 || r == 0 || r == ny - 1))
        return open_cell(i, r, nx, ny, h, hs, m, mw, n, ns);
    if (!root && (i == 0 || r == 0)) return z1;
    if (h > CC_GX) {
        float zz = z1 - r1 * (m - mw) - r11 * (n * r6 - ns * r6m);
        if (fabsf(zz) < CC_EPS) zz = 0.0f;
        if ((zz + h) <= CC_EPS) zz = -h;
        return zz;
    }
    return 0.0f;
}

/* ------------------------------------------------------------------ */
/* bulk-copy pipeline primitives (PTX, sm_90+ / sm_100a)              */
/* ------------------------------------------------------------------ */
__device__ int g_pipe_error; /* set when a pipeline wait gave up */

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint32_t bar, int count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
/* 1-D bulk copy global -> this CTA's shared memory, completing on `bar`;
 * dst, src and bytes must be multiples of 16 */
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
/* bounded wait: gives up after `limit` polls (each poll may suspend briefly) */
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int limit) {
    for (int it = 0; it < limit; it++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

constexpr int WAIT_LIMIT = 1 << 22;


/* Variant flags.  FL_ONE: lane 0 issues all of a row's copies after one
 * proxy fence (else lanes 0..5 issue one field each).  FL_ZD: Z1 and max-eta
 * are not staged; each lane loads its own float4 of them from global memory
 * one row ahead into registers (the stage then holds M, N, H and the row
 * record only, 40 % less shared memory, so more warps fit on an SM). */
constexpr int FL_ONE = 1, FL_ZD = 2;
/* FL_NC: the momentum's N of row j-1 is carried from the previous row in
 * five registers per lane instead of read from that row's stage, so a stage
 * is free (and refilled) one row earlier: a 3-stage ring keeps one row in
 * flight, and its smaller footprint lets more warps share an SM. */
constexpr int FL_NC = 4;

/* one pipeline stage holds one grid row of a warp tile (byte offsets) */
template <int FL>
struct Stage {
    static constexpr int M = 0;                 /* M: 136 floats, cols i0-4 .. i0+131 (index c+4) */
    static constexpr int N = M + 136 * 4;       /* N: 132 floats, cols i0 .. i0+131 */
    static constexpr int H = N + 132 * 4;
    static constexpr int Z = H + 132 * 4;       /* Z1 (staged variants) */
    static constexpr int X = Z + ((FL & FL_ZD) ? 0 : 132 * 4);   /* max-eta, 128 floats */
    static constexpr int C = X + ((FL & FL_ZD) ? 0 : 128 * 4);   /* row coefficient record, 8 floats */
    static constexpr int BYTES = ((C + 32) + 127) / 128 * 128;
};
constexpr int ZR_FLOATS = 136;         /* new-surface ring row: cols i0 .. i0+128 */

template <int FL>
__host__ __device__ constexpr int warp_smem_bytes(int S) {
    return ((S * Stage<FL>::BYTES + 2 * ZR_FLOATS * 4 + S * 8) + 127) / 128 * 128;
}

enum { F_M = 1, F_N = 2, F_H = 4, F_Z = 8, F_X = 16, F_C = 32 };


__device__ __forceinline__ float4 lds4(const float *p) { return *reinterpret_cast<const float4 *>(p); }

/* masked float4 store at p = &row[i] (cells at or beyond nx become 0) */
__device__ __forceinline__ void st4p(float *p, int i, int nx, const float v[4]) {
    if (i < nx) {
        float4 t;
        t.x = v[0];
        t.y = (i + 1 < nx) ? v[1] : 0.0f;
        t.z = (i + 2 < nx) ? v[2] : 0.0f;
        t.w = (i + 3 < nx) ? v[3] : 0.0f;
        *reinterpret_cast<float4 *>(p) = t;
    }
}

template <int S, bool XR24, int FL>
__device__ __forceinline__ bool warp_tile(const GcFusedGrid &Gref, int lt, int step, char *wsm, int &seq) {
    using ST = Stage<FL>;
    constexpr bool ZD = (FL & FL_ZD) != 0;
    constexpr bool ONE = (FL & FL_ONE) != 0;
    constexpr bool NC = (FL & FL_NC) != 0;
    constexpr int SB_ = ST::BYTES;
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    /* descriptor fields in registers (stores could alias a descriptor in global memory) */
    const int nx = Gref.nx, ny = Gref.ny, pitch = Gref.pitch;
    const size_t P = (size_t)pitch;
    const int tiles_x = Gref.tiles_x, step0 = Gref.step0, nsteps = Gref.nsteps, TY = Gref.ty;
    const int flags = Gref.flags;
    const float thr = Gref.thr;
    const bool root = Gref.root != 0;
    const int local = step - step0; /* 0-based index of the step being computed */
    if (local < 0 || local > nsteps) return true;
    /* buffers of levels local and local + 1: ping-pong, or level L in L % 3 */
    int cur, nxt;
    if (Gref.nbuf == 3) {
        cur = local % 3;
        nxt = cur == 2 ? 0 : cur + 1;
    } else {
        cur = Gref.cur0 ^ (local & 1);
        nxt = cur ^ 1;
    }
    const float *__restrict__ z1 = Gref.z[cur];
    const float *__restrict__ m1 = Gref.m[cur];
    const float *__restrict__ n1 = Gref.n[cur];
    float *__restrict__ z2 = Gref.z[nxt];
    float *__restrict__ m2 = Gref.m[nxt];
    float *__restrict__ n2 = Gref.n[nxt];
    float *__restrict__ zmax = Gref.zmax;
    int *__restrict__ arrival = Gref.arrival;
    const bool do_max = (flags & GC_F_MAXAMP) != 0;
    const bool do_arr = (flags & GC_F_ARRIVAL) != 0;
    const bool by_max = do_max && (flags & GC_F_ARR_BYMAX) != 0;
    const int txi = lt % tiles_x, tyi = lt / tiles_x;
    const int i0 = txi * TXW, j0 = tyi * TY;

    /* gauges: the tile holding a gauge's base cell (KI,KJ) samples the surface
     * the previous step left (its Z2 is our Z1); the 2x2 stencil reaches at
     * most into the east / south neighbour tiles, finished with that step */
    if (Gref.ng > 0) {
        const int ng = Gref.ng;
        int prev = local - 1;
        if (prev >= 0 && prev < Gref.ts_len) {
            const int *gij = Gref.gij;
            const float *gw = Gref.gw;
            float *ts = Gref.ts;
            for (int g = lane; g < ng; g += 32) {
                int ki = gij[2 * g] - 1, kj = gij[2 * g + 1] - 1;
                if (ki < i0 || ki >= i0 + TXW || kj < j0 || kj >= j0 + TY) continue;
                size_t c = (size_t)kj * P + ki;
                float l1 = z1[c], l2 = z1[c + 1], l3 = z1[c + P], l4 = z1[c + P + 1];
                float cx = gw[2 * g], cy = gw[2 * g + 1];
                float a = l1 * (1.0f - cx) * (1.0f - cy);
                float b = l2 * (cx) * (1.0f - cy);
                float d = l3 * (1.0f - cx) * (cy);
                float e = l4 * (cx) * (cy);
                ts[(size_t)prev * ng + g] = a + b + d + e;
            }
        }
    }
    if (local >= nsteps) return true; /* finished: only the last gauge sample */

    /* rows of this tile: k = 0 is row max(j0-1,0) (N, H, coefficients only),
     * k = 1..TY+1 are rows j0 .. j0+TY (the last one a halo row) */
    const int K = 1 + min(TY + 1, ny - j0);
    const int jr0 = j0 > 0 ? j0 - 1 : 0;
    const uint32_t wbase = smem_u32(wsm);
    const uint32_t bars = wbase + S * SB_ + 2 * ZR_FLOATS * 4;
    float *zr = reinterpret_cast<float *>(wsm + S * SB_);
    const int seq0 = seq;

    /* copies of one row: M (with a 4-column west halo), N, H[, Z1, max-eta]
     * and the row record; source columns and byte counts are fixed per tile */
    const int ms = i0 >= 4 ? i0 - 4 : 0;
    const uint32_t bm = 4u * (i0 >= 4 ? min(136, pitch - ms) : min(132, pitch));
    const uint32_t bn = 4u * min(132, pitch - i0), bx = 4u * min(128, pitch - i0);
    const uint32_t m_dst = ST::M + (i0 >= 4 ? 0 : 16);
    const int mk_pro = F_N | F_H | F_C;
    const int mk_halo = F_M | F_N | F_H | F_C | (ZD ? 0 : F_Z);
    const int mk_mid = mk_halo | ((!ZD && do_max) ? F_X : 0);
    const uint32_t by_pro = 2 * bn + 32u, by_halo = bm + (ZD ? 2 : 3) * bn + 32u;
    const uint32_t by_mid = by_halo + ((!ZD && do_max) ? bx : 0u);
    /* per-lane issuer (lanes 0..5 own one field each) */
    const char *cp_src = nullptr;
    size_t cp_stride = P * 4;
    uint32_t cp_dst = 0, cp_bytes = 0;
    int cp_bit = 0;
    if (!ONE) {
        if (lane == 0) { cp_src = (const char *)(m1 + ms); cp_dst = m_dst; cp_bytes = bm; cp_bit = F_M; }
        if (lane == 1) { cp_src = (const char *)(n1 + i0); cp_dst = ST::N; cp_bytes = bn; cp_bit = F_N; }
        if (lane == 2) { cp_src = (const char *)(Gref.h + i0); cp_dst = ST::H; cp_bytes = bn; cp_bit = F_H; }
        if (!ZD && lane == 3) { cp_src = (const char *)(z1 + i0); cp_dst = ST::Z; cp_bytes = bn; cp_bit = F_Z; }
        if (!ZD && lane == 4) { cp_src = (const char *)(zmax + i0); cp_dst = ST::X; cp_bytes = bx; cp_bit = F_X; }
        if (lane == 5) { cp_src = (const char *)Gref.rows; cp_dst = ST::C; cp_bytes = 32u; cp_bit = F_C; cp_stride = GC_ROWW * 4; }
    }
    auto issue = [&](int k, int st) {
        const int mask = k == 0 ? mk_pro : (k <= TY ? mk_mid : mk_halo);
        const uint32_t bytes = k == 0 ? by_pro : (k <= TY ? by_mid : by_halo);
        const int jr = k == 0 ? jr0 : j0 + k - 1;
        const uint32_t bar = bars + 8 * st;
        const uint32_t sb = wbase + st * SB_;
        if constexpr (ONE) {
            if (lane == 0) {
                fence_proxy_async(); /* the warp's earlier reads of this stage come first */
                mbar_expect_tx(bar, bytes);
                const size_t ro = (size_t)jr * P;
                if (mask & F_M) bulk_g2s(sb + m_dst, m1 + ms + ro, bm, bar);
                bulk_g2s(sb + ST::N, n1 + i0 + ro, bn, bar);
                bulk_g2s(sb + ST::H, Gref.h + i0 + ro, bn, bar);
                if (!ZD && (mask & F_Z)) bulk_g2s(sb + ST::Z, z1 + i0 + ro, bn, bar);
                if (!ZD && (mask & F_X)) bulk_g2s(sb + ST::X, zmax + i0 + ro, bx, bar);
                bulk_g2s(sb + ST::C, Gref.rows + (size_t)jr * GC_ROWW, 32u, bar);
            }
        } else {
            if (lane == 0) {
                fence_proxy_async();
                mbar_expect_tx(bar, bytes);
            }
            __syncwarp();
            if (cp_bit & mask) {
                fence_proxy_async(); /* this stage's earlier generic reads come first */
                bulk_g2s(sb + cp_dst, cp_src + (size_t)jr * cp_stride, cp_bytes, bar);
            }
        }
    };
    __syncwarp();
    {
        int st = seq0 % S;
        const int kk = min(S, K);
        for (int k = 0; k < kk; k++) {
            issue(k, st);
            st = (st + 1 == S) ? 0 : st + 1;
        }
    }
    auto wait = [&](int st, uint32_t par) {
        const bool got = mbar_wait(bars + 8 * st, par, WAIT_LIMIT);
        return __all_sync(FULL, got) != 0; /* warp-uniform outcome */
    };
    /* stages and phase parities tracked incrementally: row k+1 follows row k */
    int stB = seq0 % S, stC = 0;
    uint32_t parB = (uint32_t)((seq0 / S) & 1);
    const int c0 = 4 * lane;             /* this lane's first cell within the tile */
    const int ib = i0 + c0;
    const bool own = ib < nx;
    const int ih = i0 + TXW;
    const bool hasR = (lane == 31) && (ih < nx);
    /* unstaged Z1 / max-eta: this lane's float4 of row r, loaded one row ahead */
    float4 zq = make_float4(0.f, 0.f, 0.f, 0.f), xq = zq;
    float zqh = 0.0f;
    auto load_direct = [&](int k, float4 &zo, float4 &xo, float &zh) {
        if constexpr (ZD) {
            const int rr = j0 + k - 1;
            if (k < K) {
                const size_t ro = (size_t)rr * P;
                if (own) zo = __ldg(reinterpret_cast<const float4 *>(z1 + ro + ib));
                if (hasR) zh = __ldg(z1 + ro + ih);
                if (own && do_max && k <= TY) xo = *reinterpret_cast<const float4 *>(zmax + ro + ib);
            }
        }
    };
    load_direct(1, zq, xq, zqh);
    bool ok = wait(stB, parB);
    /* output row pointers at this lane's first cell: surface/max rows r, flux rows j = r-1 */
    float *z2p = z2 + (size_t)j0 * P + ib;
    float *zxp = zmax + (size_t)j0 * P + ib;
    float *m2p = m2 + (size_t)j0 * P + ib;
    float *n2p = n2 + (size_t)j0 * P + ib;

    /* a tile none of whose cells (halo row and column included) lies on a
     * grid edge or in the max/arrival exclusion window runs a body compiled
     * without any boundary logic */
    const int wi0 = Gref.wi0, wi1 = Gref.wi1, wj0 = Gref.wj0, wj1 = Gref.wj1;
    const bool inwin = Gref.has_win && i0 <= wi1 && i0 + TXW - 1 >= wi0 && j0 <= wj1 && j0 + TY - 1 >= wj0;
    const bool edge = inwin || !(i0 >= 1 && i0 + TXW <= nx - 2 && j0 >= 1 && j0 + TY <= ny - 2);
    /* FL_NC: N of rows r-1 (this row's stage B) and r-2 (carried) at columns c0..c0+4 */
    float nbk[5] = {0.f, 0.f, 0.f, 0.f, 0.f}, nck[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
    for (int k = 1; k <= TY + 1 && ok; k++) {
        const int r = j0 + k - 1;
        const bool rv = k < K;
        const int stA = (stB + 1 == S) ? 0 : stB + 1;
        const uint32_t parA = (stA == 0) ? (parB ^ 1u) : parB;
        float *SA = reinterpret_cast<float *>(wsm + stA * SB_);
        float *SB = reinterpret_cast<float *>(wsm + stB * SB_);
        float *SC = reinterpret_cast<float *>(wsm + stC * SB_);
        /* this row's unstaged values, and the next row's loads in flight */
        const float4 zcur = zq, xcur = xq;
        const float zhcur = zqh;
        load_direct(k + 1, zq, xq, zqh);
        if (rv) {
            ok = wait(stA, parA);
            if (!ok) break;
            if (i0 == 0 && lane == 0) SA[ST::M / 4 + 3] = SA[ST::M / 4 + 4]; /* IM1 = max(I-1,1) */
        }
        __syncwarp();
        if constexpr (NC) {
            const float *nBr = SB + ST::N / 4;
            const float4 t = lds4(nBr + c0);
            nbk[0] = t.x; nbk[1] = t.y; nbk[2] = t.z; nbk[3] = t.w; nbk[4] = nBr[c0 + 4];
        }
        float *zA = zr + (k & 1) * ZR_FLOATS, *zB = zr + ((k - 1) & 1) * ZR_FLOATS;
        auto body = [&](auto edge_tag) {
            constexpr bool EDGE = decltype(edge_tag)::value;
            if (rv) {
                const float *mA = SA + ST::M / 4 + 4, *nA = SA + ST::N / 4, *hA = SA + ST::H / 4;
                const float *nB = SB + ST::N / 4, *hB = SB + ST::H / 4;
                const float r1 = SA[ST::C / 4 + GC_R1], r11 = SA[ST::C / 4 + GC_R11], r6 = SA[ST::C / 4 + GC_R6];
                const float r6m = (r > 0) ? SB[ST::C / 4 + GC_R6] : 0.0f;
                const float4 m4 = lds4(mA + c0), n4 = lds4(nA + c0), nb4 = lds4(nB + c0);
                const float4 h4 = lds4(hA + c0), hb4 = lds4(hB + c0);
                float4 z4;
                float z1h;
                if constexpr (ZD) {
                    z4 = zcur;
                    z1h = zhcur;
                } else {
                    const float *z1A = SA + ST::Z / 4;
                    z4 = lds4(z1A + c0);
                    z1h = z1A[TXW];
                }
                const float mv[4] = {m4.x, m4.y, m4.z, m4.w}, nv[4] = {n4.x, n4.y, n4.z, n4.w};
                const float nbv[4] = {nb4.x, nb4.y, nb4.z, nb4.w}, hv[4] = {h4.x, h4.y, h4.z, h4.w};
                const float hbv[4] = {hb4.x, hb4.y, hb4.z, hb4.w}, zv[4] = {z4.x, z4.y, z4.z, z4.w};
                const float mwest = mA[c0 - 1];
                float zn[4];
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const float mw = q == 0 ? mwest : mv[q - 1];
                    if constexpr (EDGE) {
                        zn[q] = z2_cell(root, ib + q, r, nx, ny, zv[q], hv[q], hbv[q], mv[q], mw, nv[q], nbv[q], r1,
                                        r11, r6, r6m);
                    } else {
                        /* MASS_S (mass.f90:82-95) */
                        const float h = hv[q];
                        float zz = zv[q] - r1 * (mv[q] - mw) - r11 * (nv[q] * r6 - nbv[q] * r6m);
                        zz = (fabsf(zz) < CC_EPS) ? 0.0f : zz;
                        zz = ((zz + h) <= CC_EPS) ? -h : zz;
                        zn[q] = (h > CC_GX) ? zz : 0.0f;
                    }
                }
                *reinterpret_cast<float4 *>(zA + c0) = make_float4(zn[0], zn[1], zn[2], zn[3]);
                if (lane == 31 && (!EDGE || hasR)) {
                    if constexpr (EDGE) {
                        zA[TXW] = z2_cell(root, ih, r, nx, ny, z1h, hA[TXW], hB[TXW], mA[TXW], mA[TXW - 1],
                                          nA[TXW], nB[TXW], r1, r11, r6, r6m);
                    } else {
                        const float h = hA[TXW];
                        float zz = z1h - r1 * (mA[TXW] - mA[TXW - 1]) - r11 * (nA[TXW] * r6 - nB[TXW] * r6m);
                        zz = (fabsf(zz) < CC_EPS) ? 0.0f : zz;
                        zz = ((zz + h) <= CC_EPS) ? -h : zz;
                        zA[TXW] = (h > CC_GX) ? zz : 0.0f;
                    }
                }
                if (k <= TY && own) {
                    if constexpr (EDGE) st4p(z2p, ib, nx, zn);
                    else *reinterpret_cast<float4 *>(z2p) = make_float4(zn[0], zn[1], zn[2], zn[3]);
                    /* cells whose surface a child's feedback rewrites later */
                    bool skip[4] = {false, false, false, false};
                    if constexpr (EDGE) {
#pragma unroll
                        for (int q = 0; q < 4; q++)
                            skip[q] = inwin && r >= wj0 && r <= wj1 && ib + q >= wi0 && ib + q <= wi1;
                    }
                    float xo[4] = {0.0f, 0.0f, 0.0f, 0.0f}; /* max-eta before this step */
                    if (do_max) {
                        float4 x4;
                        if constexpr (ZD) x4 = xcur;
                        else x4 = lds4(SA + ST::X / 4 + c0);
                        xo[0] = x4.x; xo[1] = x4.y; xo[2] = x4.z; xo[3] = x4.w;
                        float zx[4];
#pragma unroll
                        for (int q = 0; q < 4; q++) zx[q] = (xo[q] >= zn[q] || skip[q]) ? xo[q] : zn[q];
                        if constexpr (EDGE) st4p(zxp, ib, nx, zx);
                        else *reinterpret_cast<float4 *>(zxp) = make_float4(zx[0], zx[1], zx[2], zx[3]);
                    }
                    if (do_arr) {
                        const float zhi = fmaxf(fmaxf(zn[0], zn[1]), fmaxf(zn[2], zn[3]));
                        if (zhi > thr) {
#pragma unroll
                            for (int q = 0; q < 4; q++) {
                                if (ib + q < nx && zn[q] > thr && hv[q] > CC_GX && !skip[q]) {
                                    int *a = arrival + (size_t)r * P + ib + q;
                                    /* GC_F_ARR_BYMAX: max-eta has taken every step
                                     * since the start, so a wet cell whose max so
                                     * far is at or below the threshold has not
                                     * arrived (cells starting above it start at
                                     * step 0), and the arrival field need not be read */
                                    if (by_max) {
                                        if (xo[q] <= thr) *a = local + 1;
                                    } else if (*a < 0) {
                                        *a = local + 1;
                                    }
                                }
                            }
                        }
                    }
                }
            }
            __syncwarp();
            /* momentum of row j = r-1 (MOMT_S, moment.f90:86-145) */
            const int j = r - 1;
            if (k >= 2 && j < ny && own) {
                const float *mB = SB + ST::M / 4 + 4, *mA = SA + ST::M / 4 + 4;
                const float *hB = SB + ST::H / 4, *hA = SA + ST::H / 4;
                [[maybe_unused]] float cx = 0.0f, cy = 0.0f; /* explicit R2/R4 fields need neither */
                if constexpr (!XR24) { cx = SB[ST::C / 4 + GC_CX]; cy = SB[ST::C / 4 + GC_CY]; }
                const float r3 = SB[ST::C / 4 + GC_R3], r5 = SB[ST::C / 4 + GC_R5];
                /* columns c0..c0+4 of H, N(j), N(j-1), Z2(j); c0-1..c0+3 of M(j), M(j+1) */
                float hb[5], nb[5], nc[5], zb[5], mb[5], ma[5], ha[4], za[4];
                {
                    float4 t;
                    t = lds4(hB + c0); hb[0] = t.x; hb[1] = t.y; hb[2] = t.z; hb[3] = t.w; hb[4] = hB[c0 + 4];
                    if constexpr (NC) {
#pragma unroll
                        for (int q = 0; q < 5; q++) { nb[q] = nbk[q]; nc[q] = nck[q]; }
                    } else {
                        const float *nB = SB + ST::N / 4, *nC = SC + ST::N / 4;
                        t = lds4(nB + c0); nb[0] = t.x; nb[1] = t.y; nb[2] = t.z; nb[3] = t.w; nb[4] = nB[c0 + 4];
                        t = lds4(nC + c0); nc[0] = t.x; nc[1] = t.y; nc[2] = t.z; nc[3] = t.w; nc[4] = nC[c0 + 4];
                    }
                    t = lds4(zB + c0); zb[0] = t.x; zb[1] = t.y; zb[2] = t.z; zb[3] = t.w; zb[4] = zB[c0 + 4];
                    t = lds4(mB + c0); mb[0] = mB[c0 - 1]; mb[1] = t.x; mb[2] = t.y; mb[3] = t.z; mb[4] = t.w;
                    t = lds4(mA + c0); ma[0] = mA[c0 - 1]; ma[1] = t.x; ma[2] = t.y; ma[3] = t.z; ma[4] = t.w;
                    t = lds4(hA + c0); ha[0] = t.x; ha[1] = t.y; ha[2] = t.z; ha[3] = t.w;
                    t = lds4(zA + c0); za[0] = t.x; za[1] = t.y; za[2] = t.z; za[3] = t.w;
                }
                float xm[4], xn[4];
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const int i = ib + q;
                    const float h0 = hb[q], hp1 = hb[q + 1];
                    bool mdom = true, ndom = true;
                    if constexpr (EDGE) {
                        mdom = root ? (i <= nx - 2) : (i >= 1 && i <= nx - 2 && j >= 1);
                        ndom = (root ? (j <= ny - 2) : (i >= 1 && j >= 1 && j <= ny - 2)) && i < nx;
                    }
                    /* evaluated unconditionally, then selected: four independent
                     * straight-line chains per lane */
                    const float tot_n = nb[q] + nb[q + 1] + nc[q] + nc[q + 1];
                    float r2, r4;
                    if constexpr (XR24) {
                        r2 = __ldg(Gref.r2 + (size_t)j * P + i);
                        r4 = __ldg(Gref.r4 + (size_t)j * P + i);
                    } else {
                        r2 = cx * (0.5f * (h0 + hp1));
                        r4 = cy * (0.5f * (h0 + ha[q]));
                    }
                    float vm = mb[q + 1] - r2 * (zb[q + 1] - zb[q]) + r3 * tot_n;
                    vm = (fabsf(vm) < CC_EPS) ? 0.0f : vm;
                    xm[q] = (mdom && h0 > CC_GX && hp1 > CC_GX) ? vm : 0.0f;
                    const float tot_m = mb[q] + ma[q] + mb[q + 1] + ma[q + 1];
                    float vn = nb[q] - r4 * (za[q] - zb[q]) - r5 * tot_m;
                    vn = (fabsf(vn) < CC_EPS) ? 0.0f : vn;
                    xn[q] = (ndom && h0 > CC_GX && ha[q] > CC_GX) ? vn : 0.0f;
                }
                if constexpr (EDGE) {
                    st4p(m2p, ib, nx, xm);
                    st4p(n2p, ib, nx, xn);
                } else {
                    *reinterpret_cast<float4 *>(m2p) = make_float4(xm[0], xm[1], xm[2], xm[3]);
                    *reinterpret_cast<float4 *>(n2p) = make_float4(xn[0], xn[1], xn[2], xn[3]);
                }
            }
        };
        if (edge) body(std::true_type{});
        else body(std::false_type{});
        z2p += P;
        zxp += P;
        if (k >= 2) { m2p += P; n2p += P; }
        __syncwarp();
        if constexpr (NC) {
            /* row k-1 is no longer needed (its N rides on in registers) */
#pragma unroll
            for (int q = 0; q < 5; q++) nck[q] = nbk[q];
            if (k - 1 + S < K) issue(k - 1 + S, stB);
        } else {
            /* row k-2 is no longer needed: refill its stage S rows ahead */
            if (k >= 2 && k - 2 + S < K) issue(k - 2 + S, stC);
        }
        stC = stB; stB = stA; parB = parA;
    }
    seq = seq0 + K;
    if (!ok) {
        /* record the failure, then give the copies still in flight a bounded
         * chance to land before the warp leaves */
        if (lane == 0) atomicExch(&g_pipe_error, 1);
        for (int k = 0; k < K; k++) {
            const int n = seq0 + k;
            mbar_wait(bars + 8 * (n % S), (uint32_t)((n / S) & 1), 1 << 12);
        }
        return false;
    }
    __syncwarp();
    return true;
}

template <int W, int S, int FL, bool MULTI>
__global__ void __launch_bounds__(32 * W) k_fused(GcFusedGrid one, const GcFusedGrid *__restrict__ grids,
                                                   const int2 *__restrict__ tiles, int ntiles,
                                                   const int *__restrict__ step_base, int step_off) {
    extern __shared__ __align__(128) char smem[];
    /* programmatic dependent launch: the previous step's kernel has finished
     * and its writes are visible past this point (no-op for plain launches) */
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    const int step = step_off + (step_base ? *step_base : 0);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    char *wsm = smem + warp * warp_smem_bytes<FL>(S);
    const uint32_t bars = smem_u32(wsm) + S * Stage<FL>::BYTES + 2 * ZR_FLOATS * 4;
    if (lane == 0) {
        for (int s = 0; s < S; s++) mbar_init(bars + 8 * s, 1);
        fence_mbar_init();
    }
    __syncwarp();
    int seq = 0;
    for (int tile = blockIdx.x * W + warp; tile < ntiles; tile += gridDim.x * W) {
        bool ok;
        if (MULTI) {
            const int2 w = tiles[tile];
            const GcFusedGrid &G = grids[w.x];
            ok = G.explicit_r24 ? warp_tile<S, true, FL>(G, w.y, step, wsm, seq)
                                : warp_tile<S, false, FL>(G, w.y, step, wsm, seq);
        } else {
            ok = one.explicit_r24 ? warp_tile<S, true, FL>(one, tile, step, wsm, seq)
                                  : warp_tile<S, false, FL>(one, tile, step, wsm, seq);
        }
        if (!ok) return;
    }
}

struct Variant {
    int w, s, fl;
    void (*one)(GcFusedGrid, const GcFusedGrid *, const int2 *, int, const int *, int);
    void (*multi)(GcFusedGrid, const GcFusedGrid *, const int2 *, int, const int *, int);
};

#define GC_VARIANT(W, S, FL) {W, S, FL, k_fused<W, S, FL, false>, k_fused<W, S, FL, true>}
const Variant kVariants[] = {
    GC_VARIANT(4, 6, 0), GC_VARIANT(2, 8, 0), GC_VARIANT(4, 8, 0), GC_VARIANT(8, 5, 0),
    GC_VARIANT(1, 8, 0), GC_VARIANT(2, 6, 0), GC_VARIANT(4, 5, 0), GC_VARIANT(8, 4, 0),
    GC_VARIANT(4, 6, FL_ONE), GC_VARIANT(8, 4, FL_ONE),
    GC_VARIANT(4, 6, FL_ZD), GC_VARIANT(8, 4, FL_ZD), GC_VARIANT(4, 4, FL_ZD),
    GC_VARIANT(4, 6, FL_ONE | FL_ZD), GC_VARIANT(8, 4, FL_ONE | FL_ZD), GC_VARIANT(4, 4, FL_ONE | FL_ZD),
    GC_VARIANT(4, 3, FL_NC), GC_VARIANT(2, 3, FL_NC), GC_VARIANT(4, 4, FL_NC),
};
#undef GC_VARIANT
constexpr int kNumVariants = sizeof(kVariants) / sizeof(kVariants[0]);

int variant_smem(const Variant &v) {
    /* the stage layout depends on FL_ZD alone */
    return v.w * ((v.fl & FL_ZD) ? warp_smem_bytes<FL_ZD>(v.s) : warp_smem_bytes<0>(v.s));
}

/* the dynamic shared-memory limit of a variant's kernels, set once per
 * device (the attribute belongs to the device that is current when it is set) */
constexpr int kMaxDevices = 64;
static_assert(kNumVariants <= 64, "one flag per variant");
std::atomic<uint64_t> g_prepared[kMaxDevices];
std::mutex g_prepare_mu;

void prepare(const Variant &v) {
    const int idx = (int)(&v - kVariants);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) dev = 0;
    const uint64_t bit = 1ull << idx;
    if (g_prepared[dev].load(std::memory_order_acquire) & bit) return;
    std::lock_guard<std::mutex> lock(g_prepare_mu);
    if (g_prepared[dev].load(std::memory_order_relaxed) & bit) return;
    cudaFuncSetAttribute(v.one, cudaFuncAttributeMaxDynamicSharedMemorySize, variant_smem(v));
    cudaFuncSetAttribute(v.multi, cudaFuncAttributeMaxDynamicSharedMemorySize, variant_smem(v));
    g_prepared[dev].fetch_or(bit, std::memory_order_release);
}

} // namespace

int gc_fused_num_variants() { return kNumVariants; }

/* ordinary launch, or with programmatic stream serialization when the
 * calling thread asked for it (gc_set_pdl) */
static cudaError_t launch_fused(void (*kern)(GcFusedGrid, const GcFusedGrid *, const int2 *, int, const int *, int),
                         int ctas, int threads, int smem, cudaStream_t s, const GcFusedGrid &g,
                         const GcFusedGrid *grids, const int2 *tiles, int ntiles, const int *step_base, int step_off) {
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
    return cudaLaunchKernelEx(&cfg, kern, g, grids, tiles, ntiles, step_base, step_off);
}

/* 1 if a pipeline wait in the fused kernel gave up since the last call */
int gc_fused_take_error() {
    int v = 0, z = 0;
    cudaMemcpyFromSymbol(&v, g_pipe_error, sizeof v);
    if (v) cudaMemcpyToSymbol(g_pipe_error, &z, sizeof z);
    return v;
}

/* clears the pipeline-error flag in stream order (no host memory involved) */
cudaError_t gc_fused_clear_error_async(cudaStream_t s) {
    void *addr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&addr, g_pipe_error);
    if (e != cudaSuccess) return e;
    return cudaMemsetAsync(addr, 0, sizeof(int), s);
}

GcTileCfg gc_fused_variant(int v) {
    if (v < 0 || v >= kNumVariants) v = 0;
    return GcTileCfg{kVariants[v].w, kVariants[v].s};
}

int gc_fused_tiles(int nx, int ny, int ty, int *tiles_x) {
    int tx = (nx + TXW - 1) / TXW, tyn = (ny + ty - 1) / ty;
    if (tiles_x) *tiles_x = tx;
    return tx * tyn;
}

int gc_fused_pick_ty(int variant, int ngrids, const int *nx, const int *ny, int rule, bool multi) {
    const int slots = gc_fused_max_ctas(variant, multi) * gc_fused_variant(variant).warps;
    auto tiles = [&](int ty) {
        long long t = 0;
        for (int g = 0; g < ngrids; g++) t += gc_fused_tiles(nx[g], ny[g], ty, nullptr);
        return t;
    };
    if (rule == 0) {
        /* the number of waves 16-row tiles need, then the shortest tiles
         * that keep to it (short tiles interleave members' reads of a shared
         * bathymetry tile closely in time) */
        long long waves = (tiles(16) + slots - 1) / slots;
        if (waves < 1) waves = 1;
        for (int ty = 8; ty <= 256; ty++)
            if (tiles(ty) <= waves * slots) return ty;
        return 256;
    }
    /* a launch lasts as long as its busiest warp: waves x (rows per tile plus
     * the row above, the halo row below and about one row of pipeline fill);
     * the height that minimises it, ties to fewer waves */
    int best = 16;
    long long best_cost = -1, best_waves = 0;
    for (int ty = 4; ty <= 256; ty++) {
        const long long waves = (tiles(ty) + slots - 1) / slots;
        const long long cost = waves * (ty + 3);
        if (best_cost < 0 || cost < best_cost || (cost == best_cost && waves < best_waves)) {
            best = ty;
            best_cost = cost;
            best_waves = waves;
        }
    }
    return best;
}

cudaError_t gc_fused_launch_one(int variant, const GcFusedGrid &g, int step, cudaStream_t s) {
    if (variant < 0 || variant >= kNumVariants) variant = 0;
    const Variant &v = kVariants[variant];
    int ntiles = gc_fused_tiles(g.nx, g.ny, g.ty, nullptr);
    prepare(v);
    return launch_fused(v.one, (ntiles + v.w - 1) / v.w, 32 * v.w, variant_smem(v), s, g, nullptr, nullptr, ntiles,
                        nullptr, step);
}

cudaError_t gc_fused_launch_one_at(int variant, const GcFusedGrid &g, const int *d_step_base, int step_off,
                                   cudaStream_t s) {
    if (variant < 0 || variant >= kNumVariants) variant = 0;
    const Variant &v = kVariants[variant];
    int ntiles = gc_fused_tiles(g.nx, g.ny, g.ty, nullptr);
    prepare(v);
    return launch_fused(v.one, (ntiles + v.w - 1) / v.w, 32 * v.w, variant_smem(v), s, g, nullptr, nullptr, ntiles,
                        d_step_base, step_off);
}

int gc_fused_max_ctas(int variant, bool multi) {
    if (variant < 0 || variant >= kNumVariants) variant = 0;
    const Variant &v = kVariants[variant];
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    prepare(v);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, multi ? v.multi : v.one, 32 * v.w, variant_smem(v));
    return sms * (per > 0 ? per : 1);
}

cudaError_t gc_fused_launch_multi(int variant, const GcFusedGrid *d_grids, const int2 *d_tiles,
                                  int ntiles, const int *d_step_base, int step_off, int nctas,
                                  cudaStream_t s) {
    if (variant < 0 || variant >= kNumVariants) variant = 0;
    const Variant &v = kVariants[variant];
    if (ntiles <= 0) return cudaSuccess;
    const int need = (ntiles + v.w - 1) / v.w;
    if (nctas <= 0 || nctas > need) nctas = need;
    GcFusedGrid dummy;
    memset(&dummy, 0, sizeof dummy);
    prepare(v);
    return launch_fused(v.multi, nctas, 32 * v.w, variant_smem(v), s, dummy, d_grids, d_tiles, ntiles, d_step_base,
                        step_off);
}
