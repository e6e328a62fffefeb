/*
 * Layer registry and the reference's C ABI (GPUcomcot.cu, GPUMass_s.cu,
 * GPUMoment_s.cu, GPUOpen_BD.cu, GPUall_grids.cu, GPUOutput.cu entry points).
 *
 * Every export keeps the reference's gfortran calling convention: lower-case
 * name with a trailing underscore, every argument by reference, arrays as the
 * address of a contiguous column-major NX x NY section.  Like the reference,
 * these legacy entry points have no return code and stop the program on a
 * CUDA error.  Unlike the reference they do not synchronise after every
 * launch: all work is ordered on one library stream and every call that hands
 * data back to the host synchronises, which the caller cannot tell apart.
 *
 * Time levels follow the Fortran copy semantics (CHANGE / UPDATE copy level 2
 * into level 1) although the device swaps buffers: readers of Z(:,:,2) after a
 * swap are served from the buffer that now holds level 1, which has the same
 * contents the Fortran Z(:,:,2) would have.
 */
#include <math.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <thread>
#include <vector>

#include "runtime.h"

void gc_gauge_invalidate();
bool gc_gauge_lookup(int lid, int i, int j, float *out4);
void gc_gauge_release();

static GcRuntime g_rt;
GcRuntime &gc_rt() { return g_rt; }

const char *gc_status_str(int code) {
    switch (code) {
    case GC_OK: return "ok";
    case GC_EINVAL: return "invalid argument";
    case GC_ENOMEM: return "out of device memory";
    case GC_ECUDA: return "CUDA error";
    case GC_ESTATE: return "invalid state";
    case GC_ETIMEOUT: return "timeout";
    case GC_ENOTSUP: return "not supported";
    default: return "unknown";
    }
}

GcLayer *gc_layer(int id) {
    if (id < 0 || id >= GC_MAX_LAYERS) {
        fprintf(stderr, "invalid layer id %d\n", id);
        return nullptr;
    }
    return &g_rt.layers[id];
}

static GcLayer &layer_or_die(int id) {
    GcLayer *L = gc_layer(id);
    if (!L || !L->used) {
        fprintf(stderr, "gcomcot: layer %d is not initialised\n", id);
        exit(EXIT_FAILURE);
    }
    return *L;
}

GcLayerDev GcLayer::view() const {
    GcLayerDev d;
    memset(&d, 0, sizeof d);
    d.nx = nx; d.ny = ny; d.pitch = pitch;
    d.root = (parent == -1) ? 1 : 0;
    d.laycord = laycord; d.laygov = laygov; d.linchk = linchk; d.modscm = modscm;
    d.fric_switch = fric_switch;
    d.explicit_r24 = explicit_r24 ? 1 : 0;
    d.rx = rx; d.ry = ry; d.grx = grx; d.gry = gry; d.dt = dt; d.fric_coef = fric_coef;
    int o = cur ^ 1;
    d.z1 = z[cur]; d.m1 = m[cur]; d.n1 = n[cur];
    d.z1w = z[cur]; d.m1w = m[cur]; d.n1w = n[cur];
    d.z2 = z[o]; d.m2 = m[o]; d.n2 = n[o];
    d.h = h; d.hp = hp; d.hq = hq; d.r2 = r2; d.r4 = r4; d.rows = rows; d.dz2 = dz2; d.rows2 = rows2;
    d.xflux = xflux; d.yflux = yflux; d.zmax = zmax; d.arrival = arrival;
    return d;
}

/* ------------------------------------------------------------------ */
/* storage                                                             */
/* ------------------------------------------------------------------ */
static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

int gc_layer_alloc(GcLayer &L) {
    L.pitch = (L.nx + 31) & ~31;
    size_t field = align256((size_t)L.pitch * L.ny * sizeof(float));
    size_t rows = align256((size_t)GC_ROWW * L.ny * sizeof(float));
    size_t nfield = 6 /* z,m,n x2 */ + 1 /* h */ + 1 /* zmax */ + 1 /* arrival */;
    bool cart = L.laycord == 1 || L.laygov == 1; /* layers that read HP, HQ */
    bool nls = L.laycord == 0 && L.laygov == 1;  /* nonlinear spherical: R0, R22 rows */
    if (cart) nfield += 2;           /* hp, hq */
    if (L.laygov == 1) nfield += 1;  /* dz2 */
    if (L.explicit_r24) nfield += 2; /* r2, r4 */
    size_t flux = align256((size_t)2 * L.nx * sizeof(float)) + align256((size_t)2 * L.ny * sizeof(float));
    size_t rows2b = nls ? align256((size_t)2 * L.ny * sizeof(float)) : 0;
    size_t total = nfield * field + rows + flux + rows2b;
    void *blk = nullptr;
    cudaError_t e = cudaMalloc(&blk, total);
    if (e != cudaSuccess) {
        fprintf(stderr, "gcomcot: cudaMalloc(%zu) for layer %d: %s\n", total, L.id, cudaGetErrorString(e));
        return GC_ENOMEM;
    }
    GC_CUDA_OR_RET(cudaMemsetAsync(blk, 0, total, g_rt.stream));
    char *p = (char *)blk;
    auto take = [&](size_t b) { char *q = p; p += b; return q; };
    for (int k = 0; k < 2; k++) {
        L.z[k] = (float *)take(field);
        L.m[k] = (float *)take(field);
        L.n[k] = (float *)take(field);
    }
    L.h = (float *)take(field);
    L.zmax = (float *)take(field);
    L.arrival = (int *)take(field);
    L.hp = cart ? (float *)take(field) : nullptr;
    L.hq = cart ? (float *)take(field) : nullptr;
    L.dz2 = (L.laygov == 1) ? (float *)take(field) : nullptr;
    L.r2 = L.explicit_r24 ? (float *)take(field) : nullptr;
    L.r4 = L.explicit_r24 ? (float *)take(field) : nullptr;
    L.rows = (float *)take(rows);
    L.xflux = (float *)take(align256((size_t)2 * L.nx * sizeof(float)));
    L.yflux = (float *)take(align256((size_t)2 * L.ny * sizeof(float)));
    L.rows2 = nls ? (float *)take(rows2b) : nullptr;
    L.block = blk;
    L.block_bytes = total;
    /* arrival starts at -1 (no arrival yet) */
    GC_CUDA_OR_RET(cudaMemsetAsync(L.arrival, 0xff, (size_t)L.pitch * L.ny * sizeof(int), g_rt.stream));
    L.cur = 0;
    L.z2_valid = false;
    L.mn2_valid = false;
    return GC_OK;
}

int gc_layer_upload_field(GcLayer &L, float *dst, const float *src) {
    GC_CUDA_OR_RET(cudaMemcpy2DAsync(dst, (size_t)L.pitch * sizeof(float), src,
                                     (size_t)L.nx * sizeof(float), (size_t)L.nx * sizeof(float),
                                     (size_t)L.ny, cudaMemcpyHostToDevice, g_rt.stream));
    GC_CUDA_OR_RET(cudaStreamSynchronize(g_rt.stream));
    return GC_OK;
}

int gc_layer_download_field(GcLayer &L, const float *src, float *dst) {
    GC_CUDA_OR_RET(cudaMemcpy2DAsync(dst, (size_t)L.nx * sizeof(float), src,
                                     (size_t)L.pitch * sizeof(float), (size_t)L.nx * sizeof(float),
                                     (size_t)L.ny, cudaMemcpyDeviceToHost, g_rt.stream));
    GC_CUDA_OR_RET(cudaStreamSynchronize(g_rt.stream));
    return GC_OK;
}

/* R2 = C(J) * AMAX1(HP(I,J),0) (comcot.f90:733-736) with HP from PQ_DEPTH
 * (initialization.f90:2512-2523).  Returns the per-row factors when the
 * caller's field has exactly that form in every cell, so the kernels can
 * rebuild R2 from H instead of streaming a second field. */
static bool factor_row(int nx, int ny, int j, const float *H, const float *R, bool xdir, float *hp, float *fac) {
    float best = 0.0f;
    int bi = -1;
    for (int i = 0; i < nx; i++) {
        size_t c = (size_t)j * nx + i;
        float v = 0.0f;
        if (H[c] > CC_GX) {
            size_t c2;
            if (xdir) c2 = (size_t)j * nx + std::min(i + 1, nx - 1);
            else c2 = (size_t)std::min(j + 1, ny - 1) * nx + i;
            v = 0.5f * (H[c] + H[c2]);
        }
        hp[i] = v > 0.0f ? v : 0.0f;
        if (hp[i] > best) { best = hp[i]; bi = i; }
    }
    float cands[3];
    int nc;
    if (bi < 0) {
        cands[0] = 0.0f; nc = 1;
    } else {
        float c0 = (float)((double)R[(size_t)j * nx + bi] / (double)best);
        cands[0] = c0; cands[1] = nextafterf(c0, 3.0e38f); cands[2] = nextafterf(c0, -3.0e38f);
        nc = 3;
    }
    for (int k = 0; k < nc; k++) {
        bool ok = true;
        for (int i = 0; i < nx && ok; i++) {
            float want = R[(size_t)j * nx + i];
            float got = cands[k] * hp[i];
            if (memcmp(&want, &got, sizeof(float)) != 0 && !(want == 0.0f && got == 0.0f)) ok = false;
        }
        if (ok) {
            fac[j] = cands[k];
            return true;
        }
    }
    return false;
}

/* rows are independent: host threads take every nt-th row */
static bool factor_rows(int nx, int ny, const float *H, const float *R, bool xdir, float *fac) {
    const unsigned hw = std::thread::hardware_concurrency();
    const int nt = std::max(1, std::min({(int)(hw ? hw : 1), 16, (int)(((size_t)nx * ny) >> 18) + 1}));
    std::atomic<bool> all_ok{true};
    auto work = [&](int t) {
        std::vector<float> hp((size_t)nx);
        for (int j = t; j < ny && all_ok.load(std::memory_order_relaxed); j += nt)
            if (!factor_row(nx, ny, j, H, R, xdir, hp.data(), fac)) all_ok.store(false);
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; t++) pool.emplace_back(work, t);
    work(0);
    for (auto &th : pool) th.join();
    return all_ok.load();
}

static void init_runtime() {
    if (g_rt.inited) return;
    GC_CUDA_OR_DIE(cudaStreamCreateWithFlags(&g_rt.stream, cudaStreamNonBlocking));
    g_rt.inited = true;
    g_rt.root = -1;
    const char *f = getenv("GCOMCOT_FUSE");
    g_rt.fuse_enabled = (f && f[0] == '0') ? 0 : 1;
}

void gc_swap(GcLayer &L) {
    L.cur ^= 1;
    L.z2_valid = false;
    L.mn2_valid = false;
}

/* ------------------------------------------------------------------ */
/* reference ABI                                                       */
/* ------------------------------------------------------------------ */
extern "C" {

/* GPUcomcot.cu:192-211 */
void gcomcot_init_gpu_(void) {
    int dev = 0;
    GC_CUDA_OR_DIE(cudaGetDevice(&dev));
    cudaDeviceProp prop;
    GC_CUDA_OR_DIE(cudaGetDeviceProperties(&prop, dev));
    if (!getenv("GCOMCOT_QUIET")) {
        printf("GPU INFORMATIONS:                      %s\n", prop.name);
        printf("-->Compute Capabilities [Major.Minor]: %d.%d\n", prop.major, prop.minor);
        printf("-->Streaming Multi-Processor Count:    %d\n", prop.multiProcessorCount);
    }
    init_runtime();
}

/* extension: layer physics the reference ABI cannot express (coordinate
 * system, governing equation, Cartesian ratios, friction, HP/HQ).  Call it
 * before gcomcot_init_layer_ for every layer that is not linear spherical. */
void gcomcot_set_layer_params_(int *id, int *laycord, int *laygov, float *dt, float *rx, float *ry,
                               float *grx, float *gry, int *fric_switch, float *fric_coef,
                               int *linchk, int *modscm, int *nx, int *ny, float *HP, float *HQ) {
    init_runtime();
    if (*id < 0 || *id >= GC_MAX_LAYERS) {
        fprintf(stderr, "ERROR: invalid layerid\n");
        exit(EXIT_FAILURE);
    }
    if (*laycord < 0 || *laycord > 1 || *laygov < 0 || *laygov > 3) {
        fprintf(stderr, "gcomcot: LAYCORD=%d LAYGOV=%d is not supported (0-1, 0-3)\n", *laycord, *laygov);
        exit(EXIT_FAILURE);
    }
    if (*fric_switch != 0 && *fric_switch != 1) {
        fprintf(stderr, "gcomcot: FRIC_SWITCH=%d is not supported (0 or 1)\n", *fric_switch);
        exit(EXIT_FAILURE);
    }
    GcPendingParams &p = g_rt.pending[*id];
    p.set = true;
    p.laycord = *laycord; p.laygov = *laygov; p.dt = *dt; p.rx = *rx; p.ry = *ry;
    p.grx = *grx; p.gry = *gry; p.fric_switch = *fric_switch; p.fric_coef = *fric_coef;
    p.linchk = *linchk; p.modscm = *modscm;
    size_t cells = (size_t)(*nx) * (*ny);
    p.hp.assign(HP ? HP : (const float *)nullptr, HP ? HP + cells : (const float *)nullptr);
    p.hq.assign(HQ ? HQ : (const float *)nullptr, HQ ? HQ + cells : (const float *)nullptr);
}

/* extension: the nonlinear spherical advection coefficients of PARA
 * (comcot.f90:727-733): R0, R21 (= R1) and R22, NX x NY arrays read at row
 * I = 1 like R1.  Call before gcomcot_init_layer_ for a layer with
 * LAYCORD = 0, LAYGOV = 1, after gcomcot_set_layer_params_. */
void gcomcot_set_layer_coefs_(int *id, float *R0, float *R21, float *R22, int *nx, int *ny) {
    init_runtime();
    (void)R21;
    if (*id < 0 || *id >= GC_MAX_LAYERS || *nx < 1 || *ny < 1 || !R0 || !R22) {
        fprintf(stderr, "ERROR: invalid layerid or coefficient arrays\n");
        exit(EXIT_FAILURE);
    }
    GcPendingParams &p = g_rt.pending[*id];
    p.r0.resize((size_t)*ny);
    p.r22.resize((size_t)*ny);
    for (int j = 0; j < *ny; j++) {
        p.r0[j] = R0[(size_t)j * *nx];
        p.r22[j] = R22[(size_t)j * *nx];
    }
}

/* extension: the SC_OPTION = 1 tables of a Cartesian child of a spherical
 * parent, POS(NX,NY,2) and CXY(NX,NY,4) as SUBGRID_MATCHING builds them
 * (initialization.f90:1065-1124), the parent's MODSCM (the band forecast of
 * NEWQ_SC adds the modified-scheme term when it is 0) and FIX_TOP (1: the
 * top edge blends C2*YN1; 0: C1*YN1 as all_grids.f90:1357 does).  Call
 * before gcomcot_init_layer_ of that child, whose corners are then the
 * extent of POS. */
void gcomcot_set_sc_tables_(int *id, int *pos, float *cxy, int *nx, int *ny, int *parent_modscm, int *fix_top) {
    init_runtime();
    if (*id < 0 || *id >= GC_MAX_LAYERS || *nx < 3 || *ny < 3 || !pos || !cxy) {
        fprintf(stderr, "ERROR: invalid layerid or SC tables\n");
        exit(EXIT_FAILURE);
    }
    GcPendingParams &p = g_rt.pending[*id];
    const size_t n = (size_t)(*nx) * (*ny);
    p.sc = true;
    p.sc_fix_top = *fix_top != 0;
    p.sc_modscm = *parent_modscm;
    p.sc_pos.assign(2 * n, 0);
    p.sc_cxy.assign(4 * n, 0.0f);
    for (size_t c = 0; c < n; c++) {
        for (int k = 0; k < 2; k++) p.sc_pos[2 * c + k] = pos[(size_t)k * n + c];
        for (int k = 0; k < 4; k++) p.sc_cxy[4 * c + k] = cxy[(size_t)k * n + c];
    }
}

} /* extern "C" */

/* device tables of an SC_OPTION = 1 child (see GcScView) from POS / CXY
 * in [ny][nx][2] and [ny][nx][4] order; returns nullptr when they are
 * usable, else what is wrong with them */
const char *gc_sc_tables(int nx, int ny, int cpitch, const int *pos, const float *cxy, const int corners[4],
                         int pnx, int pny, int rel_size, int fix_top, int modscm, GcScView *out, void **block,
                         size_t *bytes) {
    *block = nullptr;
    auto ki = [&](int i, int j) { return pos[2 * ((size_t)j * nx + i)]; };
    auto kj = [&](int i, int j) { return pos[2 * ((size_t)j * nx + i) + 1]; };
    /* every node inside the parent with its whole 2x2 stencil */
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++)
            if (ki(i, j) < 1 || kj(i, j) < 1 || ki(i, j) > pnx - 1 || kj(i, j) > pny - 1)
                return "a node lies outside the parent's interior";
    const int c0 = corners[0], c1 = corners[1], c2 = corners[2], c3 = corners[3];
    if (c0 < 1 || c2 < 1 || c1 > pnx || c3 > pny || c1 < c0 || c3 < c2) return "corners outside the parent";
    const int ne = 2 * ny + 2 * nx;
    std::vector<int2> epos(ne);
    std::vector<float4> ew(ne);
    auto put = [&](int k, int i, int j) {
        const size_t c = (size_t)j * nx + i;
        epos[k] = make_int2(ki(i, j), kj(i, j));
        ew[k] = make_float4(cxy[4 * c], cxy[4 * c + 1], cxy[4 * c + 2], cxy[4 * c + 3]);
    };
    for (int j = 0; j < ny; j++) { put(j, 0, j); put(ny + j, nx - 1, j); }
    for (int i = 0; i < nx; i++) { put(2 * ny + i, i, 0); put(2 * ny + nx + i, i, ny - 1); }
    /* the parent window and, per parent cell, the child nodes in it, child
     * I outermost as JNZ_SC sums them */
    const int ww = c1 - c0 + 1, wh = c3 - c2 + 1;
    std::vector<int> start((size_t)ww * wh + 1, 0), cell;
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++) {
            const int a = ki(i, j), b = kj(i, j);
            if (a >= c0 && a <= c1 && b >= c2 && b <= c3) start[(size_t)(b - c2) * ww + (a - c0) + 1]++;
        }
    for (size_t q = 0; q < (size_t)ww * wh; q++) start[q + 1] += start[q];
    cell.resize((size_t)start.back());
    std::vector<int> fill(start.begin(), start.end() - 1);
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++) {
            const int a = ki(i, j), b = kj(i, j);
            if (a >= c0 && a <= c1 && b >= c2 && b <= c3) cell[fill[(size_t)(b - c2) * ww + (a - c0)]++] = j * cpitch + i;
        }
    /* forecast bands (all_grids.f90:1131-1134, 1165-1168, 1199-1202, 1233-1236), 0-based */
    GcScView v{};
    auto band = [&](int b, int i0, int i1, int j0, int j1, bool xflux) {
        /* the M band reads column I+1, the N band row J+1 */
        if (i0 < 1 || j0 < 1 || (xflux ? i1 + 1 > pnx || j1 > pny : i1 > pnx || j1 + 1 > pny)) return false;
        v.band[b][0] = i0 - 1; v.band[b][1] = i1 - 1; v.band[b][2] = j0 - 1; v.band[b][3] = j1 - 1;
        return true;
    };
    int a = ki(0, 0), b = ki(0, ny - 1);
    bool ok = band(0, std::min(a, b) - 2, std::max(a, b) + 2, c2 - 2, c3 + 2, true);
    a = ki(nx - 1, 0); b = ki(nx - 1, ny - 1);
    ok = ok && band(1, std::min(a, b) - 2, std::max(a, b) + 2, c2 - 2, c3 + 2, true);
    a = kj(0, ny - 1); b = kj(nx - 1, ny - 1);
    ok = ok && band(2, c0 - 2, c1 + 2, std::min(a, b) - 2, std::max(a, b) + 2, false);
    a = kj(0, 0); b = kj(nx - 1, 0);
    ok = ok && band(3, c0 - 2, c1 + 2, std::min(a, b) - 2, std::max(a, b) + 2, false);
    if (!ok) return "a forecast band reaches past the parent's edge";
    const size_t b_epos = ((size_t)ne * sizeof(int2) + 255) & ~(size_t)255;
    const size_t b_ew = ((size_t)ne * sizeof(float4) + 255) & ~(size_t)255;
    const size_t b_start = (start.size() * sizeof(int) + 255) & ~(size_t)255;
    const size_t b_cell = ((cell.size() + 1) * sizeof(int) + 255) & ~(size_t)255;
    char *blk = nullptr;
    if (cudaMalloc((void **)&blk, b_epos + b_ew + b_start + b_cell) != cudaSuccess) return "device allocation failed";
    bool copied = cudaMemcpy(blk, epos.data(), ne * sizeof(int2), cudaMemcpyHostToDevice) == cudaSuccess
                  && cudaMemcpy(blk + b_epos, ew.data(), ne * sizeof(float4), cudaMemcpyHostToDevice) == cudaSuccess
                  && cudaMemcpy(blk + b_epos + b_ew, start.data(), start.size() * sizeof(int),
                                cudaMemcpyHostToDevice) == cudaSuccess
                  && (cell.empty() || cudaMemcpy(blk + b_epos + b_ew + b_start, cell.data(), cell.size() * sizeof(int),
                                                 cudaMemcpyHostToDevice) == cudaSuccess);
    if (!copied) {
        cudaFree(blk);
        return "device copy failed";
    }
    v.epos = (const int2 *)blk;
    v.ew = (const float4 *)(blk + b_epos);
    v.start = (const int *)(blk + b_epos + b_ew);
    v.cell = (const int *)(blk + b_epos + b_ew + b_start);
    v.wi0 = c0 - 1; v.wi1 = c1 - 1; v.wj0 = c2 - 1; v.wj1 = c3 - 1;
    v.fix_top = fix_top;
    v.modscm = modscm;
    v.half = (float)(rel_size * rel_size) / 2.0f;
    *out = v;
    *block = blk;
    if (bytes) *bytes = b_epos + b_ew + b_start + b_cell;
    return nullptr;
}

/* device tables of an SC_OPTION = 1 child */
static void sc_build(GcLayer &L, const GcLayer &P, const GcPendingParams &pp) {
    if (pp.sc_pos.size() != (size_t)2 * L.nx * L.ny) {
        fprintf(stderr, "gcomcot: SC tables of layer %d: sized for another layer\n", L.id);
        exit(EXIT_FAILURE);
    }
    const char *err = gc_sc_tables(L.nx, L.ny, L.pitch, pp.sc_pos.data(), pp.sc_cxy.data(), L.corners, P.nx, P.ny,
                                   L.rel_size, pp.sc_fix_top, pp.sc_modscm, &L.sc, &L.sc_block, nullptr);
    if (err) {
        fprintf(stderr, "gcomcot: SC tables of layer %d: %s\n", L.id, err);
        exit(EXIT_FAILURE);
    }
    L.has_sc = true;
    L.sc_stepped = false;
}

extern "C" {

/* GPUcomcot.cu:214-251 */
void gcomcot_init_layer_(int *layerid, int *parent, int *level, int *rel_size, int *rel_time,
                         int *corners, float *grx, float *gry, float *R1_f, float *R2_f,
                         float *R3_f, float *R4_f, float *R5_f, float *R6_f, float *R11_f,
                         float *H_f, float *Z_f, int *row, int *col) {
    init_runtime();
    if (*layerid < 0) {
        printf("ERROR: invalid layerid\n");
        exit(-1);
    }
    if (*layerid >= GC_MAX_LAYERS) {
        printf("ERROR: number of layer exceed MAX_LAYERS\n");
        exit(-1);
    }
    GcLayer &L = g_rt.layers[*layerid];
    if (L.used && L.block) cudaFree(L.block);
    if (L.spx) cudaFree(L.spx);
    if (L.spy) cudaFree(L.spy);
    if (L.sc_block) cudaFree(L.sc_block);
    L = GcLayer();
    L.used = true;
    L.id = *layerid; L.parent = *parent; L.level = *level;
    L.rel_size = *rel_size; L.rel_time = *rel_time;
    memcpy(L.corners, corners, sizeof L.corners);
    L.grx = *grx; L.gry = *gry;
    L.nx = *row; L.ny = *col;
    const GcPendingParams &pp = g_rt.pending[*layerid];
    if (pp.set) {
        L.laycord = pp.laycord; L.laygov = pp.laygov; L.linchk = pp.linchk; L.modscm = pp.modscm;
        L.fric_switch = pp.fric_switch; L.dt = pp.dt; L.rx = pp.rx; L.ry = pp.ry;
        L.fric_coef = pp.fric_coef;
        if (pp.grx != 0.0f || pp.gry != 0.0f) { L.grx = pp.grx; L.gry = pp.gry; }
    }
    if (L.nx < 3 || L.ny < 3) {
        fprintf(stderr, "gcomcot: layer %d is %dx%d, need at least 3x3\n", L.id, L.nx, L.ny);
        exit(EXIT_FAILURE);
    }
    if (L.parent != -1) {
        GcLayer *P = gc_layer(L.parent);
        if (!P || !P->used) {
            printf("Error, Root grid is not initialized\n");
            exit(EXIT_FAILURE);
        }
        int is = L.corners[0], ie = L.corners[1], js = L.corners[2], je = L.corners[3];
        /* the NEWQ forecast reads parent rows JS-3 and columns IS-3
         * (all_grids.f90:692-700,765-772), so the window must start at 4 */
        /* an SC_OPTION = 1 child keeps the size of its original window; its
         * corners are the extent of its nodes' positions (initialization.f90:1120-1123) */
        const bool sized = pp.sc || (L.nx == (ie - is + 1) * L.rel_size + 1 && L.ny == (je - js + 1) * L.rel_size + 1);
        if (is < 4 || js < 4 || ie > P->nx - 2 || je > P->ny - 2 || ie < is || je < js || !sized
            || L.rel_size < 1 || L.rel_time < 1) {
            fprintf(stderr,
                    "gcomcot: layer %d corners (%d,%d,%d,%d) ratio %d do not match %dx%d inside "
                    "parent %dx%d\n",
                    L.id, is, ie, js, je, L.rel_size, L.nx, L.ny, P->nx, P->ny);
            exit(EXIT_FAILURE);
        }
        P->children.push_back(L.id);
    } else {
        g_rt.root = L.id;
    }
    const size_t cells = (size_t)L.nx * L.ny;
    /* spherical layers: try the factored R2/R4 form, else keep the fields */
    std::vector<float> rowblk((size_t)GC_ROWW * L.ny, 0.0f);
    if (L.laycord == 0) {
        std::vector<float> cx((size_t)L.ny, 0.0f), cy((size_t)L.ny, 0.0f);
        if (L.laygov == 1) {
            /* nonlinear spherical: R2, R4 carry no depth factor (comcot.f90:736-738,
             * 745-747), one value per row */
            for (int j = 0; j < L.ny; j++) {
                cx[j] = R2_f[(size_t)j * L.nx];
                cy[j] = R4_f[(size_t)j * L.nx];
            }
            L.explicit_r24 = false;
            if (!pp.set || pp.r0.size() != (size_t)L.ny || pp.r22.size() != (size_t)L.ny) {
                fprintf(stderr, "gcomcot: nonlinear spherical layer %d needs gcomcot_set_layer_coefs_ first\n", L.id);
                exit(EXIT_FAILURE);
            }
        } else {
            bool f2 = factor_rows(L.nx, L.ny, H_f, R2_f, true, cx.data());
            bool f4 = factor_rows(L.nx, L.ny, H_f, R4_f, false, cy.data());
            L.explicit_r24 = !(f2 && f4);
        }
        for (int j = 0; j < L.ny; j++) {
            float *rw = &rowblk[(size_t)j * GC_ROWW];
            rw[GC_R1] = R1_f[(size_t)j * L.nx];
            rw[GC_R11] = R11_f[(size_t)j * L.nx];
            rw[GC_R6] = R6_f[j];
            rw[GC_R3] = R3_f[(size_t)j * L.nx];
            rw[GC_R5] = R5_f[(size_t)j * L.nx];
            rw[GC_CX] = cx[j];
            rw[GC_CY] = cy[j];
        }
    }
    if (gc_layer_alloc(L) != GC_OK) exit(EXIT_FAILURE);
    GC_CUDA_OR_DIE(cudaMemcpyAsync(L.rows, rowblk.data(), rowblk.size() * sizeof(float),
                                   cudaMemcpyHostToDevice, g_rt.stream));
    if (gc_layer_upload_field(L, L.h, H_f) != GC_OK) exit(EXIT_FAILURE);
    if (gc_layer_upload_field(L, L.z[0], Z_f) != GC_OK) exit(EXIT_FAILURE);
    /* Zmax starts from the initial Z (GPUcomcot.cu:79): a device copy */
    GC_CUDA_OR_DIE(cudaMemcpyAsync(L.zmax, L.z[0], (size_t)L.pitch * L.ny * sizeof(float), cudaMemcpyDeviceToDevice,
                                   g_rt.stream));
    if (L.explicit_r24) {
        if (gc_layer_upload_field(L, L.r2, R2_f) != GC_OK) exit(EXIT_FAILURE);
        if (gc_layer_upload_field(L, L.r4, R4_f) != GC_OK) exit(EXIT_FAILURE);
    }
    if (L.rows2) {
        std::vector<float> r2b((size_t)2 * L.ny);
        for (int j = 0; j < L.ny; j++) { r2b[2 * j] = pp.r0[j]; r2b[2 * j + 1] = pp.r22[j]; }
        GC_CUDA_OR_DIE(cudaMemcpyAsync(L.rows2, r2b.data(), r2b.size() * sizeof(float), cudaMemcpyHostToDevice,
                                       g_rt.stream));
        GC_CUDA_OR_DIE(cudaStreamSynchronize(g_rt.stream));
    }
    if (L.hp) {
        /* HP/HQ from the caller, else PQ_DEPTH (initialization.f90:2501-2526) */
        std::vector<float> hp(cells, 0.0f), hq(cells, 0.0f);
        if (pp.set && pp.hp.size() == cells && pp.hq.size() == cells) {
            hp = pp.hp; hq = pp.hq;
        } else {
            for (int j = 0; j < L.ny; j++)
                for (int i = 0; i < L.nx; i++) {
                    size_t c = (size_t)j * L.nx + i;
                    if (H_f[c] > CC_GX) {
                        hp[c] = 0.5f * (H_f[c] + H_f[(size_t)j * L.nx + std::min(i + 1, L.nx - 1)]);
                        hq[c] = 0.5f * (H_f[c] + H_f[(size_t)std::min(j + 1, L.ny - 1) * L.nx + i]);
                    }
                }
        }
        if (gc_layer_upload_field(L, L.hp, hp.data()) != GC_OK) exit(EXIT_FAILURE);
        if (gc_layer_upload_field(L, L.hq, hq.data()) != GC_OK) exit(EXIT_FAILURE);
    }
    if (pp.sc) sc_build(L, *gc_layer(L.parent), pp);
    GC_CUDA_OR_DIE(cudaStreamSynchronize(g_rt.stream));
    if (!getenv("GCOMCOT_QUIET")) printf("Initializing layer id %d\n", L.id);
}

/* GPUMass_s.cu:9-37: host arrays are only used by the reference's debug compare */
void mass_launch_(const float *Z_f, float *Z_f_complete, const float *H_f, const int *lid) {
    gc_gauge_invalidate();
    (void)Z_f; (void)Z_f_complete; (void)H_f;
    GcLayer &L = layer_or_die(*lid);
    if (L.parent == -1 && g_rt.fuse_enabled) {
        gc_flush();
        g_rt.pend_mass = 1;
        L.z2_valid = true;
        return;
    }
    gc_flush();
    gc_launch_mass(L.view(), g_rt.stream);
    g_rt.launches++;
    L.z2_valid = true;
}

/* GPUOpen_BD.cu:13-37: outermost layer only */
void openbd_launch_(float *Z_f_complete) {
    gc_gauge_invalidate();
    (void)Z_f_complete;
    GcLayer &L = layer_or_die(g_rt.root);
    if (g_rt.pend_mass && !g_rt.pend_open && g_rt.fuse_enabled) {
        g_rt.pend_open = 1;
        return;
    }
    gc_flush();
    gc_launch_open(L.view(), g_rt.stream);
    g_rt.launches++;
}

/* GPUMoment_s.cu:10-56 */
void momt_launch_(float *M_f, float *N_f, float *Z_f, const int *lid) {
    gc_gauge_invalidate();
    (void)M_f; (void)N_f; (void)Z_f;
    GcLayer &L = layer_or_die(*lid);
    if (L.parent == -1 && g_rt.pend_mass && g_rt.pend_open && !g_rt.pend_momt) {
        g_rt.pend_momt = 1;
        L.mn2_valid = true;
        return;
    }
    gc_flush();
    gc_launch_moment(L.view(), g_rt.stream);
    g_rt.launches++;
    L.mn2_valid = true;
}

/* GPUOutput.cu:11-27 */
void maxamp_launch_(const int *lid) {
    gc_gauge_invalidate();
    GcLayer &L = layer_or_die(*lid);
    if (L.parent == -1 && g_rt.pend_momt && !g_rt.pend_maxamp) {
        g_rt.pend_maxamp = 1;
        return;
    }
    gc_flush();
    GcLayerDev d = L.view();
    if (!L.z2_valid) d.z2 = L.z[L.cur];
    gc_launch_maxamp(d, g_rt.stream);
    g_rt.launches++;
}

/* extension: the sponge layer of SPONGE_COEF / SPONGE_LAYER
 * (boundaries.f90:206-345), whose device path the reference lacks (it
 * applies it to host arrays the GPU run never reads back).  COEFX, COEFY are
 * the NX x NY fields SPONGE_COEF makes; COEFX must depend on I only and
 * COEFY on J only, as SPONGE_COEF's always do.  DT is the layer's time step.
 * Call after gcomcot_init_layer_. */
void gcomcot_set_sponge_(int *id, float *coefx, float *coefy, float *dt, int *nx, int *ny) {
    GcLayer &L = layer_or_die(*id);
    if (*nx != L.nx || *ny != L.ny || !coefx || !coefy) {
        fprintf(stderr, "gcomcot: sponge coefficients of layer %d must be %dx%d\n", L.id, L.nx, L.ny);
        exit(EXIT_FAILURE);
    }
    std::vector<float> vx((size_t)L.nx), vy((size_t)L.ny);
    for (int i = 0; i < L.nx; i++) vx[i] = coefx[i];
    for (int j = 0; j < L.ny; j++) vy[j] = coefy[(size_t)j * L.nx];
    for (int j = 0; j < L.ny; j++)
        for (int i = 0; i < L.nx; i++) {
            const size_t c = (size_t)j * L.nx + i;
            if (memcmp(&coefx[c], &vx[i], sizeof(float)) != 0 || memcmp(&coefy[c], &vy[j], sizeof(float)) != 0) {
                fprintf(stderr, "gcomcot: sponge coefficients of layer %d are not COEFX(I) x COEFY(J)\n", L.id);
                exit(EXIT_FAILURE);
            }
        }
    if (!L.spx) GC_CUDA_OR_DIE(cudaMalloc((void **)&L.spx, (size_t)L.nx * sizeof(float)));
    if (!L.spy) GC_CUDA_OR_DIE(cudaMalloc((void **)&L.spy, (size_t)L.ny * sizeof(float)));
    GC_CUDA_OR_DIE(cudaMemcpy(L.spx, vx.data(), vx.size() * sizeof(float), cudaMemcpyHostToDevice));
    GC_CUDA_OR_DIE(cudaMemcpy(L.spy, vy.data(), vy.size() * sizeof(float), cudaMemcpyHostToDevice));
    L.sp_dt = *dt;
}

/* extension: SPONGE_LAYER (boundaries.f90:206-247) on the device, called
 * where comcot.f90:403-406 calls it, after MOMT_LAUNCH */
void sponge_launch_(const int *lid) {
    gc_gauge_invalidate();
    GcLayer &L = layer_or_die(*lid);
    if (!L.spx || !L.spy) {
        fprintf(stderr, "gcomcot: layer %d has no sponge coefficients (gcomcot_set_sponge_)\n", L.id);
        exit(EXIT_FAILURE);
    }
    gc_flush();
    gc_launch_sponge(L.view(), L.spx, L.spy, L.sp_dt, g_rt.stream);
    g_rt.launches++;
}

/* GPUall_grids.cu:701-705: the nested sub-cycle of every child of layer 1 */
void all_grid_launch_(void) {
    gc_gauge_invalidate();
    gc_flush();
    if (g_rt.root >= 0) gc_subcycle(g_rt.root);
}

/* GPUcomcot.cu:144-155 (CHANGE for the outer layer) */
void cuda_update_layer_(int *lid) {
    gc_gauge_invalidate();
    GcLayer &L = layer_or_die(*lid);
    gc_flush();
    if (L.parent != -1) {
        gc_launch_update_edges(L.view(), g_rt.stream);
        g_rt.launches++;
    } else {
        gc_root_change_hook(L);
    }
    gc_swap(L);
}

/* GPUOutput.cu:29-44: the 2x2 surface stencil at 1-based (i,j) */
void gcomcot_get_z_(int *lid, float *l1, float *l2, float *l3, float *l4, int *i, int *j) {
    GcLayer &L = layer_or_die(*lid);
    if (*i < 1 || *j < 1 || *i >= L.nx || *j >= L.ny) {
        fprintf(stderr, "gcomcot: gauge (%d,%d) outside layer %d\n", *i, *j, *lid);
        exit(EXIT_FAILURE);
    }
    float tmp[4];
    if (!gc_gauge_lookup(*lid, *i, *j, tmp)) {
        fprintf(stderr, "gcomcot: gauge read failed\n");
        exit(EXIT_FAILURE);
    }
    *l1 = tmp[0]; *l2 = tmp[1]; *l3 = tmp[2]; *l4 = tmp[3];
}

/* GPUOutput.cu:55-102: whole-field transfers */
void cuda_getz1_(float *Z_f, int *lid) {
    GcLayer &L = layer_or_die(*lid); gc_flush();
    if (gc_layer_download_field(L, L.z[L.cur], Z_f) != GC_OK) exit(EXIT_FAILURE);
}
void cuda_setz1_(float *Z_f, int *lid) {
    gc_gauge_invalidate();
    GcLayer &L = layer_or_die(*lid); gc_flush();
    if (gc_layer_upload_field(L, L.z[L.cur], Z_f) != GC_OK) exit(EXIT_FAILURE);
}
void cuda_getz_(float *Z_f, int *lid) {
    GcLayer &L = layer_or_die(*lid); gc_flush();
    const float *z = L.z2_valid ? L.z[L.cur ^ 1] : L.z[L.cur];
    if (gc_layer_download_field(L, z, Z_f) != GC_OK) exit(EXIT_FAILURE);
}
void cuda_setz_(float *Z_f, int *lid) {
    gc_gauge_invalidate();
    GcLayer &L = layer_or_die(*lid); gc_flush();
    if (!L.z2_valid) {
        /* Z(:,:,2) equals Z(:,:,1) at this point: materialise it before the write */
        GC_CUDA_OR_DIE(cudaMemcpyAsync(L.z[L.cur ^ 1], L.z[L.cur], (size_t)L.pitch * L.ny * sizeof(float),
                                       cudaMemcpyDeviceToDevice, g_rt.stream));
    }
    if (gc_layer_upload_field(L, L.z[L.cur ^ 1], Z_f) != GC_OK) exit(EXIT_FAILURE);
    L.z2_valid = true;
}
void cuda_getmn1_(float *M_f, float *N_f, int *lid) {
    GcLayer &L = layer_or_die(*lid); gc_flush();
    if (gc_layer_download_field(L, L.m[L.cur], M_f) != GC_OK) exit(EXIT_FAILURE);
    if (gc_layer_download_field(L, L.n[L.cur], N_f) != GC_OK) exit(EXIT_FAILURE);
}
void cuda_setmn1_(float *M_f, float *N_f, int *lid) {
    gc_gauge_invalidate();
    GcLayer &L = layer_or_die(*lid); gc_flush();
    if (gc_layer_upload_field(L, L.m[L.cur], M_f) != GC_OK) exit(EXIT_FAILURE);
    if (gc_layer_upload_field(L, L.n[L.cur], N_f) != GC_OK) exit(EXIT_FAILURE);
}
void cuda_getmn_(float *M_f, float *N_f, int *lid) {
    GcLayer &L = layer_or_die(*lid); gc_flush();
    int b = L.mn2_valid ? (L.cur ^ 1) : L.cur;
    if (gc_layer_download_field(L, L.m[b], M_f) != GC_OK) exit(EXIT_FAILURE);
    if (gc_layer_download_field(L, L.n[b], N_f) != GC_OK) exit(EXIT_FAILURE);
}
void cuda_setmn_(float *M_f, float *N_f, int *lid) {
    gc_gauge_invalidate();
    GcLayer &L = layer_or_die(*lid); gc_flush();
    if (gc_layer_upload_field(L, L.m[L.cur ^ 1], M_f) != GC_OK) exit(EXIT_FAILURE);
    if (gc_layer_upload_field(L, L.n[L.cur ^ 1], N_f) != GC_OK) exit(EXIT_FAILURE);
    L.mn2_valid = true;
}
void cuda_getzmax_(float *Zmax_f, int *lid) {
    GcLayer &L = layer_or_die(*lid); gc_flush();
    if (gc_layer_download_field(L, L.zmax, Zmax_f) != GC_OK) exit(EXIT_FAILURE);
}

/* GPUall_grids.cu:26-30 */
static void show_rec(int id) {
    GcLayer &L = g_rt.layers[id];
    printf("lid = %d\n", L.id);
    printf("parent = %d\n", L.parent);
    printf("level = %d\n", L.level);
    printf("size = %d x %d\n", L.nx, L.ny);
    for (int c : L.children) show_rec(c);
}
void gcomcot_show_grids_(void) {
    if (g_rt.root >= 0) show_rec(g_rt.root);
}

/* GPUcomcot.cu:253-256 (empty in the reference): releases everything */
void cuda_shutdown_(void) {
    if (!g_rt.inited) return;
    cudaStreamSynchronize(g_rt.stream);
    for (int k = 0; k < GC_MAX_LAYERS; k++) {
        if (g_rt.layers[k].block) cudaFree(g_rt.layers[k].block);
        if (g_rt.layers[k].spx) cudaFree(g_rt.layers[k].spx);
        if (g_rt.layers[k].spy) cudaFree(g_rt.layers[k].spy);
        if (g_rt.layers[k].sc_block) cudaFree(g_rt.layers[k].sc_block);
        g_rt.layers[k] = GcLayer();
        g_rt.pending[k] = GcPendingParams();
    }
    gc_gauge_release();
    if (g_rt.d_gauge_ij) cudaFree(g_rt.d_gauge_ij);
    if (g_rt.d_gauge_out) cudaFree(g_rt.d_gauge_out);
    if (g_rt.h_gauge_out) cudaFreeHost(g_rt.h_gauge_out);
    g_rt.d_gauge_ij = nullptr; g_rt.d_gauge_out = nullptr; g_rt.h_gauge_out = nullptr;
    g_rt.gauge_cap = 0;
    cudaStreamDestroy(g_rt.stream);
    g_rt.stream = nullptr;
    g_rt.inited = false;
    g_rt.root = -1;
    g_rt.pend_mass = g_rt.pend_open = g_rt.pend_momt = g_rt.pend_maxamp = 0;
}

} /* extern "C" */

/* ------------------------------------------------------------------ */
/* nested sub-cycle (GPUall_grids.cu:655-699; Fortran ALL_GRID order,  */
/* all_grids.f90:34-306), dispatching each child by its equations      */
/* ------------------------------------------------------------------ */
void gc_subcycle(int parent_id) {
    GcLayer &P = g_rt.layers[parent_id];
    GcPdlScope pdl(true);
    for (int cid : P.children) {
        GcLayer &C = g_rt.layers[cid];
        int nhalf = C.rel_time / 2 + 1;
        for (int k = 1; k <= C.rel_time; k++) {
            /* edge fluxes and mass: one launch at a Cartesian child's first
             * sub-step (gc_launch_edges_mass), two otherwise */
            int pre = 2;
            if (C.has_sc) {
                /* EDGE_INTERP_SC / NEWQ_SC (all_grids.f90:996-1364) */
                const GcLayerDev cv = C.view();
                if (k > 1) { gc_launch_sc_forecast(P.view(), C.sc, g_rt.stream); g_rt.launches++; }
                gc_launch_sc_edges(P.view(), cv, C.sc, k, C.rel_time, C.sc_stepped ? cv.z1 : cv.z2, g_rt.stream);
                gc_launch_mass(C.view(), g_rt.stream);
            } else if (gc_launch_edges_mass(P.view(), C.view(), C.rel_size, C.rel_time, C.corners, k, g_rt.stream)) {
                pre = 1;
            } else {
                gc_launch_edges(P.view(), C.view(), C.rel_size, C.rel_time, C.corners, k, g_rt.stream);
                gc_launch_mass(C.view(), g_rt.stream);
            }
            C.z2_valid = true;
            gc_subcycle(cid);
            /* UPDATE's edge copy writes the child's row and column 0 alone,
             * which JNZ never reads (its blocks start at child index 1), so
             * it may precede JNZ; JNZ_SC sums every child node in the window,
             * so at its sub-step the copy follows it */
            const bool late_update = C.has_sc && k == nhalf;
            if (late_update) {
                gc_launch_moment(C.view(), g_rt.stream);
                g_rt.launches += pre + 1;
            } else {
                g_rt.launches += pre + gc_launch_moment_update(C.view(), g_rt.stream);
            }
            C.mn2_valid = true;
            if (k == nhalf) {
                if (C.has_sc) gc_launch_sc_jnz(P.view(), C.view(), C.sc, g_rt.stream);
                else gc_launch_jnz(P.view(), C.view(), C.rel_size, C.rel_time, C.corners, g_rt.stream);
                g_rt.launches++;
            }
            if (late_update) {
                gc_launch_update_edges(C.view(), g_rt.stream);
                g_rt.launches++;
            }
            gc_swap(C);
            C.sc_stepped = true;
        }
    }
}
