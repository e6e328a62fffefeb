/*
 * Batched ensemble / serving engine.
 *
 * Many independent linear-spherical forecasts ("members": ensemble scenarios
 * or served requests) are stepped by ONE fused launch per time step over a
 * work list of tiles drawn from every active member, whatever their grid
 * sizes.  Members of one grid class share the bathymetry and the per-row
 * coefficients.  Tiles are ordered tile-major / member-minor so the CTAs that
 * read one bathymetry tile run together and it is served from L2.
 *
 * Each member carries its own first step, step count, ping-pong parity,
 * gauges and arrival threshold; the kernel skips members outside their
 * window, so members may be admitted and retired between any two launches
 * (continuous batching).  Chunks of steps over an unchanged member set are
 * captured once as a CUDA graph and replayed; the step number comes from a
 * device counter the graph advances.
 *
 * Member storage is taken with the stream-ordered allocator, so admitting a
 * request never waits for work in flight.  Admission is bounded by an HBM
 * budget counted by this engine.
 *
 * Nested members (an outer linear-spherical grid with one child layer, the
 * ALL_GRID sub-cycle of all_grids.f90:4-312) step with the per-phase kernels
 * in the order of comcot.f90:359-439: mass, open, the child's rel_time
 * sub-steps (edge fluxes, mass, momentum, JNZ at the half step, UPDATE),
 * momentum, then the step's outputs.  Each nested member's chain runs on its
 * own forked stream, so the chains overlap one another and the fused launch
 * of the single-grid members; in a captured chunk the fork and join become
 * graph edges.  Their ping-pong parities are fixed when a chunk is captured,
 * so chunks hold an even number of steps and a replay starts at the parity
 * of the capture.
 */
#include <string.h>

#include <algorithm>
#include <vector>

#include "fused.h"
#include "gcomcot.h"

namespace {

struct EngClass {
    int nx, ny, pitch;
    float *d_h = nullptr, *d_rows = nullptr;
    void *block = nullptr; /* storage this class owns */
    size_t bytes = 0;
    /* nested class: the outer grid of class `parent_cls` plus one child layer */
    bool nested = false;
    int parent_cls = -1;
    int cnx = 0, cny = 0, cpitch = 0;
    int corners[4] = {0, 0, 0, 0};
    int rel_size = 1, rel_time = 1;
    int laycord = 1, laygov = 1, linchk = 1, modscm = 1, fric_switch = 1;
    float dt = 0, rx = 0, ry = 0, grx = 0, gry = 0, fric_coef = 0;
    float *d_ch = nullptr, *d_chp = nullptr, *d_chq = nullptr, *d_crows = nullptr;
    float *d_crows2 = nullptr; /* [ny][2] R0, R22 of a nonlinear spherical child */
    /* SC_OPTION = 1 child: position / weight tables */
    bool has_sc = false;
    GcScView sc{};
    void *sc_block = nullptr;
    /* longitude / latitude axes (degrees), for members made from faults */
    float *d_lon = nullptr, *d_lat = nullptr;
};

struct EngMember {
    bool used = false, done = false;
    int cls = 0, nsteps = 0, step0 = 0, ng = 0;
    float thr = -1.0f;
    void *block = nullptr;
    size_t bytes = 0;
    /* time levels: nested members ping-pong two buffers (level L in L & 1);
     * single-grid members keep three (level L in L % 3), so a two-step
     * launch writes level L + 2 to a buffer it does not read */
    int nbuf = 3;
    float *z[3] = {nullptr, nullptr, nullptr}, *m[3] = {nullptr, nullptr, nullptr}, *n[3] = {nullptr, nullptr, nullptr};
    float *zmax = nullptr, *ts = nullptr, *gw = nullptr;
    int *arrival = nullptr, *gij = nullptr;
    /* nested members: the child's levels, DZ, the outer grid's NEWQ caches */
    bool nested = false;
    float *cz[2] = {nullptr, nullptr}, *cm[2] = {nullptr, nullptr}, *cn[2] = {nullptr, nullptr};
    float *cdz2 = nullptr, *xflux = nullptr, *yflux = nullptr;
    int *glayer = nullptr;
    /* SC_OPTION = 1: the outer grid's band forecast of NEWQ_SC (the fused
     * step has written the outer grid's real level 2 by then) */
    float *sm2 = nullptr, *sn2 = nullptr;
    float *h = nullptr; /* own depth (members made from faults), else the class's */
    int fty = 16; /* tile height of the outer grid's fused launch */
    /* the last global step this member needs a launch at: single-grid
     * members sample their last gauges in the launch after their last step */
    int last_step() const { return nested ? step0 + nsteps - 1 : step0 + nsteps; }
    /* the buffer holding the level after `done` steps */
    int level_buf(int done) const { return nbuf == 3 ? done % 3 : (done & 1); }
};

size_t a256(size_t x) { return (x + 255) & ~(size_t)255; }

__global__ void k_advance(int *step, int by) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *step += by;
}

constexpr int kMaxAux = 8; /* forked streams for nested members */

/* health of one field: bit 0 = a NaN or Inf, bit 1 = |value| > bound */
__global__ void k_health(const float *a, int nx, int ny, int pitch, float bound, int *flag) {
    int bits = 0;
    const long long n = (long long)nx * ny;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(k / nx), i = (int)(k - (long long)j * nx);
        const float v = a[(size_t)j * pitch + i];
        if (!isfinite(v)) bits |= 1;
        else if (fabsf(v) > bound) bits |= 2;
    }
    bits = __reduce_or_sync(0xffffffffu, bits);
    if ((threadIdx.x & 31) == 0 && bits) atomicOr(flag, bits);
}

GcLayerDev outer_view(const EngClass &C, const EngMember &M, int cur) {
    GcLayerDev d;
    memset(&d, 0, sizeof d);
    d.nx = C.nx; d.ny = C.ny; d.pitch = C.pitch;
    d.root = 1; d.laycord = 0; d.laygov = 0; d.linchk = 1; d.modscm = 1; d.fric_switch = 1;
    d.z1 = M.z[cur]; d.m1 = M.m[cur]; d.n1 = M.n[cur];
    d.z1w = M.z[cur]; d.m1w = M.m[cur]; d.n1w = M.n[cur];
    d.z2 = M.z[cur ^ 1]; d.m2 = M.m[cur ^ 1]; d.n2 = M.n[cur ^ 1];
    d.h = C.d_h; d.rows = C.d_rows;
    d.xflux = M.xflux; d.yflux = M.yflux;
    d.zmax = M.zmax; d.arrival = M.arrival;
    return d;
}

GcLayerDev child_view(const EngClass &C, const EngMember &M, int cur) {
    GcLayerDev d;
    memset(&d, 0, sizeof d);
    d.nx = C.cnx; d.ny = C.cny; d.pitch = C.cpitch;
    d.root = 0; d.laycord = C.laycord; d.laygov = C.laygov; d.linchk = C.linchk; d.modscm = C.modscm;
    d.fric_switch = C.fric_switch;
    d.rx = C.rx; d.ry = C.ry; d.grx = C.grx; d.gry = C.gry; d.dt = C.dt; d.fric_coef = C.fric_coef;
    d.z1 = M.cz[cur]; d.m1 = M.cm[cur]; d.n1 = M.cn[cur];
    d.z1w = M.cz[cur]; d.m1w = M.cm[cur]; d.n1w = M.cn[cur];
    d.z2 = M.cz[cur ^ 1]; d.m2 = M.cm[cur ^ 1]; d.n2 = M.cn[cur ^ 1];
    d.h = C.d_ch; d.hp = C.d_chp; d.hq = C.d_chq; d.rows = C.d_crows; d.dz2 = M.cdz2;
    d.rows2 = C.d_crows2;
    return d;
}

} // namespace

struct gc_engine {
    long long budget = 0, in_use = 0;
    cudaStream_t stream = nullptr;
    std::vector<EngClass> classes;
    std::vector<EngMember> members;
    int variant = 16; /* until tuned: the fastest single-grid variant on B200 */
    bool tuned = false;
    int use_graphs = 1, chunk = 32;
    int gstep = 0; /* steps issued */
    GcFusedGrid *d_grids = nullptr;
    int grids_cap = 0, ngrids = 0;
    int2 *d_tiles = nullptr;
    int tiles_cap = 0, ntiles = 0;
    int *d_step = nullptr;
    bool dirty = true;
    cudaGraphExec_t gexec = nullptr;
    long long launches = 0;
    int nctas = 0;
    /* a work list of one grid launches the single-grid kernel with this
     * descriptor by value (no descriptor loads, fewer registers) */
    bool single = false;
    GcFusedGrid one_grid;
    long long chunk_launches = 0; /* kernels in one replay of the chunk graph */
    int pdl = 1;                  /* programmatic dependent launch (GCOMCOT_PDL=0 turns it off) */
    int ty_rule = 1;              /* tile-height rule (gc_fused_pick_ty), tuned with the variant */
    /* two steps per launch (kernels_pair.cu) for the single-grid members */
    int pair_on = 1;              /* the chosen candidate uses it */
    int pair_allowed = 1;         /* GCOMCOT_PAIR=0 turns it off altogether */
    /* until tuned: one warp x 5 stages in the balanced layout, the fastest
     * single-grid form on B200 */
    int pair_variant = 7, pair_rule = 2;
    bool pair_ok = false;         /* the current members allow it */
    int2 *d_ptiles = nullptr;
    int ptiles_cap = 0, nptiles = 0;
    /* the single-grid members form one grid class of at most
     * GC_PAIR_CLASS_MAX members: pairs go out as a class launch (member
     * table in the parameter bank) instead of over the work list */
    bool pair_class = false;
    bool pair_class_on = true; /* GCOMCOT_PAIR_CLASS=0: always the work list */
    GcPairClass pcls;
    int *d_health = nullptr;      /* one int for gc_engine_member_health */
    std::vector<int> nested_ids; /* active nested members */
    cudaStream_t aux[kMaxAux] = {};
    cudaEvent_t ev_fork = nullptr, ev_join[kMaxAux] = {};
    /* per aux stream, a second stream for the child's first sub-step, which
     * runs beside the outer grid's fused step */
    cudaStream_t caux[kMaxAux] = {};
    cudaEvent_t ev_cfork[kMaxAux] = {}, ev_cjoin[kMaxAux] = {};
};

/* One outer step of a nested member whose 0-based step index is `local`
 * (it fixes the ping-pong parities) and whose device step number is
 * step_off + *d_base.
 *
 * The outer grid takes its whole step (MASS_S + OPEN + MOMT_S) in one fused
 * launch before the child runs, and its momentum is then recomputed where
 * JNZ changed the surface.  That gives the bits of the reference order
 * (mass, open, child sub-cycle with JNZ, momentum): JNZ writes the outer
 * Z(:,:,2) only inside IS..IE x JS..JE (all_grids.f90:378-411); outer M at
 * (I,J) reads Z(I,J) and Z(I+1,J), N reads Z(I,J) and Z(I,J+1), and both
 * read otherwise only level-1 fields, which nothing in the sub-cycle
 * writes; so only M on [IS-1,IE] x [JS,JE] and N on [IS,IE] x [JS-1,JE] can
 * differ, and the rectangle [IS-1,IE] x [JS-1,JE] is recomputed.  The child
 * reads the outer Z(:,:,2), M(:,:,1) and N(:,:,1) only.  Max-eta, arrival
 * and gauges follow in the outputs kernel, after the feedback. */
/* GCOMCOT_FEEDBACK=0 keeps JNZ, the window's momentum and the outputs as
 * three launches */
static bool eng_feedback_on() {
    static const bool on = [] {
        const char *v = getenv("GCOMCOT_FEEDBACK");
        return !(v && v[0] == '0');
    }();
    return on;
}

static void eng_nested_step(gc_engine *e, EngMember &M, int local, const int *d_base, int step_off, int a) {
    cudaStream_t s = e->aux[a];
    const EngClass &C = e->classes[M.cls];
    const int cur = local & 1;
    GcFusedGrid g;
    memset(&g, 0, sizeof g);
    g.nx = C.nx; g.ny = C.ny; g.pitch = C.pitch; g.root = 1; g.explicit_r24 = 0;
    g.ty = M.fty;
    gc_fused_tiles(C.nx, C.ny, g.ty, &g.tiles_x);
    /* the fused launch records max-eta and arrival outside the JNZ window
     * (IS..IE x JS..JE, 0-based IS-1..IE-1); the outputs kernel does the window */
    const int win[4] = {C.corners[0] - 1, C.corners[1] - 1, C.corners[2] - 1, C.corners[3] - 1};
    const int flags = GC_F_MAXAMP | (M.thr >= 0.0f ? GC_F_ARRIVAL | GC_F_ARR_BYMAX : 0);
    /* the step number comes from the device counter (arrival steps); the
     * member's level-1 buffer is 0 at its first step, so the kernel's parity
     * equals `cur` */
    g.step0 = M.step0; g.cur0 = 0; g.nsteps = M.nsteps; g.flags = flags; g.thr = M.thr;
    g.has_win = 1; g.wi0 = win[0]; g.wi1 = win[1]; g.wj0 = win[2]; g.wj1 = win[3];
    for (int q = 0; q < 2; q++) { g.z[q] = M.z[q]; g.m[q] = M.m[q]; g.n[q] = M.n[q]; }
    g.h = C.d_h; g.rows = C.d_rows;
    g.zmax = M.zmax; g.arrival = M.arrival;
    const GcLayerDev P = outer_view(C, M, cur);
    int cc = (int)(((long long)local * C.rel_time) & 1);
    const int nhalf = C.rel_time / 2 + 1;
    /* the child's first sub-step (JNQ, its mass and momentum, UPDATE's edge
     * copy) reads the outer grid's level-1 fluxes only, which the fused step
     * does not write, and the fused step reads nothing of the child's: they
     * run side by side, joined before JNZ.  UPDATE writes the child's row and
     * column 0 alone, which JNZ never reads, so it may precede JNZ. */
    cudaStream_t cs = e->caux[a];
    const GcLayerDev Cv1 = child_view(C, M, cc);
    /* SC_OPTION = 1: NEWQ_SC's band forecast goes to the member's scratch
     * fields in place of the outer grid's level 2 */
    GcLayerDev Pf = P;
    if (C.has_sc) { Pf.m2 = M.sm2; Pf.n2 = M.sn2; }
    cudaEventRecord(e->ev_cfork[a], s);
    cudaStreamWaitEvent(cs, e->ev_cfork[a], 0);
    /* edge fluxes and mass: one launch for a Cartesian child (JNQ's values
     * computed where the mass reads them), two otherwise */
    int pre = 2;
    if (C.has_sc) {
        gc_launch_sc_edges(Pf, Cv1, C.sc, 1, C.rel_time, Cv1.z1, cs);
        gc_launch_mass(Cv1, cs);
    } else if (gc_launch_edges_mass(P, Cv1, C.rel_size, C.rel_time, C.corners, 1, cs)) {
        pre = 1;
    } else {
        gc_launch_edges(P, Cv1, C.rel_size, C.rel_time, C.corners, 1, cs);
        gc_launch_mass(Cv1, cs);
    }
    /* JNZ_SC sums every child node inside the parent window, row and column
     * 0 included, so in the sub-step that feeds back UPDATE's edge copy
     * follows it (all_grids.f90 order: MOMENT, JNZ, UPDATE) */
    const bool late_update1 = C.has_sc && nhalf == 1;
    if (late_update1) {
        gc_launch_moment(Cv1, cs);
        e->launches += pre + 1;
    } else {
        e->launches += pre + gc_launch_moment_update(Cv1, cs);
    }
    cudaEventRecord(e->ev_cjoin[a], cs);
    gc_fused_launch_one_at(e->variant, g, d_base, step_off, s);
    cudaStreamWaitEvent(s, e->ev_cjoin[a], 0);
    auto jnz = [&](const GcLayerDev &Cv) {
        if (C.has_sc) gc_launch_sc_jnz(P, Cv, C.sc, s);
        else gc_launch_jnz(P, Cv, C.rel_size, C.rel_time, C.corners, s);
        e->launches++;
    };
    /* one sub-step and a JNZ ratio the feedback launch is built for: JNZ,
     * the window's momentum and the outputs go out as one launch at the end */
    const bool fb = nhalf == 1 && !C.has_sc && C.rel_size >= 2 && C.rel_size <= 5 && eng_feedback_on();
    if (nhalf == 1 && !fb) jnz(Cv1);
    if (late_update1) {
        gc_launch_update_edges(Cv1, s);
        e->launches++;
    }
    cc ^= 1;
    for (int t = 2; t <= C.rel_time; t++) {
        const GcLayerDev Cv = child_view(C, M, cc);
        if (C.has_sc) {
            gc_launch_sc_forecast(Pf, C.sc, s);
            gc_launch_sc_edges(Pf, Cv, C.sc, t, C.rel_time, Cv.z1, s);
            e->launches++;
        } else {
            gc_launch_edges(P, Cv, C.rel_size, C.rel_time, C.corners, t, s);
        }
        gc_launch_mass(Cv, s);
        if (C.has_sc && t == nhalf) {
            gc_launch_moment(Cv, s);
            jnz(Cv);
            gc_launch_update_edges(Cv, s);
            e->launches += 4;
        } else {
            /* UPDATE's edge copy writes the child's row and column 0 alone,
             * which JNZ never reads (its blocks start at child index 1), so
             * it may precede JNZ */
            e->launches += 2 + gc_launch_moment_update(Cv, s);
            if (t == nhalf) jnz(Cv);
        }
        cc ^= 1;
    }
    /* the window's momentum (which the surface JNZ wrote changes) and its
     * max-eta / arrival / gauges, side by side; both read the final surface,
     * neither writes what the other reads.  Fortran (IS-1 .. IE, JS-1 .. JE)
     * -> 0-based (IS-2 .. IE-1, JS-2 .. JE-1) */
    if (fb) {
        const int rect[4] = {C.corners[0] - 2, C.corners[1] - 1, C.corners[2] - 2, C.corners[3] - 1};
        gc_launch_feedback(P, Cv1, C.rel_size, C.rel_time, C.corners, rect, d_base, step_off, M.step0, flags, M.thr,
                           M.ng, M.gij, M.gw, M.glayer, M.cz[cc], C.cpitch, M.ts, M.nsteps, s);
        e->launches += 2; /* the fused step, the feedback */
        return;
    }
    cudaEventRecord(e->ev_cfork[a], s);
    cudaStreamWaitEvent(cs, e->ev_cfork[a], 0);
    gc_launch_step_outputs(P, d_base, step_off, M.step0, flags, M.thr, M.ng, M.gij, M.gw, M.glayer, M.cz[cc],
                           C.cpitch, M.ts, M.nsteps, win, cs);
    cudaEventRecord(e->ev_cjoin[a], cs);
    gc_launch_momt_s_window(P, C.corners[0] - 2, C.corners[1] - 1, C.corners[2] - 2, C.corners[3] - 1, s);
    cudaStreamWaitEvent(s, e->ev_cjoin[a], 0);
    e->launches += 3; /* the fused step, the window's momentum, the outputs */
}

/* issues `count` consecutive steps, the first being host step e->gstep + 1
 * and device step step_off0 + *d_base: the fused launch over the single-grid
 * members on the engine stream, each nested member's chain on a forked
 * stream, joined back before return */
static cudaError_t eng_launch_steps_(gc_engine *e, const int *d_base, int step_off0, int count, int pair_room);

/* the engine's kernels go out with programmatic dependent launch: each one
 * is scheduled while its predecessor in the stream runs and waits for it on
 * the device, which hides the launch gap of a chain of short kernels */
static cudaError_t eng_launch_steps(gc_engine *e, const int *d_base, int step_off0, int count, int pair_room) {
    gc_set_pdl(e->pdl != 0);
    cudaError_t err = eng_launch_steps_(e, d_base, step_off0, count, pair_room);
    gc_set_pdl(false);
    return err;
}

/* pair_room: how many of the `count` steps may go two at a time (every
 * single-grid member computes both steps of a pair) */
static cudaError_t eng_launch_steps_(gc_engine *e, const int *d_base, int step_off0, int count, int pair_room) {
    const int nn = (int)e->nested_ids.size();
    const int naux = std::min(nn, kMaxAux);
    if (naux > 0) {
        cudaError_t err = cudaEventRecord(e->ev_fork, e->stream);
        if (err != cudaSuccess) return err;
        for (int a = 0; a < naux; a++) {
            err = cudaStreamWaitEvent(e->aux[a], e->ev_fork, 0);
            if (err != cudaSuccess) return err;
        }
    }
    if (e->ntiles > 0) {
        /* two steps per launch while both lie inside every member's window
         * (the launch after a member's last step only samples its gauges) */
        int k = 0;
        if (e->pair_ok)
            for (; k + 1 < count && k + 2 <= pair_room; k += 2) {
                cudaError_t err = e->single
                                      ? gc_pair_launch_one_at(e->pair_variant, e->one_grid, d_base, step_off0 + k,
                                                              e->stream)
                                  : e->pair_class
                                      ? gc_pair_launch_class(e->pair_variant, e->pcls, d_base, step_off0 + k, e->stream)
                                      : gc_pair_launch_multi(e->pair_variant, e->d_grids, e->d_ptiles, e->nptiles,
                                                             d_base, step_off0 + k, e->stream);
                if (err != cudaSuccess) return err;
                e->launches++;
            }
        for (; k < count; k++) {
            cudaError_t err = e->single ? gc_fused_launch_one_at(e->variant, e->one_grid, d_base, step_off0 + k, e->stream)
                                        : gc_fused_launch_multi(e->variant, e->d_grids, e->d_tiles, e->ntiles, d_base,
                                                                step_off0 + k, e->nctas, e->stream);
            if (err != cudaSuccess) return err;
            e->launches++;
        }
    }
    for (int q = 0; q < nn; q++) {
        EngMember &M = e->members[e->nested_ids[q]];
        for (int k = 0; k < count; k++)
            eng_nested_step(e, M, e->gstep + 1 + k - M.step0, d_base, step_off0 + k, q % naux);
    }
    if (naux > 0) {
        for (int a = 0; a < naux; a++) {
            cudaError_t err = cudaEventRecord(e->ev_join[a], e->aux[a]);
            if (err != cudaSuccess) return err;
            err = cudaStreamWaitEvent(e->stream, e->ev_join[a], 0);
            if (err != cudaSuccess) return err;
        }
    }
    return cudaGetLastError();
}

/* forked streams and their events for up to kMaxAux nested chains; made
 * here, outside any stream capture */
static int eng_make_aux(gc_engine *e, int naux) {
    if (naux > 0 && !e->ev_fork) GC_CUDA_OR_RET(cudaEventCreateWithFlags(&e->ev_fork, cudaEventDisableTiming));
    for (int a = 0; a < naux && a < kMaxAux; a++) {
        if (e->aux[a]) continue;
        GC_CUDA_OR_RET(cudaStreamCreateWithFlags(&e->aux[a], cudaStreamNonBlocking));
        GC_CUDA_OR_RET(cudaEventCreateWithFlags(&e->ev_join[a], cudaEventDisableTiming));
        GC_CUDA_OR_RET(cudaStreamCreateWithFlags(&e->caux[a], cudaStreamNonBlocking));
        GC_CUDA_OR_RET(cudaEventCreateWithFlags(&e->ev_cfork[a], cudaEventDisableTiming));
        GC_CUDA_OR_RET(cudaEventCreateWithFlags(&e->ev_cjoin[a], cudaEventDisableTiming));
    }
    return GC_OK;
}

static int eng_rebuild(gc_engine *e) {
    std::vector<GcFusedGrid> grids;
    std::vector<int2> tiles;
    /* one tile height for the whole work list, chosen to fill whole waves */
    std::vector<int> anx, any;
    e->nested_ids.clear();
    for (size_t k = 0; k < e->members.size(); k++) {
        EngMember &M = e->members[k];
        if (!M.used || M.done) continue;
        if (M.nested) { e->nested_ids.push_back((int)k); continue; }
        anx.push_back(e->classes[M.cls].nx);
        any.push_back(e->classes[M.cls].ny);
    }
    const bool single = anx.size() == 1;
    const int ty = anx.empty() ? 16 : gc_fused_pick_ty(e->variant, (int)anx.size(), anx.data(), any.data(),
                                                       e->ty_rule, !single);
    const int pty = anx.empty() ? 32 : gc_pair_pick_ty(e->pair_variant, (int)anx.size(), anx.data(), any.data(),
                                                       e->pair_rule, !single);
    const int pte = gc_pair_short_ty(e->pair_rule, pty);
    /* two-step launches need at most 64 gauges per member */
    bool pair_ok = e->pair_on != 0 && e->pair_allowed != 0 && !anx.empty();
    std::vector<int2> ptiles;
    /* active members grouped by class */
    for (size_t c = 0; c < e->classes.size(); c++) {
        EngClass &C = e->classes[c];
        std::vector<int> idx;
        for (size_t k = 0; k < e->members.size(); k++) {
            EngMember &M = e->members[k];
            if (!M.used || M.done || M.nested || M.cls != (int)c) continue;
            idx.push_back((int)grids.size());
            GcFusedGrid g;
            memset(&g, 0, sizeof g);
            g.nx = C.nx; g.ny = C.ny; g.pitch = C.pitch; g.root = 1; g.explicit_r24 = 0;
            g.ty = ty;
            gc_fused_tiles(C.nx, C.ny, ty, &g.tiles_x);
            g.step0 = M.step0; g.cur0 = 0; g.nsteps = M.nsteps;
            g.flags = GC_F_MAXAMP | (M.thr >= 0.0f ? GC_F_ARRIVAL | GC_F_ARR_BYMAX : 0);
            g.thr = M.thr;
            g.nbuf = 3;
            g.pty = pty;
            g.pte = pte;
            gc_pair_tiles(C.nx, C.ny, pty, pte, &g.ptiles_x);
            for (int q = 0; q < 3; q++) { g.z[q] = M.z[q]; g.m[q] = M.m[q]; g.n[q] = M.n[q]; }
            g.h = M.h ? M.h : C.d_h; g.rows = C.d_rows;
            g.zmax = M.zmax; g.arrival = M.arrival;
            g.ng = M.ng; g.gij = M.gij; g.gw = M.gw; g.ts = M.ts; g.ts_len = M.nsteps;
            grids.push_back(g);
        }
        if (idx.empty()) continue;
        int nt = gc_fused_tiles(C.nx, C.ny, ty, nullptr);
        for (int t = 0; t < nt; t++)
            for (int g : idx) tiles.push_back(make_int2(g, t));
        const int npt = gc_pair_tiles(C.nx, C.ny, pty, pte, nullptr);
        for (int t = 0; t < npt; t++)
            for (int g : idx) ptiles.push_back(make_int2(g, t));
        for (int g : idx)
            if (grids[g].ng > 64) pair_ok = false;
    }
    if (eng_make_aux(e, (int)e->nested_ids.size()) != GC_OK) return GC_ECUDA;
    /* the outer grid of a nested member is stepped alone on its own stream */
    for (int id : e->nested_ids) {
        EngMember &M = e->members[id];
        M.fty = gc_fused_pick_ty(e->variant, 1, &e->classes[M.cls].nx, &e->classes[M.cls].ny, 1, false);
    }
    e->ngrids = (int)grids.size();
    e->ntiles = (int)tiles.size();
    e->single = single && e->ngrids == 1;
    if (e->single) e->one_grid = grids[0];
    if (e->ngrids > e->grids_cap) {
        if (e->d_grids) cudaFreeAsync(e->d_grids, e->stream);
        e->grids_cap = std::max(e->ngrids, 2 * e->grids_cap);
        GC_CUDA_OR_RET(cudaMallocAsync((void **)&e->d_grids, (size_t)e->grids_cap * sizeof(GcFusedGrid), e->stream));
    }
    if (e->ntiles > e->tiles_cap) {
        if (e->d_tiles) cudaFreeAsync(e->d_tiles, e->stream);
        e->tiles_cap = std::max(e->ntiles, 2 * e->tiles_cap);
        GC_CUDA_OR_RET(cudaMallocAsync((void **)&e->d_tiles, (size_t)e->tiles_cap * sizeof(int2), e->stream));
    }
    if (e->ngrids)
        GC_CUDA_OR_RET(cudaMemcpyAsync(e->d_grids, grids.data(), grids.size() * sizeof(GcFusedGrid),
                                       cudaMemcpyHostToDevice, e->stream));
    if (e->ntiles)
        GC_CUDA_OR_RET(cudaMemcpyAsync(e->d_tiles, tiles.data(), tiles.size() * sizeof(int2),
                                       cudaMemcpyHostToDevice, e->stream));
    e->nptiles = (int)ptiles.size();
    if (e->nptiles > e->ptiles_cap) {
        if (e->d_ptiles) cudaFreeAsync(e->d_ptiles, e->stream);
        e->ptiles_cap = std::max(e->nptiles, 2 * e->ptiles_cap);
        GC_CUDA_OR_RET(cudaMallocAsync((void **)&e->d_ptiles, (size_t)e->ptiles_cap * sizeof(int2), e->stream));
    }
    if (e->nptiles)
        GC_CUDA_OR_RET(cudaMemcpyAsync(e->d_ptiles, ptiles.data(), ptiles.size() * sizeof(int2),
                                       cudaMemcpyHostToDevice, e->stream));
    e->pair_ok = pair_ok;
    /* one class of single-grid members: the class launch */
    e->pair_class = false;
    if (pair_ok && !e->single && e->ngrids >= 2 && e->ngrids <= GC_PAIR_CLASS_MAX && e->pair_class_on) {
        bool same = true;
        for (int g = 1; g < e->ngrids && same; g++)
            same = grids[g].nx == grids[0].nx && grids[g].ny == grids[0].ny && grids[g].pitch == grids[0].pitch &&
                   grids[g].rows == grids[0].rows;
        if (same) {
            memset(&e->pcls, 0, sizeof e->pcls);
            e->pcls.proto = grids[0];
            e->pcls.nm = e->ngrids;
            e->pcls.ntiles = gc_pair_tiles(grids[0].nx, grids[0].ny, pty, pte, nullptr);
            for (int g = 0; g < e->ngrids; g++) {
                const GcFusedGrid &G = grids[g];
                GcPairMember &q = e->pcls.m[g];
                for (int l = 0; l < 3; l++) { q.z[l] = G.z[l]; q.m[l] = G.m[l]; q.n[l] = G.n[l]; }
                q.zmax = G.zmax; q.arrival = G.arrival; q.h = G.h;
                q.gij = G.gij; q.gw = G.gw; q.ts = G.ts;
                q.step0 = G.step0; q.nsteps = G.nsteps; q.flags = G.flags; q.ng = G.ng; q.ts_len = G.ts_len;
                q.thr = G.thr;
            }
            e->pair_class = true;
        }
    }
    /* the host copies above are from pageable memory and complete before return */
    e->nctas = e->ntiles;
    if (e->gexec) { cudaGraphExecDestroy(e->gexec); e->gexec = nullptr; }
    e->dirty = false;
    return GC_OK;
}

/* retire members whose last gauge sample has been issued */
static void eng_retire(gc_engine *e) {
    for (auto &M : e->members)
        if (M.used && !M.done && e->gstep >= M.last_step()) {
            M.done = true;
            e->dirty = true;
        }
}

/* captures and uploads the graph of one chunk of steps for the current work
 * list */
static cudaError_t eng_build_graph(gc_engine *e) {
    cudaGraph_t graph;
    long long before = e->launches;
    cudaError_t err = cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal);
    if (err != cudaSuccess) return err;
    cudaError_t lerr = eng_launch_steps(e, e->d_step, 1, e->chunk, e->chunk);
    if (lerr == cudaSuccess) k_advance<<<1, 32, 0, e->stream>>>(e->d_step, e->chunk);
    cudaError_t cerr = cudaStreamEndCapture(e->stream, &graph);
    e->chunk_launches = e->launches - before + 1; /* + k_advance */
    e->launches = before;
    if (lerr != cudaSuccess) return lerr;
    if (cerr != cudaSuccess) return cerr;
    err = cudaGraphInstantiate(&e->gexec, graph, 0);
    cudaGraphDestroy(graph);
    if (err != cudaSuccess) return err;
    return cudaGraphUpload(e->gexec, e->stream);
}

static int eng_issue(gc_engine *e, int nsteps) {
    int issued = 0;
    while (issued < nsteps) {
        eng_retire(e);
        if (e->dirty && eng_rebuild(e) != GC_OK) return GC_ECUDA;
        if (e->ntiles == 0 && e->nested_ids.empty()) break;
        /* steps until the next member finishes: the member set is constant */
        int horizon = nsteps - issued;
        /* steps that every single-grid member computes (not only samples) */
        int room = horizon;
        for (auto &M : e->members)
            if (M.used && !M.done) {
                horizon = std::min(horizon, M.last_step() - e->gstep);
                if (!M.nested) room = std::min(room, M.step0 + M.nsteps - 1 - e->gstep);
            }
        if (horizon <= 0) horizon = 1;
        if (room < 0) room = 0;
        if (e->use_graphs && horizon >= e->chunk && (!e->pair_ok || room >= e->chunk)) {
            /* the device counter must equal the host's step count */
            GC_CUDA_OR_RET(cudaMemcpyAsync(e->d_step, &e->gstep, sizeof(int), cudaMemcpyHostToDevice, e->stream));
            if (!e->gexec) GC_CUDA_OR_RET(eng_build_graph(e));
            int reps = (e->pair_ok ? std::min(horizon, room) : horizon) / e->chunk;
            if (reps * e->chunk > nsteps - issued) reps = (nsteps - issued) / e->chunk;
            if (reps <= 0) reps = 0;
            for (int r = 0; r < reps; r++) {
                GC_CUDA_OR_RET(cudaGraphLaunch(e->gexec, e->stream));
                e->launches += e->chunk_launches;
            }
            e->gstep += reps * e->chunk;
            issued += reps * e->chunk;
            if (reps > 0) continue;
        }
        int n = std::min(horizon, nsteps - issued);
        if (eng_launch_steps(e, nullptr, e->gstep + 1, n, room) != cudaSuccess) return GC_ECUDA;
        e->gstep += n;
        issued += n;
    }
    eng_retire(e);
    return issued;
}

extern "C" {

int gc_engine_create(long long hbm_budget_bytes, gc_engine **out) {
    if (!out) return GC_EINVAL;
    gc_engine *e = new gc_engine();
    e->budget = hbm_budget_bytes;
    if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete e;
        return GC_ECUDA;
    }
    cudaMemPool_t pool;
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t thr = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    if (cudaMallocAsync((void **)&e->d_step, sizeof(int), e->stream) != cudaSuccess) {
        cudaStreamDestroy(e->stream);
        delete e;
        return GC_ECUDA;
    }
    const char *v = getenv("GCOMCOT_FUSED_VARIANT");
    if (v) { e->variant = atoi(v); e->tuned = true; }
    const char *pd = getenv("GCOMCOT_PDL");
    if (pd && pd[0] == '0') e->pdl = 0;
    const char *pr = getenv("GCOMCOT_PAIR");
    if (pr && pr[0] == '0') e->pair_on = e->pair_allowed = 0;
    const char *pc = getenv("GCOMCOT_PAIR_CLASS");
    if (pc && pc[0] == '0') e->pair_class_on = false;
    *out = e;
    return GC_OK;
}

int gc_engine_destroy(gc_engine *e) {
    if (!e) return GC_EINVAL;
    cudaStreamSynchronize(e->stream);
    if (e->gexec) cudaGraphExecDestroy(e->gexec);
    for (auto &M : e->members)
        if (M.block) cudaFreeAsync(M.block, e->stream);
    for (auto &C : e->classes) {
        if (C.block) cudaFreeAsync(C.block, e->stream);
        if (C.sc_block) cudaFree(C.sc_block);
        if (C.d_lon) cudaFreeAsync(C.d_lon, e->stream);
    }
    if (e->d_grids) cudaFreeAsync(e->d_grids, e->stream);
    if (e->d_tiles) cudaFreeAsync(e->d_tiles, e->stream);
    if (e->d_ptiles) cudaFreeAsync(e->d_ptiles, e->stream);
    if (e->d_step) cudaFreeAsync(e->d_step, e->stream);
    if (e->d_health) cudaFreeAsync(e->d_health, e->stream);
    cudaStreamSynchronize(e->stream);
    for (int a = 0; a < kMaxAux; a++) {
        if (e->aux[a]) cudaStreamDestroy(e->aux[a]);
        if (e->ev_join[a]) cudaEventDestroy(e->ev_join[a]);
        if (e->caux[a]) cudaStreamDestroy(e->caux[a]);
        if (e->ev_cfork[a]) cudaEventDestroy(e->ev_cfork[a]);
        if (e->ev_cjoin[a]) cudaEventDestroy(e->ev_cjoin[a]);
    }
    if (e->ev_fork) cudaEventDestroy(e->ev_fork);
    cudaStreamDestroy(e->stream);
    delete e;
    return GC_OK;
}

int gc_engine_add_class(gc_engine *e, int nx, int ny, const float *H, const float *rows) {
    if (!e || nx < 3 || ny < 3 || !H || !rows) return GC_EINVAL;
    EngClass C;
    C.nx = nx; C.ny = ny; C.pitch = (nx + 31) & ~31;
    size_t field = a256((size_t)C.pitch * ny * sizeof(float));
    size_t rb = a256((size_t)GC_ROWW * ny * sizeof(float));
    C.bytes = field + rb;
    if (e->in_use + (long long)C.bytes > e->budget) return GC_ENOMEM;
    void *blk = nullptr;
    GC_CUDA_OR_RET(cudaMallocAsync(&blk, C.bytes, e->stream));
    C.block = blk;
    C.d_h = (float *)blk;
    C.d_rows = (float *)((char *)blk + field);
    GC_CUDA_OR_RET(cudaMemcpy2DAsync(C.d_h, (size_t)C.pitch * sizeof(float), H, (size_t)nx * sizeof(float),
                                     (size_t)nx * sizeof(float), (size_t)ny, cudaMemcpyHostToDevice, e->stream));
    /* caller's [7][ny] blocks -> the device's interleaved [ny][8] records */
    std::vector<float> rec((size_t)GC_ROWW * ny, 0.0f);
    for (int k = 0; k < GC_NROW; k++)
        for (int j = 0; j < ny; j++) rec[(size_t)j * GC_ROWW + k] = rows[(size_t)k * ny + j];
    GC_CUDA_OR_RET(cudaMemcpyAsync(C.d_rows, rec.data(), rec.size() * sizeof(float), cudaMemcpyHostToDevice,
                                   e->stream));
    e->in_use += (long long)C.bytes;
    e->classes.push_back(C);
    return (int)e->classes.size() - 1;
}

} /* extern "C" */

static size_t eng_member_bytes(const EngClass &C, int nsteps, int ngauges, bool own_h = false) {
    size_t field = a256((size_t)C.pitch * C.ny * sizeof(float));
    size_t tsb = a256((size_t)nsteps * ngauges * sizeof(float));
    size_t gb = a256((size_t)2 * ngauges * sizeof(int)) + a256((size_t)2 * ngauges * sizeof(float));
    /* single-grid members: three levels of Z, M, N; nested: two */
    size_t bytes = ((C.nested ? 8 : 11) + (own_h ? 1 : 0)) * field + tsb + gb;
    if (C.nested) {
        size_t cfield = a256((size_t)C.cpitch * C.cny * sizeof(float));
        bytes += 7 * cfield + a256((size_t)2 * C.nx * sizeof(float)) + a256((size_t)2 * C.ny * sizeof(float))
                 + a256((size_t)ngauges * sizeof(int));
        if (C.has_sc) bytes += 2 * field;
    }
    return bytes;
}

static int eng_add_member(gc_engine *e, int cls, const float *z0, const float *cz0, int nsteps, int ngauges,
                          const int *glayer, const int *gij, const float *gw, float arrival_thr,
                          const gc_fault *faults = nullptr, int nfaults = 0) {
    if (!e || cls < 0 || cls >= (int)e->classes.size() || (!z0 && !faults) || nsteps < 1 || ngauges < 0)
        return GC_EINVAL;
    if (ngauges > 0 && (!gij || !gw)) return GC_EINVAL;
    EngClass &C = e->classes[cls];
    for (int g = 0; g < ngauges; g++) {
        const bool child = glayer && glayer[g] != 0;
        if (child && !C.nested) return GC_EINVAL;
        if (glayer && (glayer[g] < 0 || glayer[g] > 1)) return GC_EINVAL;
        const int nx = child ? C.cnx : C.nx, ny = child ? C.cny : C.ny;
        if (gij[2 * g] < 1 || gij[2 * g + 1] < 1 || gij[2 * g] >= nx || gij[2 * g + 1] >= ny) return GC_EINVAL;
    }
    size_t field = a256((size_t)C.pitch * C.ny * sizeof(float));
    size_t tsb = a256((size_t)nsteps * ngauges * sizeof(float));
    const bool own_h = faults != nullptr;
    if (own_h && (C.nested || !C.d_lon || nfaults < 1)) return C.nested ? GC_ENOTSUP : GC_EINVAL;
    size_t bytes = eng_member_bytes(C, nsteps, ngauges, own_h);
    if (e->in_use + (long long)bytes > e->budget) return GC_ENOMEM;
    EngMember M;
    M.used = true;
    M.cls = cls; M.nsteps = nsteps; M.ng = ngauges; M.thr = arrival_thr;
    M.step0 = e->gstep + 1;
    M.bytes = bytes;
    M.nested = C.nested;
    GC_CUDA_OR_RET(cudaMallocAsync(&M.block, bytes, e->stream));
    char *p = (char *)M.block;
    M.nbuf = C.nested ? 2 : 3;
    for (int q = 0; q < M.nbuf; q++) {
        M.z[q] = (float *)p; p += field;
        M.m[q] = (float *)p; p += field;
        M.n[q] = (float *)p; p += field;
    }
    M.zmax = (float *)p; p += field;
    M.arrival = (int *)p; p += field;
    M.ts = (float *)p; p += tsb;
    M.gij = (int *)p; p += a256((size_t)2 * ngauges * sizeof(int));
    M.gw = (float *)p; p += a256((size_t)2 * ngauges * sizeof(float));
    GC_CUDA_OR_RET(cudaMemsetAsync(M.block, 0, (size_t)3 * M.nbuf * field, e->stream));
    GC_CUDA_OR_RET(cudaMemsetAsync(M.arrival, 0xff, field, e->stream));
    if (own_h) {
        /* still water, then the faults' deformation on Z and on the member's own H */
        M.h = (float *)p;
        p += field;
        GC_CUDA_OR_RET(cudaMemcpyAsync(M.h, C.d_h, field, cudaMemcpyDeviceToDevice, e->stream));
        int rc = gc_okada_apply(faults, nfaults, 0, C.nx, C.ny, C.pitch, C.d_lon, C.d_lat, 0.0f, 0.0f, M.z[0], M.h,
                                e->stream);
        if (rc != GC_OK) {
            cudaFreeAsync(M.block, e->stream);
            return rc;
        }
    } else {
        GC_CUDA_OR_RET(cudaMemcpy2DAsync(M.z[0], (size_t)C.pitch * sizeof(float), z0, (size_t)C.nx * sizeof(float),
                                         (size_t)C.nx * sizeof(float), (size_t)C.ny, cudaMemcpyHostToDevice,
                                         e->stream));
    }
    GC_CUDA_OR_RET(cudaMemcpyAsync(M.zmax, M.z[0], field, cudaMemcpyDeviceToDevice, e->stream));
    if (arrival_thr >= 0.0f) {
        gc_launch_arrival_start(M.arrival, M.z[0], M.h ? M.h : C.d_h, C.nx, C.ny, C.pitch, arrival_thr, e->stream);
        GC_CUDA_OR_RET(cudaGetLastError());
    }
    if (ngauges > 0) {
        GC_CUDA_OR_RET(cudaMemcpyAsync(M.gij, gij, (size_t)2 * ngauges * sizeof(int), cudaMemcpyHostToDevice,
                                       e->stream));
        GC_CUDA_OR_RET(cudaMemcpyAsync(M.gw, gw, (size_t)2 * ngauges * sizeof(float), cudaMemcpyHostToDevice,
                                       e->stream));
    }
    if (C.nested) {
        size_t cfield = a256((size_t)C.cpitch * C.cny * sizeof(float));
        char *c0 = p;
        for (int q = 0; q < 2; q++) {
            M.cz[q] = (float *)p; p += cfield;
            M.cm[q] = (float *)p; p += cfield;
            M.cn[q] = (float *)p; p += cfield;
        }
        M.cdz2 = (float *)p; p += cfield;
        M.xflux = (float *)p; p += a256((size_t)2 * C.nx * sizeof(float));
        M.yflux = (float *)p; p += a256((size_t)2 * C.ny * sizeof(float));
        M.glayer = (int *)p;
        p += a256((size_t)ngauges * sizeof(int));
        if (C.has_sc) {
            M.sm2 = (float *)p; p += field;
            M.sn2 = (float *)p; p += field;
        }
        GC_CUDA_OR_RET(cudaMemsetAsync(c0, 0, (size_t)(p - c0), e->stream));
        if (cz0)
            GC_CUDA_OR_RET(cudaMemcpy2DAsync(M.cz[0], (size_t)C.cpitch * sizeof(float), cz0,
                                             (size_t)C.cnx * sizeof(float), (size_t)C.cnx * sizeof(float),
                                             (size_t)C.cny, cudaMemcpyHostToDevice, e->stream));
        if (ngauges > 0) {
            std::vector<int> gl((size_t)ngauges, 0);
            if (glayer)
                for (int g = 0; g < ngauges; g++) gl[g] = glayer[g];
            GC_CUDA_OR_RET(cudaMemcpyAsync(M.glayer, gl.data(), gl.size() * sizeof(int), cudaMemcpyHostToDevice,
                                           e->stream));
            /* the pageable copy is staged before return, but keep `gl` alive until it ran */
            GC_CUDA_OR_RET(cudaStreamSynchronize(e->stream));
        }
    }
    e->in_use += (long long)bytes;
    /* reuse a released slot id when there is one */
    int id = -1;
    for (size_t k = 0; k < e->members.size(); k++)
        if (!e->members[k].used) { id = (int)k; break; }
    if (id < 0) { e->members.push_back(M); id = (int)e->members.size() - 1; }
    else e->members[id] = M;
    e->dirty = true;
    return id;
}

extern "C" {

long long gc_engine_member_bytes(gc_engine *e, int cls) {
    if (!e || cls < 0 || cls >= (int)e->classes.size()) return GC_EINVAL;
    return (long long)eng_member_bytes(e->classes[cls], 0, 0);
}

int gc_engine_add_member(gc_engine *e, int cls, const float *z0, int nsteps, int ngauges, const int *gij,
                         const float *gw, float arrival_thr) {
    return eng_add_member(e, cls, z0, nullptr, nsteps, ngauges, nullptr, gij, gw, arrival_thr);
}

int gc_engine_add_nested_member(gc_engine *e, int cls, const float *z0, const float *child_z0, int nsteps,
                                int ngauges, const int *glayer, const int *gij, const float *gw,
                                float arrival_thr) {
    if (e && cls >= 0 && cls < (int)e->classes.size() && e->classes[cls].has_sc && child_z0) {
        /* at its first sub-step the reference's SC edges test wetness on the
         * child's level 2, which is still zero (all_grids.f90:1029); the
         * engine tests level 1, the same once both levels are equal */
        const EngClass &C = e->classes[cls];
        for (size_t c = 0; c < (size_t)C.cnx * C.cny; c++)
            if (child_z0[c] != 0.0f) return GC_ENOTSUP;
    }
    return eng_add_member(e, cls, z0, child_z0, nsteps, ngauges, glayer, gij, gw, arrival_thr);
}

int gc_engine_set_class_axes(gc_engine *e, int cls, const float *lon, const float *lat) {
    if (!e || cls < 0 || cls >= (int)e->classes.size() || !lon || !lat) return GC_EINVAL;
    EngClass &C = e->classes[cls];
    if (C.nested) return GC_ENOTSUP;
    if (!C.d_lon) {
        const size_t bytes = a256((size_t)C.nx * sizeof(float)) + a256((size_t)C.ny * sizeof(float));
        if (e->in_use + (long long)bytes > e->budget) return GC_ENOMEM;
        GC_CUDA_OR_RET(cudaMallocAsync((void **)&C.d_lon, bytes, e->stream));
        C.d_lat = (float *)((char *)C.d_lon + a256((size_t)C.nx * sizeof(float)));
        e->in_use += (long long)bytes;
        C.bytes += bytes;
    }
    GC_CUDA_OR_RET(cudaMemcpyAsync(C.d_lon, lon, (size_t)C.nx * sizeof(float), cudaMemcpyHostToDevice, e->stream));
    GC_CUDA_OR_RET(cudaMemcpyAsync(C.d_lat, lat, (size_t)C.ny * sizeof(float), cudaMemcpyHostToDevice, e->stream));
    GC_CUDA_OR_RET(cudaStreamSynchronize(e->stream));
    return GC_OK;
}

int gc_engine_add_member_faults(gc_engine *e, int cls, const gc_fault *faults, int nfaults, int nsteps, int ngauges,
                                const int *gij, const float *gw, float arrival_thr) {
    if (!faults || nfaults < 1) return GC_EINVAL;
    return eng_add_member(e, cls, nullptr, nullptr, nsteps, ngauges, nullptr, gij, gw, arrival_thr, faults, nfaults);
}

int gc_engine_add_nested_class(gc_engine *e, int parent_cls, const gc_child_desc *d) {
    if (!e || !d || parent_cls < 0 || parent_cls >= (int)e->classes.size()) return GC_EINVAL;
    const EngClass &Pc = e->classes[parent_cls];
    if (Pc.nested || !d->h) return GC_EINVAL;
    const int is = d->corners[0], ie = d->corners[1], js = d->corners[2], je = d->corners[3];
    /* the NEWQ forecast reads outer rows JS-3 and columns IS-3
     * (all_grids.f90:692-700,765-772), and the edge fluxes reach IE+2 / JE+2 */
    const bool sc = d->sc_pos != nullptr;
    if (sc && (!d->sc_cxy || d->laycord != 1)) return GC_EINVAL;
    /* an SC_OPTION = 1 child keeps its window's size; its corners are the extent of POS */
    const bool sized = sc || (d->nx == (ie - is + 1) * d->rel_size + 1 && d->ny == (je - js + 1) * d->rel_size + 1);
    if (d->rel_size < 1 || d->rel_time < 1 || is < 4 || js < 4 || ie > Pc.nx - 2 || je > Pc.ny - 2 || ie < is
        || je < js || !sized || d->nx < 3 || d->ny < 3)
        return GC_EINVAL;
    if ((d->laycord != 0 && d->laycord != 1) || d->laygov < 0 || d->laygov > 3) return GC_EINVAL;
    /* spherical children need their row coefficients; LAYGOV 3 on a
     * spherical layer carries R2 / R4 without the depth factor, which only
     * the reference-ABI path (full R2 / R4 fields) runs */
    if (d->laycord == 0 && (!d->rows || d->laygov == 3 || (d->laygov == 1 && !d->rows2))) return GC_ENOTSUP;
    if (d->fric_switch != 0 && d->fric_switch != 1) return GC_EINVAL;
    EngClass C = Pc;
    C.block = nullptr;
    C.nested = true;
    C.parent_cls = parent_cls;
    C.cnx = d->nx; C.cny = d->ny; C.cpitch = (d->nx + 31) & ~31;
    memcpy(C.corners, d->corners, sizeof C.corners);
    C.rel_size = d->rel_size; C.rel_time = d->rel_time;
    C.laycord = d->laycord; C.laygov = d->laygov; C.linchk = d->linchk; C.modscm = d->modscm;
    C.fric_switch = d->fric_switch;
    C.dt = d->dt; C.rx = d->rx; C.ry = d->ry; C.grx = d->grx; C.gry = d->gry; C.fric_coef = d->fric_coef;
    const size_t cells = (size_t)d->nx * d->ny;
    const size_t cfield = a256((size_t)C.cpitch * C.cny * sizeof(float));
    const size_t rb = a256((size_t)GC_ROWW * C.cny * sizeof(float));
    const size_t rb2 = a256((size_t)2 * C.cny * sizeof(float));
    C.bytes = 3 * cfield + rb + rb2;
    if (e->in_use + (long long)C.bytes > e->budget) return GC_ENOMEM;
    /* HP/HQ from the caller, else PQ_DEPTH (initialization.f90:2501-2526) */
    std::vector<float> hp(cells, 0.0f), hq(cells, 0.0f);
    if (d->hp && d->hq) {
        hp.assign(d->hp, d->hp + cells);
        hq.assign(d->hq, d->hq + cells);
    } else {
        for (int j = 0; j < d->ny; j++)
            for (int i = 0; i < d->nx; i++) {
                size_t c = (size_t)j * d->nx + i;
                if (d->h[c] > CC_GX) {
                    hp[c] = 0.5f * (d->h[c] + d->h[(size_t)j * d->nx + std::min(i + 1, d->nx - 1)]);
                    hq[c] = 0.5f * (d->h[c] + d->h[(size_t)std::min(j + 1, d->ny - 1) * d->nx + i]);
                }
            }
    }
    std::vector<float> rec((size_t)GC_ROWW * C.cny, 0.0f);
    if (d->rows)
        for (int k = 0; k < GC_NROW; k++)
            for (int j = 0; j < C.cny; j++) rec[(size_t)j * GC_ROWW + k] = d->rows[(size_t)k * C.cny + j];
    void *blk = nullptr;
    GC_CUDA_OR_RET(cudaMallocAsync(&blk, C.bytes, e->stream));
    C.block = blk;
    char *p = (char *)blk;
    C.d_ch = (float *)p; p += cfield;
    C.d_chp = (float *)p; p += cfield;
    C.d_chq = (float *)p; p += cfield;
    C.d_crows = (float *)p; p += rb;
    C.d_crows2 = (float *)p;
    GC_CUDA_OR_RET(cudaMemsetAsync(blk, 0, C.bytes, e->stream));
    const size_t sp = (size_t)C.cpitch * sizeof(float), hpitch = (size_t)d->nx * sizeof(float);
    GC_CUDA_OR_RET(cudaMemcpy2DAsync(C.d_ch, sp, d->h, hpitch, hpitch, (size_t)d->ny, cudaMemcpyHostToDevice,
                                     e->stream));
    GC_CUDA_OR_RET(cudaMemcpy2DAsync(C.d_chp, sp, hp.data(), hpitch, hpitch, (size_t)d->ny,
                                     cudaMemcpyHostToDevice, e->stream));
    GC_CUDA_OR_RET(cudaMemcpy2DAsync(C.d_chq, sp, hq.data(), hpitch, hpitch, (size_t)d->ny,
                                     cudaMemcpyHostToDevice, e->stream));
    GC_CUDA_OR_RET(cudaMemcpyAsync(C.d_crows, rec.data(), rec.size() * sizeof(float), cudaMemcpyHostToDevice,
                                   e->stream));
    std::vector<float> rec2((size_t)2 * C.cny, 0.0f);
    if (d->rows2)
        for (int j = 0; j < C.cny; j++) {
            rec2[2 * (size_t)j] = d->rows2[j];
            rec2[2 * (size_t)j + 1] = d->rows2[(size_t)C.cny + j];
        }
    GC_CUDA_OR_RET(cudaMemcpyAsync(C.d_crows2, rec2.data(), rec2.size() * sizeof(float), cudaMemcpyHostToDevice,
                                   e->stream));
    GC_CUDA_OR_RET(cudaStreamSynchronize(e->stream)); /* the host vectors end here */
    if (sc) {
        size_t sb = 0;
        const char *err = gc_sc_tables(d->nx, d->ny, C.cpitch, d->sc_pos, d->sc_cxy, d->corners, Pc.nx, Pc.ny,
                                       d->rel_size, d->sc_fix_top != 0, d->parent_modscm, &C.sc, &C.sc_block, &sb);
        if (err || e->in_use + (long long)(C.bytes + sb) > e->budget) {
            if (C.sc_block) cudaFree(C.sc_block);
            cudaFreeAsync(C.block, e->stream);
            return err ? GC_EINVAL : GC_ENOMEM;
        }
        C.has_sc = true;
        C.bytes += sb;
    }
    e->in_use += (long long)C.bytes;
    e->classes.push_back(C);
    return (int)e->classes.size() - 1;
}

int gc_engine_step(gc_engine *e, int nsteps) {
    if (!e || nsteps < 0) return GC_EINVAL;
    return eng_issue(e, nsteps);
}

int gc_engine_sync(gc_engine *e) {
    if (!e) return GC_EINVAL;
    GC_CUDA_OR_RET(cudaStreamSynchronize(e->stream));
    GC_CUDA_OR_RET(cudaGetLastError());
    const int a = gc_fused_take_error(), b = gc_pair_take_error();
    if (a || b) return GC_ETIMEOUT;
    return GC_OK;
}

int gc_engine_query(gc_engine *e) {
    if (!e) return GC_EINVAL;
    const cudaError_t q = cudaStreamQuery(e->stream);
    if (q == cudaErrorNotReady) return 0;
    GC_CUDA_OR_RET(q);
    return 1;
}

int gc_engine_member_done(gc_engine *e, int id) {
    if (!e || id < 0 || id >= (int)e->members.size() || !e->members[id].used) return GC_EINVAL;
    eng_retire(e);
    return e->members[id].done ? 1 : 0;
}

int gc_engine_member_steps(gc_engine *e, int id) {
    if (!e || id < 0 || id >= (int)e->members.size() || !e->members[id].used) return GC_EINVAL;
    const EngMember &M = e->members[id];
    return std::min(std::max(e->gstep - M.step0 + 1, 0), M.nsteps);
}

int gc_engine_read(gc_engine *e, int id, float *z, float *m, float *n, float *zmax, int *arrival, float *ts) {
    if (!e || id < 0 || id >= (int)e->members.size() || !e->members[id].used) return GC_EINVAL;
    EngMember &M = e->members[id];
    EngClass &C = e->classes[M.cls];
    /* level 1 after the member's completed steps */
    int done_steps = std::min(std::max(e->gstep - M.step0 + 1, 0), M.nsteps);
    int cur = M.level_buf(done_steps);
    size_t sp = (size_t)C.pitch * sizeof(float), dp = (size_t)C.nx * sizeof(float);
    auto dl = [&](void *dst, const void *src) {
        return cudaMemcpy2DAsync(dst, dp, src, sp, dp, (size_t)C.ny, cudaMemcpyDeviceToHost, e->stream);
    };
    if (z) GC_CUDA_OR_RET(dl(z, M.z[cur]));
    if (m) GC_CUDA_OR_RET(dl(m, M.m[cur]));
    if (n) GC_CUDA_OR_RET(dl(n, M.n[cur]));
    if (zmax) GC_CUDA_OR_RET(dl(zmax, M.zmax));
    if (arrival) GC_CUDA_OR_RET(dl(arrival, M.arrival));
    if (ts && M.ng > 0)
        GC_CUDA_OR_RET(cudaMemcpyAsync(ts, M.ts, (size_t)M.nsteps * M.ng * sizeof(float), cudaMemcpyDeviceToHost,
                                       e->stream));
    GC_CUDA_OR_RET(cudaStreamSynchronize(e->stream));
    return GC_OK;
}

int gc_engine_read_async(gc_engine *e, int id, float *z, float *m, float *n, float *zmax, int *arrival, float *ts,
                         void **done) {
    if (!e || id < 0 || id >= (int)e->members.size() || !e->members[id].used || !done) return GC_EINVAL;
    EngMember &M = e->members[id];
    EngClass &C = e->classes[M.cls];
    const int done_steps = std::min(std::max(e->gstep - M.step0 + 1, 0), M.nsteps);
    const int cur = M.level_buf(done_steps);
    size_t sp = (size_t)C.pitch * sizeof(float), dp = (size_t)C.nx * sizeof(float);
    auto dl = [&](void *dst, const void *src) {
        return cudaMemcpy2DAsync(dst, dp, src, sp, dp, (size_t)C.ny, cudaMemcpyDeviceToHost, e->stream);
    };
    if (z) GC_CUDA_OR_RET(dl(z, M.z[cur]));
    if (m) GC_CUDA_OR_RET(dl(m, M.m[cur]));
    if (n) GC_CUDA_OR_RET(dl(n, M.n[cur]));
    if (zmax) GC_CUDA_OR_RET(dl(zmax, M.zmax));
    if (arrival) GC_CUDA_OR_RET(dl(arrival, M.arrival));
    if (ts && M.ng > 0)
        GC_CUDA_OR_RET(cudaMemcpyAsync(ts, M.ts, (size_t)M.nsteps * M.ng * sizeof(float), cudaMemcpyDeviceToHost,
                                       e->stream));
    cudaEvent_t ev;
    GC_CUDA_OR_RET(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    GC_CUDA_OR_RET(cudaEventRecord(ev, e->stream));
    *done = (void *)ev;
    return GC_OK;
}

int gc_event_query(void *ev) {
    if (!ev) return GC_EINVAL;
    const cudaError_t q = cudaEventQuery((cudaEvent_t)ev);
    if (q == cudaErrorNotReady) return 0;
    GC_CUDA_OR_RET(q);
    return 1;
}

int gc_event_wait(void *ev) {
    if (!ev) return GC_EINVAL;
    GC_CUDA_OR_RET(cudaEventSynchronize((cudaEvent_t)ev));
    return GC_OK;
}

int gc_event_release(void *ev) {
    if (!ev) return GC_EINVAL;
    GC_CUDA_OR_RET(cudaEventDestroy((cudaEvent_t)ev));
    return GC_OK;
}

void *gc_host_alloc(long long bytes) {
    void *p = nullptr;
    if (bytes <= 0 || cudaHostAlloc(&p, (size_t)bytes, cudaHostAllocDefault) != cudaSuccess) return nullptr;
    return p;
}

int gc_host_free(void *p) {
    if (!p) return GC_EINVAL;
    GC_CUDA_OR_RET(cudaFreeHost(p));
    return GC_OK;
}

int gc_engine_read_child(gc_engine *e, int id, float *z, float *m, float *n) {
    if (!e || id < 0 || id >= (int)e->members.size() || !e->members[id].used || !e->members[id].nested)
        return GC_EINVAL;
    EngMember &M = e->members[id];
    EngClass &C = e->classes[M.cls];
    int done_steps = std::min(std::max(e->gstep - M.step0 + 1, 0), M.nsteps);
    int cur = (int)(((long long)done_steps * C.rel_time) & 1);
    size_t sp = (size_t)C.cpitch * sizeof(float), dp = (size_t)C.cnx * sizeof(float);
    auto dl = [&](void *dst, const void *src) {
        return cudaMemcpy2DAsync(dst, dp, src, sp, dp, (size_t)C.cny, cudaMemcpyDeviceToHost, e->stream);
    };
    if (z) GC_CUDA_OR_RET(dl(z, M.cz[cur]));
    if (m) GC_CUDA_OR_RET(dl(m, M.cm[cur]));
    if (n) GC_CUDA_OR_RET(dl(n, M.cn[cur]));
    GC_CUDA_OR_RET(cudaStreamSynchronize(e->stream));
    return GC_OK;
}

/* Scans the member's max-eta and current surfaces (outer grid and child).
 * The running maximum does not keep a NaN (a NaN maximum is replaced by the
 * next surface), but a NaN in a wet cell's surface persists: every stencil
 * operation and clamp of the step passes it on, so the current surface
 * shows it.  An Inf or |eta| beyond the bound shows in either field.
 * Returns 0 (healthy), a bit set (1: a NaN or Inf, 2: |eta| above `bound`
 * metres) or a negative status. */
int gc_engine_member_health(gc_engine *e, int id, float bound) {
    if (!e || id < 0 || id >= (int)e->members.size() || !e->members[id].used || !(bound > 0.0f))
        return GC_EINVAL;
    EngMember &M = e->members[id];
    EngClass &C = e->classes[M.cls];
    if (!e->d_health) GC_CUDA_OR_RET(cudaMallocAsync((void **)&e->d_health, sizeof(int), e->stream));
    GC_CUDA_OR_RET(cudaMemsetAsync(e->d_health, 0, sizeof(int), e->stream));
    const int done_steps = std::min(std::max(e->gstep - M.step0 + 1, 0), M.nsteps);
    const int cur = M.level_buf(done_steps);
    k_health<<<256, 256, 0, e->stream>>>(M.zmax, C.nx, C.ny, C.pitch, bound, e->d_health);
    k_health<<<256, 256, 0, e->stream>>>(M.z[cur], C.nx, C.ny, C.pitch, bound, e->d_health);
    e->launches += 2;
    if (M.nested) {
        const int ccur = (int)(((long long)done_steps * C.rel_time) & 1);
        k_health<<<64, 256, 0, e->stream>>>(M.cz[ccur], C.cnx, C.cny, C.cpitch, bound, e->d_health);
        e->launches++;
    }
    int h = 0;
    GC_CUDA_OR_RET(cudaMemcpyAsync(&h, e->d_health, sizeof(int), cudaMemcpyDeviceToHost, e->stream));
    GC_CUDA_OR_RET(cudaStreamSynchronize(e->stream));
    return h;
}

int gc_engine_release(gc_engine *e, int id) {
    if (!e || id < 0 || id >= (int)e->members.size() || !e->members[id].used) return GC_EINVAL;
    EngMember &M = e->members[id];
    if (!M.done) e->dirty = true;
    GC_CUDA_OR_RET(cudaFreeAsync(M.block, e->stream));
    e->in_use -= (long long)M.bytes;
    M = EngMember();
    return GC_OK;
}

long long gc_engine_bytes_in_use(gc_engine *e) { return e ? e->in_use : GC_EINVAL; }

/* candidates: c < nv * R1 is the one-step kernel, variant c % nv with
 * tile-height rule c / nv; above that the two-step kernel, variant p % np
 * with rule p / np (p = c - nv * R1) */

static int eng_num_candidates() {
    return gc_fused_num_variants() * GC_TY_RULES + gc_pair_num_variants() * GC_PAIR_RULES;
}

static bool eng_set_candidate(gc_engine *e, int c) {
    const int nv = gc_fused_num_variants(), n1 = nv * GC_TY_RULES, np = gc_pair_num_variants();
    if (c < 0 || c >= eng_num_candidates()) return false;
    if (c < n1) {
        e->variant = c % nv;
        e->ty_rule = c / nv;
        e->pair_on = 0;
    } else {
        const int q = c - n1;
        e->pair_variant = q % np;
        e->pair_rule = q / np;
        e->pair_on = 1;
    }
    e->dirty = true;
    return true;
}

int gc_engine_config(gc_engine *e, int variant, int use_graphs, int graph_chunk) {
    if (!e) return GC_EINVAL;
    if (variant >= 0) {
        if (!eng_set_candidate(e, variant)) return GC_EINVAL;
        e->tuned = true;
    }
    e->use_graphs = use_graphs ? 1 : 0;
    /* even, so a replayed chunk starts at the ping-pong parity it was captured at */
    if (graph_chunk > 0) e->chunk = (graph_chunk + 1) & ~1;
    e->dirty = true;
    return GC_OK;
}

/* Times real steps of every candidate on the current members and keeps the
 * fastest per step.  Every candidate computes bit-identical results, so the
 * tuning steps are ordinary steps of the run. */
int gc_engine_autotune(gc_engine *e, int reps) {
    if (!e || reps < 1) return GC_EINVAL;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const int nv = gc_fused_num_variants(), n1 = nv * GC_TY_RULES;
    int best = -1;
    float best_ms = 3.0e38f;
    int saved_graphs = e->use_graphs;
    e->use_graphs = 0;
    /* per-step time of candidate c over `rounds` x its steps (whole pairs for
     * the two-step ones), after one warm launch; with `chunks` > 0, as the
     * run issues them: graph replays of `chunks` step chunks after a warm
     * chunk (which also builds the graph).  < 0 when the members ran out of
     * steps. */
    auto time_candidate = [&](int c, int rounds, int chunks = 0) -> float {
        eng_set_candidate(e, c);
        e->use_graphs = chunks > 0 ? saved_graphs : 0;
        const int n = chunks > 0 ? chunks * e->chunk : (c >= n1 ? 2 * reps : reps) * rounds;
        if (eng_issue(e, chunks > 0 ? e->chunk : (c >= n1 ? 2 : 1)) < 0) return -1.0f; /* warm */
        cudaEventRecord(a, e->stream);
        int got = eng_issue(e, n);
        cudaEventRecord(b, e->stream);
        cudaEventSynchronize(b);
        if (got < n) return -1.0f;
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, a, b);
        return ms / (float)got;
    };
    std::vector<std::pair<float, int>> times;
    bool short_of_steps = false;
    for (int c = 0; c < eng_num_candidates(); c++) {
        if (c >= n1 && !e->pair_allowed) break;
        const float ms = time_candidate(c, 1);
        if (ms < 0.0f) {
            short_of_steps = true;
            break;
        }
        times.push_back({ms, c});
        if (ms < best_ms) { best_ms = ms; best = c; }
    }
    /* the three fastest again, over more steps and issued as the run will
     * issue them (step-chunk graphs when the engine uses them): one short
     * window of eager launches cannot separate candidates a few percent
     * apart */
    if (!short_of_steps && times.size() > 1) {
        std::sort(times.begin(), times.end());
        float best2 = 3.0e38f;
        int pick = -1;
        for (size_t k = 0; k < times.size() && k < 3; k++) {
            const float ms = saved_graphs ? time_candidate(times[k].second, 0, 2) : time_candidate(times[k].second, 3);
            if (ms < 0.0f) break;
            if (ms < best2) { best2 = ms; pick = times[k].second; }
        }
        if (pick >= 0) best = pick;
    }
    if (best < 0) best = e->pair_allowed ? n1 : 16;
    eng_set_candidate(e, best);
    e->tuned = true;
    e->use_graphs = saved_graphs;
    e->dirty = true;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return best;
}

int gc_engine_prepare(gc_engine *e) {
    if (!e) return GC_EINVAL;
    eng_retire(e);
    if (e->dirty && eng_rebuild(e) != GC_OK) return GC_ECUDA;
    if (e->use_graphs && !e->gexec && (e->ntiles > 0 || !e->nested_ids.empty()))
        GC_CUDA_OR_RET(eng_build_graph(e));
    GC_CUDA_OR_RET(cudaStreamSynchronize(e->stream));
    return GC_OK;
}

int gc_engine_variant(gc_engine *e) {
    if (!e) return GC_EINVAL;
    if (e->pair_on && e->pair_allowed)
        return gc_fused_num_variants() * GC_TY_RULES + e->pair_variant + gc_pair_num_variants() * e->pair_rule;
    return e->variant + gc_fused_num_variants() * e->ty_rule;
}
int gc_engine_num_variants(void) { return gc_fused_num_variants(); }
int gc_engine_num_candidates(void) { return eng_num_candidates(); }

void *gc_engine_stream(gc_engine *e) { return e ? (void *)e->stream : nullptr; }
long long gc_engine_launches(gc_engine *e) { return e ? e->launches : GC_EINVAL; }

} /* extern "C" */
