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
    size_t bytes = 0;
};

struct EngMember {
    bool used = false, done = false;
    int cls = 0, nsteps = 0, step0 = 0, ng = 0;
    float thr = -1.0f;
    void *block = nullptr;
    size_t bytes = 0;
    float *z[2] = {nullptr, nullptr}, *m[2] = {nullptr, nullptr}, *n[2] = {nullptr, nullptr};
    float *zmax = nullptr, *ts = nullptr, *gw = nullptr;
    int *arrival = nullptr, *gij = nullptr;
};

size_t a256(size_t x) { return (x + 255) & ~(size_t)255; }

__global__ void k_advance(int *step, int by) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *step += by;
}

} // namespace

struct gc_engine {
    long long budget = 0, in_use = 0;
    cudaStream_t stream = nullptr;
    std::vector<EngClass> classes;
    std::vector<EngMember> members;
    int variant = 1;
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
};

static int eng_rebuild(gc_engine *e) {
    std::vector<GcFusedGrid> grids;
    std::vector<int2> tiles;
    /* one tile height for the whole work list, chosen to fill whole waves */
    std::vector<int> anx, any;
    for (auto &M : e->members)
        if (M.used && !M.done) { anx.push_back(e->classes[M.cls].nx); any.push_back(e->classes[M.cls].ny); }
    const int ty = anx.empty() ? 16 : gc_fused_pick_ty(e->variant, (int)anx.size(), anx.data(), any.data());
    /* active members grouped by class */
    for (size_t c = 0; c < e->classes.size(); c++) {
        EngClass &C = e->classes[c];
        std::vector<int> idx;
        for (size_t k = 0; k < e->members.size(); k++) {
            EngMember &M = e->members[k];
            if (!M.used || M.done || M.cls != (int)c) continue;
            idx.push_back((int)grids.size());
            GcFusedGrid g;
            memset(&g, 0, sizeof g);
            g.nx = C.nx; g.ny = C.ny; g.pitch = C.pitch; g.root = 1; g.explicit_r24 = 0;
            g.ty = ty;
            gc_fused_tiles(C.nx, C.ny, ty, &g.tiles_x);
            g.step0 = M.step0; g.cur0 = 0; g.nsteps = M.nsteps;
            g.flags = GC_F_MAXAMP | (M.thr >= 0.0f ? GC_F_ARRIVAL : 0);
            g.thr = M.thr;
            for (int q = 0; q < 2; q++) { g.z[q] = M.z[q]; g.m[q] = M.m[q]; g.n[q] = M.n[q]; }
            g.h = C.d_h; g.rows = C.d_rows;
            g.zmax = M.zmax; g.arrival = M.arrival;
            g.ng = M.ng; g.gij = M.gij; g.gw = M.gw; g.ts = M.ts; g.ts_len = M.nsteps;
            grids.push_back(g);
        }
        int nt = gc_fused_tiles(C.nx, C.ny, ty, nullptr);
        for (int t = 0; t < nt; t++)
            for (int g : idx) tiles.push_back(make_int2(g, t));
    }
    e->ngrids = (int)grids.size();
    e->ntiles = (int)tiles.size();
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
    /* the host copies above are from pageable memory and complete before return */
    e->nctas = e->ntiles;
    if (e->gexec) { cudaGraphExecDestroy(e->gexec); e->gexec = nullptr; }
    e->dirty = false;
    return GC_OK;
}

/* retire members whose last gauge sample has been issued */
static void eng_retire(gc_engine *e) {
    for (auto &M : e->members)
        if (M.used && !M.done && e->gstep >= M.step0 + M.nsteps) {
            M.done = true;
            e->dirty = true;
        }
}

static int eng_issue(gc_engine *e, int nsteps) {
    int issued = 0;
    while (issued < nsteps) {
        eng_retire(e);
        if (e->dirty && eng_rebuild(e) != GC_OK) return GC_ECUDA;
        if (e->ntiles == 0) break;
        /* steps until the next member finishes: the member set is constant */
        int horizon = nsteps - issued;
        for (auto &M : e->members)
            if (M.used && !M.done) horizon = std::min(horizon, M.step0 + M.nsteps - e->gstep);
        if (horizon <= 0) horizon = 1;
        if (e->use_graphs && horizon >= e->chunk) {
            if (!e->gexec) {
                GC_CUDA_OR_RET(cudaMemcpyAsync(e->d_step, &e->gstep, sizeof(int), cudaMemcpyHostToDevice,
                                               e->stream));
                cudaGraph_t graph;
                GC_CUDA_OR_RET(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
                for (int k = 1; k <= e->chunk; k++)
                    gc_fused_launch_multi(e->variant, e->d_grids, e->d_tiles, e->ntiles, e->d_step, k,
                                          e->nctas, e->stream);
                k_advance<<<1, 32, 0, e->stream>>>(e->d_step, e->chunk);
                GC_CUDA_OR_RET(cudaStreamEndCapture(e->stream, &graph));
                GC_CUDA_OR_RET(cudaGraphInstantiate(&e->gexec, graph, 0));
                cudaGraphDestroy(graph);
            } else {
                /* the device counter must equal the host's step count */
                GC_CUDA_OR_RET(cudaMemcpyAsync(e->d_step, &e->gstep, sizeof(int), cudaMemcpyHostToDevice,
                                               e->stream));
            }
            int reps = horizon / e->chunk;
            if (reps * e->chunk > nsteps - issued) reps = (nsteps - issued) / e->chunk;
            if (reps <= 0) reps = 0;
            for (int r = 0; r < reps; r++) {
                GC_CUDA_OR_RET(cudaGraphLaunch(e->gexec, e->stream));
                e->launches += e->chunk;
            }
            e->gstep += reps * e->chunk;
            issued += reps * e->chunk;
            if (reps > 0) continue;
        }
        int n = std::min(horizon, nsteps - issued);
        for (int k = 0; k < n; k++) {
            cudaError_t err = gc_fused_launch_multi(e->variant, e->d_grids, e->d_tiles, e->ntiles, nullptr,
                                                    e->gstep + 1, e->nctas, e->stream);
            if (err != cudaSuccess) return GC_ECUDA;
            e->gstep++;
            e->launches++;
        }
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
        if (C.d_h) cudaFreeAsync(C.d_h, e->stream);
    }
    if (e->d_grids) cudaFreeAsync(e->d_grids, e->stream);
    if (e->d_tiles) cudaFreeAsync(e->d_tiles, e->stream);
    if (e->d_step) cudaFreeAsync(e->d_step, e->stream);
    cudaStreamSynchronize(e->stream);
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

long long gc_engine_member_bytes(gc_engine *e, int cls) {
    if (!e || cls < 0 || cls >= (int)e->classes.size()) return GC_EINVAL;
    EngClass &C = e->classes[cls];
    size_t field = a256((size_t)C.pitch * C.ny * sizeof(float));
    return (long long)(8 * field);
}

int gc_engine_add_member(gc_engine *e, int cls, const float *z0, int nsteps, int ngauges, const int *gij,
                         const float *gw, float arrival_thr) {
    if (!e || cls < 0 || cls >= (int)e->classes.size() || !z0 || nsteps < 1 || ngauges < 0) return GC_EINVAL;
    if (ngauges > 0 && (!gij || !gw)) return GC_EINVAL;
    EngClass &C = e->classes[cls];
    for (int g = 0; g < ngauges; g++)
        if (gij[2 * g] < 1 || gij[2 * g + 1] < 1 || gij[2 * g] >= C.nx || gij[2 * g + 1] >= C.ny) return GC_EINVAL;
    size_t field = a256((size_t)C.pitch * C.ny * sizeof(float));
    size_t tsb = a256((size_t)nsteps * ngauges * sizeof(float));
    size_t gb = a256((size_t)2 * ngauges * sizeof(int)) + a256((size_t)2 * ngauges * sizeof(float));
    size_t bytes = 8 * field + tsb + gb;
    if (e->in_use + (long long)bytes > e->budget) return GC_ENOMEM;
    EngMember M;
    M.used = true;
    M.cls = cls; M.nsteps = nsteps; M.ng = ngauges; M.thr = arrival_thr;
    M.step0 = e->gstep + 1;
    M.bytes = bytes;
    GC_CUDA_OR_RET(cudaMallocAsync(&M.block, bytes, e->stream));
    char *p = (char *)M.block;
    for (int q = 0; q < 2; q++) {
        M.z[q] = (float *)p; p += field;
        M.m[q] = (float *)p; p += field;
        M.n[q] = (float *)p; p += field;
    }
    M.zmax = (float *)p; p += field;
    M.arrival = (int *)p; p += field;
    M.ts = (float *)p; p += tsb;
    M.gij = (int *)p; p += a256((size_t)2 * ngauges * sizeof(int));
    M.gw = (float *)p;
    GC_CUDA_OR_RET(cudaMemsetAsync(M.block, 0, 6 * field, e->stream));
    GC_CUDA_OR_RET(cudaMemsetAsync(M.arrival, 0xff, field, e->stream));
    GC_CUDA_OR_RET(cudaMemcpy2DAsync(M.z[0], (size_t)C.pitch * sizeof(float), z0, (size_t)C.nx * sizeof(float),
                                     (size_t)C.nx * sizeof(float), (size_t)C.ny, cudaMemcpyHostToDevice, e->stream));
    GC_CUDA_OR_RET(cudaMemcpyAsync(M.zmax, M.z[0], field, cudaMemcpyDeviceToDevice, e->stream));
    if (ngauges > 0) {
        GC_CUDA_OR_RET(cudaMemcpyAsync(M.gij, gij, (size_t)2 * ngauges * sizeof(int), cudaMemcpyHostToDevice,
                                       e->stream));
        GC_CUDA_OR_RET(cudaMemcpyAsync(M.gw, gw, (size_t)2 * ngauges * sizeof(float), cudaMemcpyHostToDevice,
                                       e->stream));
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

int gc_engine_step(gc_engine *e, int nsteps) {
    if (!e || nsteps < 0) return GC_EINVAL;
    return eng_issue(e, nsteps);
}

int gc_engine_sync(gc_engine *e) {
    if (!e) return GC_EINVAL;
    GC_CUDA_OR_RET(cudaStreamSynchronize(e->stream));
    GC_CUDA_OR_RET(cudaGetLastError());
    if (gc_fused_take_error()) return GC_ETIMEOUT;
    return GC_OK;
}

int gc_engine_member_done(gc_engine *e, int id) {
    if (!e || id < 0 || id >= (int)e->members.size() || !e->members[id].used) return GC_EINVAL;
    eng_retire(e);
    return e->members[id].done ? 1 : 0;
}

int gc_engine_read(gc_engine *e, int id, float *z, float *m, float *n, float *zmax, int *arrival, float *ts) {
    if (!e || id < 0 || id >= (int)e->members.size() || !e->members[id].used) return GC_EINVAL;
    EngMember &M = e->members[id];
    EngClass &C = e->classes[M.cls];
    /* level 1 after the member's completed steps */
    int done_steps = std::min(std::max(e->gstep - M.step0 + 1, 0), M.nsteps);
    int cur = done_steps & 1;
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

int gc_engine_config(gc_engine *e, int variant, int use_graphs, int graph_chunk) {
    if (!e) return GC_EINVAL;
    if (variant >= 0) {
        if (variant >= gc_fused_num_variants()) return GC_EINVAL;
        e->variant = variant;
        e->tuned = true;
    }
    e->use_graphs = use_graphs ? 1 : 0;
    if (graph_chunk > 0) e->chunk = graph_chunk;
    e->dirty = true;
    return GC_OK;
}

/* Times `reps` real steps of every tile variant on the current members and
 * keeps the fastest.  Every variant computes bit-identical results, so the
 * tuning steps are ordinary steps of the run. */
int gc_engine_autotune(gc_engine *e, int reps) {
    if (!e || reps < 1) return GC_EINVAL;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    int best = e->variant;
    float best_ms = 3.0e38f;
    int saved_graphs = e->use_graphs;
    e->use_graphs = 0;
    for (int v = 0; v < gc_fused_num_variants(); v++) {
        e->variant = v;
        e->dirty = true;
        if (eng_issue(e, 1) < 0) return GC_ECUDA; /* warm */
        cudaEventRecord(a, e->stream);
        int got = eng_issue(e, reps);
        cudaEventRecord(b, e->stream);
        cudaEventSynchronize(b);
        if (got < reps) break;
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, a, b);
        if (ms < best_ms) { best_ms = ms; best = v; }
    }
    e->variant = best;
    e->tuned = true;
    e->use_graphs = saved_graphs;
    e->dirty = true;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return best;
}

int gc_engine_variant(gc_engine *e) { return e ? e->variant : GC_EINVAL; }
void *gc_engine_stream(gc_engine *e) { return e ? (void *)e->stream : nullptr; }
long long gc_engine_launches(gc_engine *e) { return e ? e->launches : GC_EINVAL; }

} /* extern "C" */
