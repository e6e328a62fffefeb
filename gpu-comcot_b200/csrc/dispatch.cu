/*
 * Deferred outer-layer work and the extended C API.
 *
 * The reference's driver calls MASS_LAUNCH, OPENBD_LAUNCH, MOMT_LAUNCH and
 * MAXAMP_LAUNCH one after another for layer 1 (comcot.f90:362,367,399,421).
 * The legacy entry points only record those calls; the first call that needs
 * their results (a read, a nested sub-cycle, the time-level swap) flushes
 * them.  A complete mass -> open -> momentum [-> max] sequence on a linear
 * spherical layer is issued as one fused kernel (kernels_fused.cu); any other
 * pattern falls back to one kernel per phase.  The order of effects is the
 * order of the calls either way.
 */
#include <string.h>

#include <vector>

#include "fused.h"
#include "runtime.h"

bool gc_fused_step(GcLayer &L, bool maxamp, bool arrival, int step, float thr, int ngauges,
                   const int *d_ij, float *d_out, cudaStream_t s);

struct GcArrivalCfg {
    bool on = false;
    float thr = 0.0f;
    int step = 1;
};
static GcArrivalCfg g_arr;

void gc_flush() {
    GcRuntime &rt = gc_rt();
    /* each step's kernels are scheduled while the previous one runs and wait
     * for it on the device */
    GcPdlScope pdl(true);
    if (!(rt.pend_mass | rt.pend_open | rt.pend_momt | rt.pend_maxamp)) return;
    GcLayer &L = rt.layers[rt.root];
    bool done = false;
    if (rt.fuse_enabled && rt.pend_mass && rt.pend_open && rt.pend_momt && L.laycord == 0 && L.laygov == 0) {
        done = gc_fused_step(L, rt.pend_maxamp != 0, false, 0, 0.0f, 0, nullptr, nullptr, rt.stream);
        if (done) rt.launches++;
    }
    if (!done) {
        GcLayerDev d = L.view();
        if (rt.pend_mass) { gc_launch_mass(d, rt.stream); rt.launches++; }
        if (rt.pend_open) { gc_launch_open(d, rt.stream); rt.launches++; }
        if (rt.pend_momt) { gc_launch_moment(d, rt.stream); rt.launches++; }
        if (rt.pend_maxamp) { gc_launch_maxamp(d, rt.stream); rt.launches++; }
    }
    rt.pend_mass = rt.pend_open = rt.pend_momt = rt.pend_maxamp = 0;
}

bool gc_arrival_on() { return g_arr.on; }

/* called by cuda_update_layer_ for the outermost layer before its swap */
void gc_root_change_hook(GcLayer &L) {
    if (!g_arr.on) return;
    GcLayerDev d = L.view();
    gc_launch_arrival(d, g_arr.step, g_arr.thr, gc_rt().stream);
    gc_rt().launches++;
    g_arr.step++;
}

extern "C" {

/* extension: record, per wet cell of layer `id`, the first outer step after
 * which the surface exceeds `thr` (metres); 0 for a wet cell already above it
 * when the call is made, -1 until then elsewhere.  The reference has no
 * arrival-time product; this is evaluated at every CHANGE of layer 1. */
void gcomcot_set_arrival_(int *id, float *thr) {
    (void)id;
    g_arr.on = true;
    g_arr.thr = *thr;
    g_arr.step = 1;
    GcRuntime &rt = gc_rt();
    if (rt.inited && rt.root >= 0) {
        GcLayer &L = rt.layers[rt.root];
        gc_launch_arrival_start(L.arrival, L.z[L.cur], L.h, L.nx, L.ny, L.pitch, *thr, rt.stream);
        rt.launches++;
    }
}

void gcomcot_get_arrival_(int *arr, int *id) {
    GcLayer *L = gc_layer(*id);
    if (!L || !L->used) exit(EXIT_FAILURE);
    gc_flush();
    GC_CUDA_OR_DIE(cudaMemcpy2DAsync(arr, (size_t)L->nx * sizeof(int), L->arrival,
                                     (size_t)L->pitch * sizeof(int), (size_t)L->nx * sizeof(int),
                                     (size_t)L->ny, cudaMemcpyDeviceToHost, gc_rt().stream));
    GC_CUDA_OR_DIE(cudaStreamSynchronize(gc_rt().stream));
}

/* number of kernels this library has launched since initialisation */
long long gcomcot_launch_count(void) { return gc_rt().launches; }

/* 1: mass/open/momentum of layer 1 may be fused (default); 0: one kernel per phase */
void gcomcot_set_fusion(int on) { gc_rt().fuse_enabled = on ? 1 : 0; }

/* blocks until all queued work finished; returns 0 or a negative status */
int gcomcot_sync(void) {
    gc_flush();
    GC_CUDA_OR_RET(cudaStreamSynchronize(gc_rt().stream));
    GC_CUDA_OR_RET(cudaGetLastError());
    const int a = gc_fused_take_error(), b = gc_pair_take_error();
    if (a || b) return GC_ETIMEOUT;
    return GC_OK;
}

void gcomcot_set_wait_limit(int polls) { gc_pair_set_wait_limit(polls); }

void gcomcot_inject_stall(void) { gc_pair_stall_next(); }

/* the library's stream, for callers that time work with CUDA events */
void *gcomcot_stream(void) { return (void *)gc_rt().stream; }

} /* extern "C" */
