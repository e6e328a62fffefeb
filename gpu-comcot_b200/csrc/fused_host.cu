/*
 * Host side of the fused step for the reference-ABI path: builds the grid
 * descriptor of the outer layer and issues one launch per outer step.
 */
#include <string.h>

#include "fused.h"
#include "runtime.h"

static int g_variant = -1;

int gc_default_variant() {
    if (g_variant >= 0) return g_variant;
    const char *v = getenv("GCOMCOT_FUSED_VARIANT");
    /* 16: 4 warps x 3 stages, N of row r-2 carried in registers, 20 warps
     * per SM (the fastest on the 2401x2001 single grid on B200) */
    g_variant = v ? atoi(v) : 16;
    if (g_variant < 0 || g_variant >= gc_fused_num_variants()) g_variant = 0;
    return g_variant;
}

void gc_fill_fused_grid(const GcLayer &L, GcFusedGrid &g) {
    memset(&g, 0, sizeof g);
    g.nx = L.nx; g.ny = L.ny; g.pitch = L.pitch;
    g.root = (L.parent == -1) ? 1 : 0;
    g.explicit_r24 = L.explicit_r24 ? 1 : 0;
    for (int k = 0; k < 2; k++) { g.z[k] = L.z[k]; g.m[k] = L.m[k]; g.n[k] = L.n[k]; }
    g.h = L.h; g.rows = L.rows; g.r2 = L.r2; g.r4 = L.r4;
    g.zmax = L.zmax; g.arrival = L.arrival;
}

bool gc_fused_step(GcLayer &L, bool maxamp, bool arrival, int step, float thr, int ngauges,
                   const int *d_ij, float *d_out, cudaStream_t s) {
    (void)ngauges; (void)d_ij; (void)d_out;
    if (L.laycord != 0 || L.laygov != 0) return false;
    if (L.parent != -1 && !L.children.empty()) return false;
    GcFusedGrid g;
    gc_fill_fused_grid(L, g);
    int v = gc_default_variant();
    static int cached_nx = -1, cached_ny = -1, cached_v = -1, cached_ty = 16;
    if (cached_nx != L.nx || cached_ny != L.ny || cached_v != v) {
        /* the single-grid kernel; rule 1 (fewest rows for the busiest warp) */
        cached_ty = gc_fused_pick_ty(v, 1, &L.nx, &L.ny, 1, false);
        cached_nx = L.nx; cached_ny = L.ny; cached_v = v;
    }
    g.ty = cached_ty;
    gc_fused_tiles(L.nx, L.ny, g.ty, &g.tiles_x);
    g.step0 = step;
    g.cur0 = L.cur;
    g.nsteps = 0x3fffffff;
    g.flags = (maxamp ? GC_F_MAXAMP : 0) | (arrival ? GC_F_ARRIVAL : 0);
    g.thr = thr;
    cudaError_t e = gc_fused_launch_one(v, g, step, s);
    if (e != cudaSuccess) {
        fprintf(stderr, "gcomcot: fused launch failed: %s\n", cudaGetErrorString(e));
        exit(EXIT_FAILURE);
    }
    return true;
}
