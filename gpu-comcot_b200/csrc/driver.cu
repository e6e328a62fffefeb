/*
 * The reference driver's per-step call sequence as a library entry point, the
 * gauge snapshot that serves gcomcot_get_z_ after the first step with one
 * device round trip per step, and the DEBUG_CORE comparators.
 */
#include <math.h>
#include <string.h>

#include <vector>

#include "gcomcot.h"
#include "runtime.h"

/* ------------------------------------------------------------------ */
/* gauge snapshot                                                      */
/* ------------------------------------------------------------------ */
struct GaugeReg {
    int lid, i, j;
};
static std::vector<GaugeReg> g_reg;
static bool g_snap_valid = false;
static bool g_ij_stale = true;    /* the device copy of the stencil indices needs an upload */
static int *g_d_ij = nullptr;     /* [2*cap] */
static float *g_h_out = nullptr;  /* mapped pinned [4*cap] */
static float *g_d_out = nullptr;  /* device alias of g_h_out */
static int g_cap = 0;

void gc_gauge_invalidate() { g_snap_valid = false; }

static int ensure_cap(int n) {
    if (n <= g_cap) return GC_OK;
    int cap = n < 64 ? 64 : 2 * n;
    if (g_d_ij) cudaFree(g_d_ij);
    if (g_h_out) cudaFreeHost(g_h_out);
    g_ij_stale = true;
    GC_CUDA_OR_RET(cudaMalloc(&g_d_ij, (size_t)2 * cap * sizeof(int)));
    GC_CUDA_OR_RET(cudaHostAlloc((void **)&g_h_out, (size_t)4 * cap * sizeof(float), cudaHostAllocMapped));
    GC_CUDA_OR_RET(cudaHostGetDevicePointer((void **)&g_d_out, g_h_out, 0));
    g_cap = cap;
    return GC_OK;
}

/* samples every registered gauge stencil of the current state, one launch
 * per layer that has gauges, then waits */
static int snapshot() {
    GcRuntime &rt = gc_rt();
    GcPdlScope pdl(true); /* the gauge kernel waits for the step on the device */
    int n = (int)g_reg.size();
    if (ensure_cap(n) != GC_OK) return GC_ECUDA;
    if (g_ij_stale) {
        /* only when the set of gauges changed: a copy from pageable memory
         * waits for the stream, which would cost a second round trip a step */
        std::vector<int> ij((size_t)2 * n);
        for (int g = 0; g < n; g++) { ij[2 * g] = g_reg[g].i; ij[2 * g + 1] = g_reg[g].j; }
        GC_CUDA_OR_RET(cudaMemcpy(g_d_ij, ij.data(), ij.size() * sizeof(int), cudaMemcpyHostToDevice));
        g_ij_stale = false;
    }
    /* gauges are registered grouped by first use; launch per run of equal lid */
    int g0 = 0;
    while (g0 < n) {
        int lid = g_reg[g0].lid, g1 = g0;
        while (g1 < n && g_reg[g1].lid == lid) g1++;
        GcLayer *L = gc_layer(lid);
        GcLayerDev d = L->view();
        if (!L->z2_valid) d.z2 = L->z[L->cur];
        gc_launch_gauges(d, g1 - g0, g_d_ij + 2 * g0, g_d_out + 4 * g0, rt.stream);
        rt.launches++;
        g0 = g1;
    }
    GC_CUDA_OR_RET(cudaStreamSynchronize(rt.stream));
    g_snap_valid = true;
    return GC_OK;
}

static int g_last = -1; /* registry slot of the previous lookup */

/* serves gcomcot_get_z_; returns false when the caller must fall back */
bool gc_gauge_lookup(int lid, int i, int j, float *out4) {
    int n = (int)g_reg.size();
    int found = -1;
    /* a driver asks for its gauges in the same order every step: try the
     * slot after the previous one first */
    const int guess = (g_last + 1 < n) ? g_last + 1 : 0;
    if (guess < n && g_reg[guess].lid == lid && g_reg[guess].i == i && g_reg[guess].j == j) found = guess;
    for (int g = 0; found < 0 && g < n; g++)
        if (g_reg[g].lid == lid && g_reg[g].i == i && g_reg[g].j == j) found = g;
    if (found < 0) {
        /* keep same-layer gauges contiguous */
        size_t pos = g_reg.size();
        for (size_t k = g_reg.size(); k > 0; k--)
            if (g_reg[k - 1].lid == lid) { pos = k; break; }
        g_reg.insert(g_reg.begin() + pos, GaugeReg{lid, i, j});
        found = (int)pos;
        g_snap_valid = false;
        g_ij_stale = true;
    }
    if (!g_snap_valid) {
        gc_flush();
        if (snapshot() != GC_OK) return false;
    }
    memcpy(out4, g_h_out + 4 * found, 4 * sizeof(float));
    g_last = found;
    return true;
}

void gc_gauge_release() {
    if (g_d_ij) cudaFree(g_d_ij);
    if (g_h_out) cudaFreeHost(g_h_out);
    g_d_ij = nullptr; g_h_out = nullptr; g_d_out = nullptr; g_cap = 0;
    g_reg.clear();
    g_last = -1;
    g_snap_valid = false;
    g_ij_stale = true;
}

extern "C" {

int gcomcot_drive(int nsteps, int maxamp, int ngauges, const int *g_layer, const int *g_i,
                  const int *g_j, float *out4) {
    GcRuntime &rt = gc_rt();
    if (!rt.inited || rt.root < 0) return GC_ESTATE;
    int root = rt.root;
    bool nested = !rt.layers[root].children.empty();
    for (int k = 0; k < nsteps; k++) {
        mass_launch_(nullptr, nullptr, nullptr, &root);
        openbd_launch_(nullptr);
        if (nested) all_grid_launch_();
        momt_launch_(nullptr, nullptr, nullptr, &root);
        if (maxamp) maxamp_launch_(&root);
        for (int g = 0; g < ngauges; g++) {
            float *o = out4 + ((size_t)k * ngauges + g) * 4;
            int lid = g_layer[g], i = g_i[g], j = g_j[g];
            gcomcot_get_z_(&lid, o, o + 1, o + 2, o + 3, &i, &j);
        }
        cuda_update_layer_(&root);
    }
    return gcomcot_sync();
}

/* GPUall_grids.cu:299-394: device JNQ/NEWQ for (idO, idA) at sub-step t,
 * then a cell-by-cell comparison of the child's boundary fluxes with the
 * caller's, printed like the reference (absolute tolerance 1e-4) */
void edgeinterp_dbglaunch_(float *mO, float *nO, int *idO, float *mA, float *nA, int *idA, int *t,
                           float *yflux, float *xflux) {
    (void)mO; (void)nO; (void)yflux; (void)xflux;
    GcLayer *P = gc_layer(*idO), *C = gc_layer(*idA);
    if (!P || !C || !P->used || !C->used) exit(EXIT_FAILURE);
    gc_flush();
    gc_launch_edges(P->view(), C->view(), C->rel_size, C->rel_time, C->corners, *t, gc_rt().stream);
    std::vector<float> m((size_t)C->nx * C->ny), n((size_t)C->nx * C->ny);
    if (gc_layer_download_field(*C, C->m[C->cur], m.data()) != GC_OK) exit(EXIT_FAILURE);
    if (gc_layer_download_field(*C, C->n[C->cur], n.data()) != GC_OK) exit(EXIT_FAILURE);
    for (int j = 0; j < C->ny; j++) {
        for (int side = 0; side < 2; side++) {
            size_t id = (size_t)j * C->nx + (side ? C->nx - 1 : 0);
            if (fabsf(m[id] - mA[id]) >= 1.0e-4f)
                printf("(%s) i = %d, %f, %f, diff=%f\n", side ? "right" : "left", j, m[id], mA[id],
                       fabsf(m[id] - mA[id]));
        }
    }
    for (int i = 0; i < C->nx; i++) {
        for (int side = 0; side < 2; side++) {
            size_t id = (size_t)(side ? C->ny - 1 : 0) * C->nx + i;
            if (fabsf(n[id] - nA[id]) >= 1.0e-4f)
                printf("(%s) i = %d, %f, %f, diff=%f\n", side ? "top" : "bottom", i, n[id], nA[id],
                       fabsf(n[id] - nA[id]));
        }
    }
}

/* GPUall_grids.cu:626-643: device JNZ, then compare the parent surface */
void jnz_dbglaunch_(float *Z_f, int *outid, int *inid) {
    GcLayer *P = gc_layer(*outid), *C = gc_layer(*inid);
    if (!P || !C || !P->used || !C->used) exit(EXIT_FAILURE);
    gc_flush();
    gc_launch_jnz(P->view(), C->view(), C->rel_size, C->rel_time, C->corners, gc_rt().stream);
    P->z2_valid = true;
    std::vector<float> z((size_t)P->nx * P->ny);
    if (gc_layer_download_field(*P, P->z[P->cur ^ 1], z.data()) != GC_OK) exit(EXIT_FAILURE);
    for (int j = 0; j < P->ny; j++)
        for (int i = 0; i < P->nx; i++) {
            size_t id = (size_t)j * P->nx + i;
            if (fabsf(z[id] - Z_f[id]) >= 1.0e-4f)
                printf("JNZ, layerid=%d(i,j)=(%d,%d), %f %f, diff=%lf\n", *inid, i, j, z[id], Z_f[id],
                       (double)fabsf(z[id] - Z_f[id]));
        }
}

} /* extern "C" */
