/*
 * Host-side layer registry shared by the reference-ABI entry points, the
 * step driver and the fused-path dispatcher.
 */
#ifndef GC_RUNTIME_H
#define GC_RUNTIME_H

#include <vector>

#include "gc_internal.h"

struct GcLayer {
    bool used = false;
    int id = 0, parent = -1, level = 1, rel_size = 1, rel_time = 1;
    int corners[4] = {1, 1, 1, 1};
    int nx = 0, ny = 0, pitch = 0;
    int laycord = 0, laygov = 0, linchk = 1, modscm = 1, fric_switch = 1;
    float grx = 0, gry = 0, rx = 0, ry = 0, dt = 0, fric_coef = 0;
    bool explicit_r24 = false;
    /* device storage: one allocation carved into fields */
    void *block = nullptr;
    size_t block_bytes = 0;
    float *z[2] = {nullptr, nullptr}, *m[2] = {nullptr, nullptr}, *n[2] = {nullptr, nullptr};
    float *h = nullptr, *hp = nullptr, *hq = nullptr, *r2 = nullptr, *r4 = nullptr;
    float *rows = nullptr, *dz2 = nullptr, *xflux = nullptr, *yflux = nullptr, *zmax = nullptr;
    float *rows2 = nullptr; /* [ny][2] R0, R22 of nonlinear spherical layers */
    int *arrival = nullptr;
    float *spx = nullptr, *spy = nullptr; /* sponge coefficients per column / per row */
    bool has_sc = false;      /* SC_OPTION = 1 child */
    GcScView sc{};            /* its device tables (in sc_block) */
    void *sc_block = nullptr;
    bool sc_stepped = false;  /* after its first sub-step the level-1 buffer holds the reference's Z(:,:,2) */
    float sp_dt = 0.0f;
    int cur = 0;          /* buffer index holding time level 1 */
    bool z2_valid = false; /* level-2 buffer holds the reference's Z(:,:,2) */
    bool mn2_valid = false;
    std::vector<int> children; /* ids in registration order */
    GcLayerDev view() const;
};

struct GcPendingParams {
    bool set = false;
    int laycord = 0, laygov = 0, linchk = 1, modscm = 1, fric_switch = 1;
    float dt = 0, rx = 0, ry = 0, grx = 0, gry = 0, fric_coef = 0;
    std::vector<float> hp, hq;
    std::vector<float> r0, r22; /* per row, from gcomcot_set_layer_coefs_ */
    /* SC_OPTION = 1 tables from gcomcot_set_sc_tables_, [ny][nx][2] and [ny][nx][4] */
    bool sc = false;
    int sc_fix_top = 0, sc_modscm = 1;
    std::vector<int> sc_pos;
    std::vector<float> sc_cxy;
};

struct GcRuntime {
    bool inited = false;
    cudaStream_t stream = nullptr;
    GcLayer layers[GC_MAX_LAYERS];
    GcPendingParams pending[GC_MAX_LAYERS];
    int root = -1;
    /* deferred outer-layer work (fused when the call sequence allows) */
    int pend_mass = 0, pend_open = 0, pend_momt = 0, pend_maxamp = 0;
    int fuse_enabled = 1;
    long long launches = 0;
    /* gauge staging */
    int *d_gauge_ij = nullptr;
    float *d_gauge_out = nullptr;
    float *h_gauge_out = nullptr;
    int gauge_cap = 0;
};

GcRuntime &gc_rt();
GcLayer *gc_layer(int id);
void gc_flush();
void gc_subcycle(int parent_id);
void gc_swap(GcLayer &L);
void gc_root_change_hook(GcLayer &L);
/* arrival tracking of the outer layer is on (gcomcot_set_arrival_) */
bool gc_arrival_on();
/* the fused kernels' descriptor of a layer (both time levels, per-row factors) */
struct GcFusedGrid;
void gc_fill_fused_grid(const GcLayer &L, GcFusedGrid &g);
int gc_layer_alloc(GcLayer &L);
int gc_layer_upload_field(GcLayer &L, float *dst, const float *src_nx_ny);
int gc_layer_download_field(GcLayer &L, const float *src, float *dst_nx_ny);

#endif
