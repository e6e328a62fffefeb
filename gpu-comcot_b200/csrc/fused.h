/*
 * Descriptor of one grid in the fused linear-spherical step and in the
 * batched work-list launch (ensemble members, serving slots).
 */
#ifndef GC_FUSED_H
#define GC_FUSED_H

#include "gc_internal.h"

#define GC_F_MAXAMP 1
#define GC_F_ARRIVAL 2
/* arrival decided from max-eta (set by the engine, whose members record
 * max-eta every step and start arrival at 0 where the initial surface is
 * already above the threshold on a wet cell) */
#define GC_F_ARR_BYMAX 4
/* two-step kernel: gauge records are the raw 2x2 surface stencils (four
 * values per gauge and step, as gcomcot_get_z_ returns them) instead of the
 * GET_TS bilinear value */
#define GC_F_STENCIL 8

struct GcFusedGrid {
    int nx, ny, pitch, root, explicit_r24;
    int tiles_x;      /* tiles along I (128 columns each) */
    int ty;           /* rows per tile */
    int step0, cur0;  /* at step `step0`, buffer `cur0` holds time level 1 */
    int nsteps;       /* steps this grid runs; the step after the last only samples gauges */
    int flags;        /* GC_F_MAXAMP | GC_F_ARRIVAL */
    float thr;        /* arrival threshold */
    /* time levels: nbuf 2 (or 0): level L of the window in buffer cur0 ^ (L & 1);
     * nbuf 3: level L in buffer L % 3 (the engine's single-grid members, which
     * the two-step kernel also steps) */
    int nbuf;
    /* two-step kernel: tiles along I, rows per tile, and rows per tile of
     * the edge strips and of the other strips' first and last tile rows (0:
     * every tile pty rows) */
    int ptiles_x, pty, pte;
    float *z[3], *m[3], *n[3];
    const float *h, *rows, *r2, *r4;
    float *zmax;
    int *arrival;
    /* gauges: the step-s kernel samples the surface left by step s-1 into
     * ts[(s-1-step0)*ng + g] (bilinear, GET_TS weights) when s-1 >= step0 */
    int ng;
    const int *gij;     /* [2*ng] 1-based (KI, KJ) */
    const float *gw;    /* [2*ng] (CX, CY) */
    float *ts;
    int ts_len;         /* steps the ts buffer can hold */
    /* when has_win: cells [wi0,wi1] x [wj0,wj1] (0-based, inclusive) get no
     * max-eta or arrival update, since a nested child's feedback rewrites
     * their surface after this launch (zero-filled descriptors have none) */
    int has_win, wi0, wi1, wj0, wj1;
};

/* one launch variant: warps per CTA and pipeline stages per warp */
struct GcTileCfg {
    int warps, stages;
};

int gc_fused_num_variants();
GcTileCfg gc_fused_variant(int v);
/* rows per tile for a work list of grids (nx[k], ny[k]); rule 0: the
 * shortest tiles that keep the wave count of 16-row tiles, rule 1: the
 * height that minimises the busiest warp's rows (the autotuner tries both) */
constexpr int GC_TY_RULES = 2;
int gc_fused_pick_ty(int variant, int ngrids, const int *nx, const int *ny, int rule = 0, bool multi = true);
/* launches the fused step over a work list: tiles[t] = {grid, tile within
 * that grid}; step = *step_base + step_off (step_base may be NULL) */
cudaError_t gc_fused_launch_multi(int variant, const GcFusedGrid *d_grids, const int2 *d_tiles,
                                  int ntiles, const int *d_step_base, int step_off, int nctas,
                                  cudaStream_t s);
/* resident CTAs on the device: of the work-list kernel (multi) or of the
 * single-grid kernel */
int gc_fused_max_ctas(int variant, bool multi = true);
/* 1 if a pipeline wait in the fused kernel gave up since the last call (clears it) */
int gc_fused_take_error();
/* clears that flag in stream order on `s` */
cudaError_t gc_fused_clear_error_async(cudaStream_t s);
/* single grid, descriptor by value */
cudaError_t gc_fused_launch_one(int variant, const GcFusedGrid &g, int step, cudaStream_t s);
/* single grid at step step_off + *d_step_base (d_step_base may be NULL) */
cudaError_t gc_fused_launch_one_at(int variant, const GcFusedGrid &g, const int *d_step_base, int step_off,
                                   cudaStream_t s);
int gc_fused_tiles(int nx, int ny, int ty, int *tiles_x);

/* ---- two steps per launch (kernels_pair.cu): grids with nbuf 3, the
 * outermost layer only, factored R2/R4, max-eta on, arrival by max-eta,
 * at most 64 gauges; both steps inside every grid's window ---- */
int gc_pair_num_variants();
GcTileCfg gc_pair_variant(int v);
/* tiles of one grid: strip t stores columns [120t+4, 120t+123] (the first
 * [0, 123], the last to the grid's edge); tiles are ty rows, except that
 * with te > 0 the two edge strips take te-row tiles, and so do the other
 * strips' first and last tile rows (te == 0: every tile ty rows) */
int gc_pair_tiles(int nx, int ny, int ty, int te, int *tiles_x);
/* pair tile-height rules: 0 and 1 uniform (1: at least 24 rows), 2 the
 * balanced layout (shorter tiles where the boundary makes rows dearer) */
constexpr int GC_PAIR_RULES = 3;
int gc_pair_short_ty(int rule, int ty);
int gc_pair_max_ctas(int variant, bool multi = true);
int gc_pair_pick_ty(int variant, int ngrids, const int *nx, const int *ny, int rule, bool multi = true);
/* A class launch of the two-step kernel: members of one grid class (same
 * geometry, row records and tile layout) stepped by one launch whose member
 * table is a kernel parameter, so a tile's member and its buffers derive from
 * the block index and the parameter bank alone (warp-uniform values) instead
 * of a descriptor loaded from memory.  Tiles are member-minor: tile t is
 * member t % nm, class tile t / nm. */
constexpr int GC_PAIR_CLASS_MAX = 64;
struct GcPairMember {
    float *z[3], *m[3], *n[3];
    float *zmax;
    int *arrival;
    const float *h;
    const int *gij;
    const float *gw;
    float *ts;
    int step0, nsteps, flags, ng, ts_len;
    float thr;
};
struct GcPairClass {
    GcFusedGrid proto; /* the geometry; its member fields are not read */
    int nm, ntiles;    /* members, tiles per member */
    GcPairMember m[GC_PAIR_CLASS_MAX];
};
cudaError_t gc_pair_launch_class(int variant, const GcPairClass &c, const int *d_step_base, int step_off,
                                 cudaStream_t s);
/* steps (*d_step_base + step_off) and the next one */
cudaError_t gc_pair_launch_one_at(int variant, const GcFusedGrid &g, const int *d_step_base, int step_off,
                                  cudaStream_t s);
cudaError_t gc_pair_launch_multi(int variant, const GcFusedGrid *d_grids, const int2 *d_tiles, int ntiles,
                                 const int *d_step_base, int step_off, cudaStream_t s);
/* 1 if a pipeline wait of the two-step kernel gave up since the last call (clears it) */
int gc_pair_take_error();
/* polls before a pipeline wait of the two-step kernel gives up (default 2^22) */
void gc_pair_set_wait_limit(int polls);
/* the next two-step launch makes its first warp wait for a row nothing
 * delivers (no copy is issued for it): the bounded wait then gives up */
void gc_pair_stall_next();

#endif
