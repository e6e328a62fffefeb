/*
 * libgcomcot: B200 (sm_100a) implementation of COMCOT's time-stepping hot
 * path behind the reference GPU-comcot C ABI.
 *
 * Part 1 are the reference's exports, unchanged in name, argument list and
 * meaning (gfortran implicit interface: lower-case name + '_', every argument
 * by reference, arrays as contiguous column-major NX x NY sections).  Like the
 * reference they return nothing and stop the program on a CUDA error.
 * Part 2 are additions a Fortran caller can bind the same way.
 * Part 3 is a plain C API with status returns (0 = ok, < 0 = error).
 */
#ifndef GCOMCOT_H
#define GCOMCOT_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------- Part 1: the reference ABI ---------------- */

/* replaces GPUcomcot.cu:192 gcomcot_init_gpu_ */
void gcomcot_init_gpu_(void);
/* replaces GPUcomcot.cu:214 gcomcot_init_layer_ (R1,R11,R3,R5 read at I=1;
 * R6 is [NY]; R2/R4 are kept as per-row factors when they have the PARA form) */
void gcomcot_init_layer_(int *layerid, int *parent, int *level, int *rel_size, int *rel_time,
                         int *corners, float *grx, float *gry, float *R1, float *R2, float *R3,
                         float *R4, float *R5, float *R6, float *R11, float *H, float *Z, int *nx,
                         int *ny);
/* replaces GPUMass_s.cu:9 mass_launch_ (host arrays unused, as in the reference) */
void mass_launch_(const float *Z1, float *Z2, const float *H, const int *lid);
/* replaces GPUMoment_s.cu:10 momt_launch_ */
void momt_launch_(float *M2, float *N2, float *Z2, const int *lid);
/* replaces GPUOpen_BD.cu:13 openbd_launch_ (outermost layer) */
void openbd_launch_(float *Z2);
/* replaces GPUall_grids.cu:701 all_grid_launch_ (nested sub-cycle) */
void all_grid_launch_(void);
/* replaces GPUOutput.cu:11 maxamp_launch_ */
void maxamp_launch_(const int *lid);
/* replaces GPUcomcot.cu:144 cuda_update_layer_ (time-level rotation) */
void cuda_update_layer_(int *lid);
/* replaces GPUOutput.cu:29 gcomcot_get_z_ (2x2 surface stencil at 1-based i,j) */
void gcomcot_get_z_(int *lid, float *l1, float *l2, float *l3, float *l4, int *i, int *j);
/* replace GPUOutput.cu:55-102 whole-field transfers */
void cuda_getz_(float *Z, int *lid);
void cuda_setz_(float *Z, int *lid);
void cuda_getz1_(float *Z, int *lid);
void cuda_setz1_(float *Z, int *lid);
void cuda_getmn_(float *M, float *N, int *lid);
void cuda_setmn_(float *M, float *N, int *lid);
void cuda_getmn1_(float *M, float *N, int *lid);
void cuda_setmn1_(float *M, float *N, int *lid);
void cuda_getzmax_(float *Zmax, int *lid);
/* replaces GPUall_grids.cu:26 gcomcot_show_grids_ */
void gcomcot_show_grids_(void);
/* replaces GPUcomcot.cu:253 cuda_shutdown_ (the reference's is empty; this frees) */
void cuda_shutdown_(void);
/* replace the DEBUG_CORE comparators GPUall_grids.cu:299 and :626: run the
 * device step and print cells that differ from the caller's arrays by more
 * than the reference tolerance (1e-4) */
void edgeinterp_dbglaunch_(float *mO, float *nO, int *idO, float *mA, float *nA, int *idA, int *t,
                           float *yflux, float *xflux);
void jnz_dbglaunch_(float *Z_f, int *outid, int *inid);

/* ---------------- Part 2: Fortran-callable additions ---------------- */

/* no counterpart in the reference, whose device path treats every layer as
 * linear spherical: coordinate system / equations / Cartesian ratios /
 * friction / HP,HQ of a layer.  Call before gcomcot_init_layer_. */
void gcomcot_set_layer_params_(int *id, int *laycord, int *laygov, float *dt, float *rx, float *ry,
                               float *grx, float *gry, int *fric_switch, float *fric_coef,
                               int *linchk, int *modscm, int *nx, int *ny, float *HP, float *HQ);
/* no counterpart in the reference, whose device path has no nonlinear
 * spherical solver: R0, R21, R22 of PARA (comcot.f90:727-733) for a layer
 * with LAYCORD 0, LAYGOV 1 (CONMASS_S / CONMOME_S); NX x NY arrays read at
 * row I = 1.  Call after gcomcot_set_layer_params_, before
 * gcomcot_init_layer_. */
void gcomcot_set_layer_coefs_(int *id, float *R0, float *R21, float *R22, int *nx, int *ny);
/* no device counterpart in the reference (comcot.f90:403-406 applies
 * SPONGE_LAYER to host arrays): the sponge band of SPONGE_COEF
 * (boundaries.f90:250-345).  COEFX, COEFY are NX x NY fields, COEFX a
 * function of I only and COEFY of J only; DT the layer's step.  Call after
 * gcomcot_init_layer_. */
void gcomcot_set_sponge_(int *id, float *coefx, float *coefy, float *dt, int *nx, int *ny);
/* SPONGE_LAYER (boundaries.f90:206-247) on the device; call after momt_launch_ */
void sponge_launch_(const int *lid);
/* no device counterpart in the reference (its device path couples every
 * child as linear spherical): the SC_OPTION = 1 tables of a Cartesian child
 * of a spherical parent, POS(NX,NY,2) and CXY(NX,NY,4) from
 * SUBGRID_MATCHING (initialization.f90:1065-1124), the parent's MODSCM, and
 * FIX_TOP (1: the top edge blends C2*YN1 instead of the C1*YN1 of
 * all_grids.f90:1357).  Call before gcomcot_init_layer_ of that child. */
void gcomcot_set_sc_tables_(int *id, int *pos, float *cxy, int *nx, int *ny, int *parent_modscm, int *fix_top);
/* no counterpart in the reference: arrival-step tracking on the outer layer
 * (the first outer step after which a wet cell's surface exceeds `thr`; 0 for
 * a wet cell already above it at this call, -1 until then elsewhere).  Call
 * it after gcomcot_init_layer_ of the outer layer. */
void gcomcot_set_arrival_(int *id, float *thr);
void gcomcot_get_arrival_(int *arrival, int *id);

/* ---------------- Part 3: C API ---------------- */

/* kernels launched by the library since initialisation */
long long gcomcot_launch_count(void);
/* 1 (default): fuse mass/open/momentum/max of layer 1 into one kernel */
void gcomcot_set_fusion(int on);
/* waits for queued work; returns 0 or a negative status */
int gcomcot_sync(void);
/* the cudaStream_t the library issues work on */
void *gcomcot_stream(void);
/* no counterpart in the reference (whose kernels never wait on one another):
 * the polls after which a pipeline wait of the two-step kernel gives up,
 * sets the library's error flag and lets its warp leave (default 2^22;
 * <= 0 restores it).  gcomcot_sync / gc_engine_sync then return
 * GC_ETIMEOUT. */
void gcomcot_set_wait_limit(int polls);
/* diagnostics, no counterpart in the reference: the next two-step launch
 * makes its first warp wait for a row that no copy delivers (nothing is
 * issued for it), so the bounded wait above gives up; for tests of the
 * failure path without faulting a GPU */
void gcomcot_inject_stall(void);

/* Runs `nsteps` outer steps through the Part-1 entry points in the order of
 * comcot.f90:359-439 (MASS, OPEN, ALL_GRID, MOMENT, MAX_AMP, GET_TS per
 * gauge, CHANGE).  Gauge g reads layer g_layer[g] at 1-based (g_i, g_j);
 * stencil values go to out4[(k*ngauges + g)*4 + 0..3].  Returns 0 or < 0. */
int gcomcot_drive(int nsteps, int maxamp, int ngauges, const int *g_layer, const int *g_i,
                  const int *g_j, float *out4);

/* ---- on-device source generation (source_okada.cu) ---- */

/* One rectangular fault plane as the reference's FAULT type describes it
 * (type_module.f90:130-147): focal depth to the top edge, length, width and
 * dislocation in metres; strike, dip and slip (rake) in degrees; epicentre
 * longitude/latitude; the origin of a Cartesian layer; sw = 0 puts the
 * epicentre at the plane's centre, 9 at the centre of its top edge. */
typedef struct {
    double hh, l, w, d;
    double th, dl, rd;
    double x0, y0;
    double xo, yo;
    int sw;
} gc_fault;

/* replaces deform.f90:2-240 (GET_FLOOR_DEFORM with DEFORM_OKADA for
 * instantaneous faults): adds each fault's seafloor deformation to the
 * surface d_z and subtracts it from the depth d_h (device arrays, row pitch
 * `pitch` floats; either may be NULL), in fault order.  laycord 0: cell
 * positions from the device axes d_x[nx] (longitude) and d_y[ny] (latitude);
 * 1: from the spacings dx, dy in metres.  Returns 0 or < 0. */
int gc_okada_apply(const gc_fault *faults, int nf, int laycord, int nx, int ny, int pitch, const float *d_x,
                   const float *d_y, float dx, float dy, float *d_z, float *d_h, void *stream);

/* ---- batched ensemble / serving engine (engine.cu) ---- */
typedef struct gc_engine gc_engine;

/* A grid class: bathymetry and per-row coefficients shared by all members.
 * rows is [7][ny]: R1(1,J), R11(1,J), R6(J), R3(1,J), R5(1,J), CX(J), CY(J)
 * with R2 = CX(J)*max(HP,0), R4 = CY(J)*max(HQ,0) (comcot.f90:713-752). */
int gc_engine_create(long long hbm_budget_bytes, gc_engine **out);
int gc_engine_destroy(gc_engine *e);
int gc_engine_add_class(gc_engine *e, int nx, int ny, const float *H, const float *rows);
/* a member (scenario / request) on class `cls`: initial surface z0 [nx*ny],
 * nsteps to run, gauges (1-based KI,KJ and weights CX,CY), arrival threshold
 * (< 0 disables).  Returns the member id (>= 0) or a negative status; fails
 * with -2 when the budget has no room. */
int gc_engine_add_member(gc_engine *e, int cls, const float *z0, int nsteps, int ngauges,
                         const int *gij, const float *gw, float arrival_thr);
/* advances every active member by up to `nsteps` steps (members stop at
 * their own step count); returns the number of steps issued or < 0 */
int gc_engine_step(gc_engine *e, int nsteps);
/* 1 once the member has run all its steps (after gc_engine_sync) */
int gc_engine_member_done(gc_engine *e, int member);
/* outer steps the member has been issued so far (complete after
 * gc_engine_sync); gc_engine_read returns the state after that many steps */
int gc_engine_member_steps(gc_engine *e, int member);
int gc_engine_sync(gc_engine *e);
/* 1 when all work issued so far has finished, 0 while it runs (does not
 * wait; gc_engine_sync still reports errors) */
int gc_engine_query(gc_engine *e);
/* results of a member: any pointer may be NULL */
int gc_engine_read(gc_engine *e, int member, float *z, float *m, float *n, float *zmax,
                   int *arrival, float *ts);
int gc_engine_release(gc_engine *e, int member);
/* the same results copied asynchronously, queued on the engine's stream
 * behind the member's issued steps, into host memory the caller owns (from
 * gc_host_alloc, so the copies do not stall the host); *done receives an event
 * that completes with the copies (gc_event_query / gc_event_wait, then
 * gc_event_release).  The member may be released right after: its storage is
 * freed in stream order, behind the copies. */
int gc_engine_read_async(gc_engine *e, int member, float *z, float *m, float *n, float *zmax,
                         int *arrival, float *ts, void **done);
/* 1 when the event completed, 0 while pending, < 0 on error */
int gc_event_query(void *event);
int gc_event_wait(void *event);
int gc_event_release(void *event);
/* page-locked host memory for asynchronous reads (NULL when refused) */
void *gc_host_alloc(long long bytes);
int gc_host_free(void *p);

/* A nested grid class: the outer grid of class `parent_cls` with one child
 * layer (ALL_GRID sub-cycle, all_grids.f90:4-312).
 * corners = IS, IE, JS, JE in the outer grid (1-based, at least 4 cells from
 * its edge); nx = (IE-IS+1)*rel_size+1, ny likewise.  laycord/laygov select
 * the child's solver: (1,1) CONMASS/CONMOME with wet/dry and Manning
 * friction, (1,0) MASS_C/MOMT_C, (1,2|3) MASS_C_D/MOMT_C_D, (0,0)
 * MASS_S/MOMT_S, (0,1) CONMASS_S/CONMOME_S, (0,2) MASS_S_D/MOMT_S_D; a
 * spherical child needs `rows`, its [7][ny] block (R1, R11, R6, R3, R5, R2
 * and R4 per row), and a nonlinear spherical one also `rows2`, [2][ny]
 * (R0, R22 per row).  hp/hq may be NULL (then PQ_DEPTH of h).
 * SC_OPTION = 1 (a Cartesian child coupled through the UTM tables,
 * all_grids.f90:996-1425): sc_pos [ny][nx][2] 1-based (KI, KJ) and sc_cxy
 * [ny][nx][4] as SUBGRID_MATCHING builds them, corners their extent (nx, ny
 * then need not follow the corners), sc_fix_top and parent_modscm as in
 * gcomcot_set_sc_tables_; members of such a class start from a flat child
 * surface.  Members of a nested class step with the per-phase kernels. */
typedef struct {
    int nx, ny;
    int corners[4];
    int rel_size, rel_time;
    int laycord, laygov, linchk, modscm, fric_switch;
    float dt, rx, ry, grx, gry, fric_coef;
    const float *h, *hp, *hq, *rows;
    const float *rows2;
    const int *sc_pos;
    const float *sc_cxy;
    int sc_fix_top, parent_modscm;
} gc_child_desc;
int gc_engine_add_nested_class(gc_engine *e, int parent_cls, const gc_child_desc *child);
/* a member of a nested class: child_z0 may be NULL (still water); gauge g
 * reads layer glayer[g] (0 outer grid, 1 child; NULL = all outer) at
 * 1-based gij of that layer */
int gc_engine_add_nested_member(gc_engine *e, int cls, const float *z0, const float *child_z0, int nsteps,
                                int ngauges, const int *glayer, const int *gij, const float *gw,
                                float arrival_thr);
/* the child's Z, M, N (level 1 after the member's completed steps) */
int gc_engine_read_child(gc_engine *e, int member, float *z, float *m, float *n);
/* longitude [nx] and latitude [ny] axes of a (non-nested) class, in degrees,
 * needed by members created from fault parameters */
int gc_engine_set_class_axes(gc_engine *e, int cls, const float *lon, const float *lat);
/* a member whose initial state comes from faults on the device: still water
 * plus the seafloor deformation (gc_okada_apply), with its own depth H minus
 * the deformation (the reference's UPDATE_BATH, initialization.f90:2410-2434) */
int gc_engine_add_member_faults(gc_engine *e, int cls, const gc_fault *faults, int nfaults, int nsteps,
                                int ngauges, const int *gij, const float *gw, float arrival_thr);
/* no counterpart in the reference (which has no failure detection): scans
 * the member's max-eta and current surfaces; 0 = healthy, bit 0 = a NaN or
 * Inf appeared, bit 1 = |eta| exceeded `bound` metres, < 0 = error */
int gc_engine_member_health(gc_engine *e, int member, float bound);
long long gc_engine_bytes_in_use(gc_engine *e);
long long gc_engine_member_bytes(gc_engine *e, int cls);
/* tile variant (autotuned when < 0; v + gc_engine_num_variants() * r also
 * picks tile-height rule r) and use of CUDA graphs for step chunks */
int gc_engine_config(gc_engine *e, int variant, int use_graphs, int graph_chunk);
int gc_engine_autotune(gc_engine *e, int reps);
/* builds the work list and the step-chunk graph for the current members
 * ahead of the next gc_engine_step (otherwise the first chunk pays for them) */
int gc_engine_prepare(gc_engine *e);
int gc_engine_variant(gc_engine *e);
/* number of compiled tile variants (all compute identical results) */
int gc_engine_num_variants(void);
/* candidates gc_engine_autotune times, one step set each: variants x tile-height rules */
int gc_engine_num_candidates(void);
long long gc_engine_launches(gc_engine *e);
/* the cudaStream_t the engine issues its kernels on */
void *gc_engine_stream(gc_engine *e);
/* the two-step kernel's tile layout of an nx x ny grid at tile height ty
 * under tile-height rule `rule` (0, 1: uniform; 2: balanced): returns the
 * number of tiles; with 0 <= lt < that number, out5 = {first column of the
 * tile's 128-column strip, first and last stored column, first output row,
 * rows} of tile lt (rows past the grid's last are not stored).  Host-only
 * (no device work); the kernel runs the same code. */
int gc_pair_layout_tile(int nx, int ny, int ty, int rule, int lt, int *out5);

/* ---- one fused step without any allocation (noalloc.cu) ---- */

/* one grid of gcomcot_fused_step_noalloc: device arrays the caller owns,
 * row-pitched (element (i,j) at p[j*pitch + i], pitch a multiple of 32 floats,
 * every array 16-byte aligned).  rows is [ny][8]: R1(1,J), R11(1,J), R6(J),
 * R3(1,J), R5(1,J), CX(J), CY(J), unused -- R2 = CX*max(HP,0), R4 = CY*max(HQ,0). */
typedef struct {
    int nx, ny, pitch;
    const float *z1, *m1, *n1; /* time level 1, read */
    float *z2, *m2, *n2;       /* time level 2, written */
    const float *h;            /* still-water depth */
    const float *rows;         /* per-row coefficient records */
    float *zmax;               /* running maximum, updated in place; NULL to skip */
} gc_grid_step_io;

/* No counterpart in the reference.  For callers that cannot allocate device
 * memory (codes that own all device memory, pipelines with a fixed reserved
 * budget, loops where an allocation's device synchronisation is not
 * acceptable): one outer step (MASS_S + OPEN + MOMT_S + max) of every grid in
 * one launch on `stream`, with its work list in a fixed array built into the
 * library (at most 64 grids and 24576 tiles of 128 columns; larger requests
 * return -1).  The grid list travels in the launch parameters of a small
 * kernel that fills the array, so nothing is copied from host memory and the
 * call returns once its work is queued.  Calls share that array: calls that
 * overlap on the GPU race.  The first call on a device does a one-time set-up
 * and should come before any stream capture.  A bounded pipeline wait that
 * gives up is reported by gcomcot_sync() (GC_ETIMEOUT) after the caller has
 * synchronised `stream`.  Returns 0 or a negative status. */
int gcomcot_fused_step_noalloc(int ngrids, const gc_grid_step_io *grids, void *stream);

#ifdef __cplusplus
}
#endif

#endif
