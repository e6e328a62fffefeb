/*
 * Internal definitions of the B200 COMCOT library: device layer view, row
 * coefficient layout, launch helpers and error plumbing.
 *
 * Device layout of one layer (Fortran (I,J) -> 0-based (i,j) = (I-1,J-1)):
 *   every NX x NY field is stored row-pitched, I fastest, with the row
 *   pitch rounded up to 32 floats (128 B) so every row starts on a 128-byte
 *   boundary; element (i,j) is at p[j*pitch + i].
 *   Z, M, N are ping-pong pairs; `cur` names the buffer holding time level 1
 *   (the reference's Zdat/MNdat), the other holds level 2 (Zout/MNout).
 *   Per-row coefficients live in one [ny][GC_ROWW] array (see GcRow): the
 *   eight floats of a row are contiguous, 32 bytes, so one bulk copy
 *   fetches them.
 */
#ifndef GC_INTERNAL_H
#define GC_INTERNAL_H

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include "comcot_consts.h"
#include "comcot_math.h"

#define GC_MAX_LAYERS 20

/* rows of the per-row coefficient block: R1(1,J), R11(1,J), R6(J),
 * R3(1,J), R5(1,J) from PARA (comcot.f90:713-752), and the factored
 * R2 = CX(J)*max(HP,0), R4 = CY(J)*max(HQ,0) multipliers. */
enum GcRow { GC_R1 = 0, GC_R11, GC_R6, GC_R3, GC_R5, GC_CX, GC_CY, GC_NROW };
#define GC_ROWW 8 /* floats per row record (7 used, 1 pad) */

/* What a kernel needs to know about one layer.  Passed by value. */
struct GcLayerDev {
    int nx, ny, pitch;
    int root;          /* 1 for the outermost layer (reference layer id 1) */
    int laycord, laygov, linchk, modscm, fric_switch;
    int explicit_r24;  /* 1: R2/R4 stored as fields; 0: factored per row */
    float rx, ry, grx, gry, dt, fric_coef;
    const float *z1, *m1, *n1;   /* time level 1 */
    float *z2, *m2, *n2;         /* time level 2 */
    float *m1w, *n1w;            /* writable alias of level 1 (nesting edges) */
    float *z1w;
    const float *h, *hp, *hq;
    const float *r2, *r4;        /* only when explicit_r24 */
    const float *rows;           /* [ny][GC_ROWW] */
    const float *rows2;          /* [ny][2] R0, R22 (nonlinear spherical layers) */
    float *dz2;                  /* nonlinear layers */
    float *xflux, *yflux;        /* [2*nx], [2*ny] forecast caches */
    float *zmax;
    int *arrival;
};

#define GC_AT(p, L, i, j) ((p)[(size_t)(j) * (size_t)(L).pitch + (size_t)(i)])
#define GC_ROW(L, k, j) ((L).rows[(size_t)(j) * GC_ROWW + (size_t)(k)])

/* status codes of the extended API */
#define GC_OK 0
#define GC_EINVAL -1
#define GC_ENOMEM -2
#define GC_ECUDA -3
#define GC_ESTATE -4
#define GC_ETIMEOUT -5
#define GC_ENOTSUP -6

const char *gc_status_str(int code);

#define GC_CUDA_OR_RET(call)                                                       \
    do {                                                                           \
        cudaError_t e_ = (call);                                                   \
        if (e_ != cudaSuccess) {                                                   \
            fprintf(stderr, "gcomcot: %s at %s:%d\n", cudaGetErrorString(e_),      \
                    __FILE__, __LINE__);                                           \
            return GC_ECUDA;                                                       \
        }                                                                          \
    } while (0)

/* legacy entry points mirror the reference: print and exit on a CUDA error */
#define GC_CUDA_OR_DIE(call)                                                       \
    do {                                                                           \
        cudaError_t e_ = (call);                                                   \
        if (e_ != cudaSuccess) {                                                   \
            fprintf(stderr, "gcomcot: %s in %s at line %d\n",                      \
                    cudaGetErrorString(e_), __FILE__, __LINE__);                   \
            exit(EXIT_FAILURE);                                                    \
        }                                                                          \
    } while (0)

/* ---- per-phase kernels (kernels_phase.cu) ---- */
/* launches from this host thread use programmatic dependent launch */
void gc_set_pdl(bool on);
bool gc_pdl_on();
/* programmatic dependent launch for the launches in a scope */
struct GcPdlScope {
    bool prev;
    explicit GcPdlScope(bool on) : prev(gc_pdl_on()) { gc_set_pdl(on); }
    ~GcPdlScope() { gc_set_pdl(prev); }
};
void gc_launch_mass(const GcLayerDev &L, cudaStream_t s);
void gc_launch_open(const GcLayerDev &L, cudaStream_t s);
void gc_launch_moment(const GcLayerDev &L, cudaStream_t s);
/* linear spherical momentum over the 0-based cells [i0,i1] x [j0,j1] only */
void gc_launch_momt_s_window(const GcLayerDev &L, int i0, int i1, int j0, int j1, cudaStream_t s);
void gc_launch_update_edges(const GcLayerDev &L, cudaStream_t s);
/* a child's momentum followed by UPDATE's edge copy; the copy rides in the
 * momentum launch where that is safe.  Returns the launches issued. */
int gc_launch_moment_update(const GcLayerDev &L, cudaStream_t s);
void gc_launch_edges(const GcLayerDev &P, const GcLayerDev &C, int rel_size, int rel_time,
                     const int *corners, int t, cudaStream_t s);
void gc_launch_jnz(const GcLayerDev &P, const GcLayerDev &C, int rel_size, int rel_time,
                   const int *corners, cudaStream_t s);
/* JNQ at sub-step t together with a Cartesian child's MASS_C / CONMASS, in
 * one launch; false (nothing launched) where that form does not apply (t > 1,
 * other child kinds): then call gc_launch_edges and gc_launch_mass */
bool gc_launch_edges_mass(const GcLayerDev &P, const GcLayerDev &C, int rel_size, int rel_time,
                          const int *corners, int t, cudaStream_t s);
/* SC_OPTION = 1 coupling of a Cartesian child to a spherical parent: the
 * parent cell (KI, KJ) and bilinear weights of every child edge node, and
 * for JNZ_SC, per parent cell of the child's window, the child nodes that
 * fall in it (CSR, in the reference's summation order) */
struct GcScView {
    const int2 *epos;    /* [2*ny + 2*nx] 1-based (KI, KJ): left, right, bottom, top edge nodes */
    const float4 *ew;    /* [2*ny + 2*nx] weights of (KI,KJ), (KI+1,KJ), (KI,KJ+1), (KI+1,KJ+1) */
    const int *start;    /* [(wi1-wi0+1)*(wj1-wj0+1) + 1] */
    const int *cell;     /* child offsets j*pitch + i */
    int wi0, wi1, wj0, wj1; /* parent window, 0-based inclusive */
    int band[4][4];      /* forecast bands i0, i1, j0, j1 (0-based): left M, right M, top N, bottom N */
    int fix_top;         /* 1: top edge blends C2*YN1 (the reference uses C1*YN1) */
    int modscm;          /* the parent's MODSCM (0 adds the modified-scheme term) */
    float half;          /* REL_SIZE**2 / 2 */
};
const char *gc_sc_tables(int nx, int ny, int cpitch, const int *pos, const float *cxy, const int corners[4],
                         int pnx, int pny, int rel_size, int fix_top, int modscm, GcScView *out, void **block,
                         size_t *bytes);
void gc_launch_sc_edges(const GcLayerDev &P, const GcLayerDev &C, const GcScView &sv, int t, int rel_time,
                        const float *zwet, cudaStream_t s);
void gc_launch_sc_forecast(const GcLayerDev &P, const GcScView &sv, cudaStream_t s);
void gc_launch_sc_jnz(const GcLayerDev &P, const GcLayerDev &C, const GcScView &sv, cudaStream_t s);
void gc_launch_maxamp(const GcLayerDev &L, cudaStream_t s);
void gc_launch_sponge(const GcLayerDev &L, const float *spx, const float *spy, float dt, cudaStream_t s);
/* arrival at the start of tracking: 0 on a wet cell already above `thr`, -1 elsewhere */
void gc_launch_arrival_start(int *arrival, const float *z, const float *h, int nx, int ny, int pitch, float thr,
                             cudaStream_t s);
void gc_launch_arrival(const GcLayerDev &L, int step, float thr, cudaStream_t s);
void gc_launch_gauges(const GcLayerDev &L, int ng, const int *d_ij, float *d_out, cudaStream_t s);
/* max-eta (flags & 1), arrival (flags & 2) and gauge samples after one outer
 * step of a batched nested member; step = step_off + *step_base; max/arrival
 * over the 0-based window win = {i0, i1, j0, j1} (NULL: the whole layer) */
void gc_launch_step_outputs(const GcLayerDev &L, const int *step_base, int step_off, int step0, int flags,
                            float thr, int ng, const int *gij, const float *gw, const int *glayer,
                            const float *cz, int cpitch, float *ts, int ts_len, const int *win, cudaStream_t s);
/* JNZ (window `corners`, 1-based IS, IE, JS, JE), the linear spherical
 * momentum over the 0-based rectangle rect = {i0, i1, j0, j1} and the
 * outputs of gc_launch_step_outputs over the JNZ window, in one launch;
 * false (nothing launched) for a ratio it is not built for */
bool gc_launch_feedback(const GcLayerDev &P, const GcLayerDev &C, int rel_size, int rel_time, const int *corners,
                        const int *rect, const int *step_base, int step_off, int step0, int flags, float thr, int ng,
                        const int *gij, const float *gw, const int *glayer, const float *cz, int cpitch, float *ts,
                        int ts_len, cudaStream_t s);

/* ---- fused step (kernels_fused.cu) ---- */
struct GcFusedGrid;
struct GcTile;

#endif
