/*
 * CPU oracle for the COMCOT time-stepping hot path -- TEST INFRASTRUCTURE.
 *
 * This is a plain-C restatement of the reference Fortran solvers.  It exists
 * only to check the CUDA library: tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline / --impl reference legs load it; the product never
 * does.  It is built twice from the same source, with REAL = float (the
 * reference's default REAL arithmetic) and REAL = double (the FP64 twin used
 * to state the float error per configuration).
 *
 * Parity pin: the reference ships no golden vectors or fixtures.  The FP32
 * build is pinned against outputs of the reference's own CUDA kernels
 * compiled from their sources and run on a B200 (tests/golden/, made by
 * oracle/make_ref_goldens.py), for the stencils where the reference GPU path
 * and the Fortran agree; see the header of that script for the cases.
 *
 * Index convention: Fortran (I,J), 1-based, column-major, I fastest:
 * element (I,J) of an NX x NY field is a[(J-1)*NX + (I-1)].
 */
#ifndef COMCOT_ORACLE_H
#define COMCOT_ORACLE_H

#ifndef REAL
#define REAL float
#endif

typedef struct {
    int id, parent, level, nx, ny;
    int laycord;      /* 0 spherical, 1 Cartesian              (type_module.f90:93) */
    int laygov;       /* 0 linear, 1 nonlinear                 (type_module.f90:94) */
    int linchk;       /* 1: convection terms on                (comcot.f90:541-549) */
    int modscm;       /* 0: modified scheme (root linear only) (comcot.f90:545-551,601) */
    int fric_switch;  /* 0 constant Manning, 1 no friction     (type_module.f90:64) */
    int rel_size, rel_time;
    int corners[4];   /* IS, IE, JS, JE in the parent           (type_module.f90:99) */
    double dt, rx, ry, grx, gry, fric_coef;
    REAL *r1, *r11, *r6, *r3, *r5;        /* [ny] per-row spherical coefficients */
    REAL *r0, *r22;                       /* [ny] nonlinear spherical advection (PARA, comcot.f90:727-733) */
    REAL *r2, *r4;                        /* [nx*ny] */
    REAL *h, *hp, *hq;                    /* [nx*ny] */
    REAL *z1, *z2, *m1, *m2, *n1, *n2;    /* [nx*ny] time levels 1 and 2 */
    REAL *dz2;                            /* [nx*ny] DZ(:,:,2); DZ(:,:,1) is always 0 */
    REAL *xflux, *yflux;                  /* [2*nx], [2*ny] nesting forecast caches */
    REAL *zmax;                           /* [nx*ny] or NULL */
    int  *arrival;                        /* [nx*ny] or NULL */
    REAL *spx, *spy;                      /* [nx*ny] SPONGE_COEFX/Y of the outer layer, or NULL */
    int sc_option;                        /* 1: Cartesian child coupled through POS/CXY (SC_OPTION = 1) */
    int sc_fix_top;                       /* 1: top edge blends C2*YN1 instead of the reference's C1*YN1 */
    int *pos;                             /* [ny][nx][2] 1-based (KI, KJ) in the parent, SC_OPTION = 1 */
    REAL *cxy;                            /* [ny][nx][4] bilinear weights, SC_OPTION = 1 */
} ocl_layer;

void ocl_set_threads(int n);
int  ocl_get_threads(void);

void ocl_mass(ocl_layer *L);
void ocl_moment(ocl_layer *L);
void ocl_open(ocl_layer *L);
void ocl_change(ocl_layer *L);
void ocl_update(ocl_layer *L);
void ocl_jnq(ocl_layer *P, ocl_layer *C);
void ocl_newq(ocl_layer *P, ocl_layer *C, int t);
void ocl_jnz(ocl_layer *P, ocl_layer *C);
/* SC_OPTION = 1 coupling (all_grids.f90:996-1425) */
void ocl_edge_sc(ocl_layer *P, ocl_layer *C);
void ocl_newq_sc(ocl_layer *P, ocl_layer *C, int t);
void ocl_jnz_sc(ocl_layer *P, ocl_layer *C);
void ocl_maxamp(ocl_layer *L);
/* SPONGE_LAYER (boundaries.f90:206-247): after the momentum step */
void ocl_sponge(ocl_layer *L);
/* SPONGE_COEF with H_CALC (boundaries.f90:250-385): coefficient fields of a
 * layer with axes x[nx], y[ny] (degrees, or metres for laycord 1) */
void ocl_sponge_coef(int nx, int ny, int laycord, const REAL *x, const REAL *y, const REAL *h, REAL *coefx,
                     REAL *coefy);
void ocl_arrival_start(ocl_layer *L, double thr);
void ocl_arrival(ocl_layer *L, int step, double thr);
void ocl_all_grid(ocl_layer *layers, int n);
void ocl_step(ocl_layer *layers, int n, int step, double arrival_thr);
double ocl_gauge(ocl_layer *L, int ki, int kj, double cx, double cy);
/* outer steps first .. first + nsteps - 1 (continues an earlier run) */
int  ocl_run_from(ocl_layer *layers, int n, int first, int nsteps, double arrival_thr, int ngauges,
                  const int *g_layer, const int *g_ki, const int *g_kj, const double *g_cx,
                  const double *g_cy, REAL *ts);
int  ocl_run(ocl_layer *layers, int n, int nsteps, double arrival_thr,
             int ngauges, const int *g_layer, const int *g_ki, const int *g_kj,
             const double *g_cx, const double *g_cy, REAL *ts);

void ocl_pq_depth(int nx, int ny, const REAL *h, REAL *hp, REAL *hq);
void ocl_para(int nx, int ny, int laygov, double dt, double dx_min,
              const double *lat, const double *del_y_min, const REAL *hp, const REAL *hq,
              REAL *r1, REAL *r11, REAL *r2, REAL *r3, REAL *r4, REAL *r5, REAL *r6);
/* R0 and R22 of PARA (comcot.f90:727,733) per row */
void ocl_para_nl(int ny, double dt, double dx_min, const double *lat, const double *del_y_min, REAL *r0,
                 REAL *r22);
int  ocl_rel_time(double dt_parent, double dx_m, double dy_m, double hmax, int nonlinear,
                  double *dt_child);
void ocl_corners(int nx_p, const double *xp, int ny_p, const double *yp,
                 double xs, double xe, double ys, double ye, int *corners);

/* one rectangular fault plane (type_module.f90:130-147); angles in degrees,
 * lengths in metres, positions in degrees */
typedef struct {
    double hh, l, w, d;       /* focal depth to the top edge, length, width, dislocation */
    double th, dl, rd;        /* strike, dip, slip (rake) */
    double x0, y0;            /* epicentre longitude, latitude */
    double xo, yo;            /* domain origin (Cartesian layers) */
    int sw;                   /* 0: epicentre at the plane's centre; 9: at its top edge's centre */
} ocl_fault;

/* DEFORM_OKADA (deform.f90:74-187) for every cell of a layer: laycord 0 uses
 * the longitudes x[nx] / latitudes y[ny], laycord 1 the spacings dx, dy */
void ocl_okada(const ocl_fault *f, int laycord, int nx, int ny, const double *x, const double *y, double dx,
               double dy, REAL *deform);
/* GET_FLOOR_DEFORM (deform.f90:2-72) for instantaneous faults: per fault,
 * Z += DEFORM and H -= DEFORM, in fault order */
void ocl_okada_apply(const ocl_fault *f, int nf, int laycord, int nx, int ny, const double *x, const double *y,
                     double dx, double dy, REAL *z, REAL *h);
void ocl_stereo(REAL lonin, REAL latin, REAL lon0, REAL lat0, REAL *xo, REAL *yo);

float ocl_expf(float x);
float ocl_powf(float x, float y);

#endif
