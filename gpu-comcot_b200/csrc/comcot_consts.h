/*
 * Physical and numerical constants of the COMCOT time stepper.
 *
 * Values are the single-precision constants of the reference's COMMON /CONS/
 * block (comcot.f90:454-470, BLOCK DATA) and of the routines' DATA statements:
 *   ELMAX = -50, GRAV = 9.807, GX = 1e-5, EPS = 1e-10, V_LIMIT = 20,
 *   R_EARTH = 6378000, RAD_DEG = 0.01745329252, RAD_MIN = 2.90888208665721e-4
 *   UB = 99 (boundaries.f90:30), CORI_W = 7.2722e-5 (comcot.f90:708),
 *   TWLVTH = 0.08333333333333 (moment.f90:160), wave-breaking onset 0.08
 *   and full 0.65 of sqrt(g*d) (moment.f90:1302-1305),
 *   Manning exponent 2.3333333 (moment.f90:460).
 * Every comparison in the kernels uses these float values, so thresholds
 * decide exactly as the Fortran REAL arithmetic does.
 */
#ifndef COMCOT_CONSTS_H
#define COMCOT_CONSTS_H

#define CC_ELMAX    (-50.0f)
#define CC_GRAV     (9.807f)
#define CC_GX       (1.0e-5f)
#define CC_EPS      (1.0e-10f)
#define CC_VLIMIT   (20.0f)
#define CC_UB       (99.0f)
#define CC_TWLVTH   (0.08333333333333f)
#define CC_MANNEXP  (2.3333333f)
#define CC_DFMIN    (1.0e-3f)
#define CC_BRK_F    (0.08f)
#define CC_BRK_I    (0.65f)
#define CC_SPAN     10

#define CC_R_EARTH  6378000.0
#define CC_RAD_DEG  0.01745329252
#define CC_RAD_MIN  0.000290888208665721
#define CC_CORI_W   7.2722e-5
#define CC_PI       3.14159265358979

#endif
