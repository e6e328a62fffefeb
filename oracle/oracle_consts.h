/*
 * Constants of the CPU oracle -- TEST INFRASTRUCTURE.
 *
 * Written from the reference's Fortran, independently of the library's own
 * constants header, so that a wrong constant in the library cannot also sit
 * in the oracle it is checked against.  tests/test_oracle_constants_cpu.py
 * checks both headers against tests/golden/ref_constants.json, which
 * tests/golden/make_ref_constants.py extracts from the Fortran DATA
 * statements themselves.
 *
 *   COMMON /CONS/ BLOCK DATA (comcot.f90:454-470): ELMAX -50.0, GRAV 9.807,
 *     PI 3.14159265358979, R_EARTH 6378000.0, GX 1.0E-5, EPS 1.0E-10,
 *     V_LIMIT 20.0, RAD_DEG 0.01745329252, RAD_MIN 0.000290888208665721
 *   OPEN: DATA UB/99.0/ (boundaries.f90:30)
 *   MOMT_C / CONMOME: DATA TWLVTH/0.08333333333333/ (moment.f90:75,162)
 *   Manning friction exponent DF**(2.3333333) (moment.f90:460,657)
 *   face depth floor DF >= 1.0E-3 (moment.f90:446-448)
 *   WAVE_BREAKING onset 0.08*C and full breaking 0.65*C (moment.f90:1303-1304)
 *   nonlinear buffer width SPAN = 10 (moment.f90:368)
 *   PARA: DATA CORI_W/7.2722E-5/ (comcot.f90:709)
 */
#ifndef ORACLE_CONSTS_H
#define ORACLE_CONSTS_H

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
