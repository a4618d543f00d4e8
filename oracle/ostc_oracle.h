/*
 * ostc_oracle.h -- CPU restatement (serial FP64, plain C) of OpenSTC's per-step right-hand side and
 * SSP-RK3 update for calorically perfect air.  TEST INFRASTRUCTURE ONLY: the parity tests, the smoke
 * check and the CPU-baseline leg of bench.py call it as the checker; the product never links it.
 *
 * Each routine cites the reference file:line it restates (paths relative to the OpenSTC-MixingLayer
 * source tree).  The oracle keeps the reference's memory layout (ghost-padded SoA, k-ghost layers
 * even in 2-D) and its operation order, so that a plain FP64 build of it and the reference's FP64
 * CUDA build agree to rounding.
 */
#ifndef OSTC_ORACLE_H
#define OSTC_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Boundary type codes follow the reference labels (BoundCond.cu:232-258). */
enum { ORC_SYMMETRY = 3, ORC_FARFIELD = 4, ORC_OUTFLOW = 6, ORC_PERIODIC = 8 };

typedef struct {
  int type;          /* ORC_* */
  int raw[6];        /* x1 x2 y1 y2 z1 z2 exactly as in "boundary   0.txt" (0-based node indices) */
  /* farfield state (used when type == ORC_FARFIELD), FarField ctor BoundCond.cpp:586-669 */
  double density, u, v, w, pressure, temperature, acoustic_speed, gamma, entropy, mw;
} orc_face_in;

typedef struct {
  int mx, my, mz;            /* grid nodes of the block */
  int reconstruction;        /* 1 = 1st order, 2 = MUSCL, 3 = NND2, 4 = AWENO5, 5 = AWENO7 (Parameter.cpp:195-209) */
  int inviscid_scheme;       /* as in setup.txt (informational; the solver is `riemann`) */
  int riemann;               /* 1 = Lax-Friedrichs, 2 = Roe, 3 = AUSM+, 4 = HLLC: the solver the
                                reference's switches select (InviscidScheme.cu:145-159, 345-359,
                                SchemeSelector.cuh:24-45) */
  double entropy_fix_factor; /* Roe entropy fix (Parameter.cpp:474) */
  int viscous_order;         /* 0 = inviscid, 2 = 2nd-order central (SchemeSelector.cuh:47-67) */
  double cfl, prandtl;
  int fixed_time_step;
  double dt;                 /* used when fixed_time_step != 0 */
  int n_face;
  orc_face_in face[16];      /* in the order of the boundary file */
} orc_case;

typedef struct orc_ctx orc_ctx;

/* x, y, z: interior node coordinates, [mz][my][mx] with i fastest (already scaled to metres). */
orc_ctx *orc_create(const orc_case *c, const double *x, const double *y, const double *z);
void orc_destroy(orc_ctx *o);
int orc_ngg(const orc_ctx *o);
/* bv: [6][mz][my][mx] interior (rho, u, v, w, p, T).  Runs the reference initialisation sequence. */
void orc_set_state(orc_ctx *o, const double *bv);
/* Interior copies of cv[5][N], bv[6][N] and mul[N] (any pointer may be NULL). */
void orc_get_state(const orc_ctx *o, double *cv, double *bv, double *mul);
/* Metric (9 entries, row-major 1-based (r,c) -> (r-1)*3+c-1) and Jacobian on the interior nodes. */
void orc_get_metric(const orc_ctx *o, double *metric9, double *jac);
/* Right-hand side dq[5][N] of the current state.  mask: 1 = inviscid (AWENO + Riemann + CDS, or a
 * primitive reconstruction + Riemann),
 * 2 = viscous; the reference evaluates them in that order (RK.cuh:138-139). */
void orc_rhs(orc_ctx *o, unsigned mask, double *dq);
/* n full SSP-RK3 steps (RK.cuh:85-185).  Returns the last dt. */
double orc_step(orc_ctx *o, int n);
double orc_time(const orc_ctx *o);
/* Local CFL time step of the current state and its minimum (TimeAdvanceFunc.cuh:28-83). */
double orc_dt(orc_ctx *o);

#ifdef __cplusplus
}
#endif
#endif
