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
enum { ORC_WALL = 2, ORC_SYMMETRY = 3, ORC_FARFIELD = 4, ORC_INFLOW = 5, ORC_OUTFLOW = 6, ORC_SUBSONIC_INFLOW = 7,
       ORC_PERIODIC = 8, ORC_BACK_PRESSURE = 9 };
/* subsonic inflow: pressure / temperature hold the total pressure / temperature and u, v, w the flow
 * direction; back pressure: pressure holds the back pressure (BoundCond.cpp:704-768) */

typedef struct {
  int type;          /* ORC_* */
  int raw[6];        /* x1 x2 y1 y2 z1 z2 exactly as in "boundary   0.txt" (0-based node indices) */
  /* farfield state (used when type == ORC_FARFIELD), FarField ctor BoundCond.cpp:586-669 */
  double density, u, v, w, pressure, temperature, acoustic_speed, gamma, entropy, mw;
  /* walls (type == ORC_WALL, Wall ctor BoundCond.cpp:497-560): 1 adiabatic, 0 isothermal at temperature */
  int wall_adiabatic;
  /* constant inflow (type == ORC_INFLOW, Inflow ctor BoundCond.cpp:157-214): the state above and the
   * mass fractions of a mixture */
  double y[16];
  /* inflow_type 2 (mixing-layer problems, BoundCond.cpp:10-98, apply_inflow BoundCond.cuh:384-430):
   * the state above is the upper stream, `lower` (rho u v w p T) and y_lower the lower one, blended in
   * u by tanh(2 y / delta_omega).  The white-noise fluctuation is not restated (curand). */
  int inflow_type;
  double delta_omega;
  double lower[6];
  double y_lower[16];
} orc_face_in;

/* Mixture tables (Species / Reaction, ChemData.cpp; DParameter.cu:57-155), row-major [i][j]. */
#define ORC_MAX_SPEC 16
#define ORC_MAX_REAC 64
typedef struct {
  int n_spec, n_reac;
  double mw[ORC_MAX_SPEC], t_low[ORC_MAX_SPEC], t_mid[ORC_MAX_SPEC];
  double low[ORC_MAX_SPEC * 7], high[ORC_MAX_SPEC * 7];
  double lj_potent_inv[ORC_MAX_SPEC], vis_coeff[ORC_MAX_SPEC];
  double wj_div_wi_1_4[ORC_MAX_SPEC * ORC_MAX_SPEC], sqrt_wiwj_8[ORC_MAX_SPEC * ORC_MAX_SPEC];
  double binary_diff[ORC_MAX_SPEC * ORC_MAX_SPEC], kb_over_eps_jk[ORC_MAX_SPEC * ORC_MAX_SPEC];
  int label[ORC_MAX_REAC], rev_type[ORC_MAX_REAC], order[ORC_MAX_REAC];
  int stoi_f[ORC_MAX_REAC * ORC_MAX_SPEC], stoi_b[ORC_MAX_REAC * ORC_MAX_SPEC];
  double A[ORC_MAX_REAC], b[ORC_MAX_REAC], Ea[ORC_MAX_REAC], A2[ORC_MAX_REAC], b2[ORC_MAX_REAC], Ea2[ORC_MAX_REAC];
  double third_body[ORC_MAX_REAC * ORC_MAX_SPEC];
  double troe_alpha[ORC_MAX_REAC], troe_t3[ORC_MAX_REAC], troe_t1[ORC_MAX_REAC], troe_t2[ORC_MAX_REAC];
} orc_chem;

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
  /* multi-component mixture (species = 1): n_spec > 0 and chem set; finite_rate = 1 adds the
   * chemical source (reaction = 1, MixtureModel::FR) */
  int n_spec;
  int finite_rate;
  const orc_chem *chem;
  double weno_eps_scale;     /* rho_inf^2 v_inf^2 of the reference state (DParameter.cu:26-29) */
  double v_ref;              /* v_inf (component-wise WENO eps scaling, WENO.cu:1471-1473) */
  /* default initialisation of every node, ghosts included (Field.cu:316-345): has_init, then
   * rho u v w p T and the mass fractions */
  int has_init;
  double init_bv[6];
  double init_sv[ORC_MAX_SPEC];
  /* 0: explicit chemistry (the reference's RK3); 1: point-implicit -- after the fluxes the species
   * part of dq is replaced by the solution of (I - dt J_chem) x = dq_s (EPI, solve_chem_system,
   * FiniteRateChem.cu:197-254, 302-357) with the step's dt */
  int chem_mode;
  /* steady driver (steady_simulation, SteadySim.cuh:15-140): local time steps; implicit_method 0
   * (explicit, plus the point-implicit chemistry of chem_src_method) or 1 (DPLUR with dplur_inner
   * inner iterations, DPLUR.cuh:282-322); chem_src_method 0 explicit, 1 EPI, 2 diagonal (DA) */
  int implicit_method, dplur_inner, chem_src_method;
  /* dual time stepping (dual_time_stepping, DualTimeStepping.cuh:32-252; temporal_scheme 2): physical
   * step dt (the case's dt), inner iterations and their adaptation (inner_converged,
   * DualTimeStepping.cu:32-135) */
  int inner_iteration, max_inner_iteration, iteration_adjust_step;
  /* problem_type 1: every node, ghosts included, starts from the two-stream profile
   * (initialize_mixing_layer_with_info, Initialize.cu:259-326) instead of the default state */
  int problem_type;
  double ml_upper[6], ml_lower[6], ml_y_upper[ORC_MAX_SPEC], ml_y_lower[ORC_MAX_SPEC], ml_delta_omega;
} orc_case;

typedef struct orc_ctx orc_ctx;

/* x, y, z: interior node coordinates, [mz][my][mx] with i fastest (already scaled to metres). */
orc_ctx *orc_create(const orc_case *c, const double *x, const double *y, const double *z);
void orc_destroy(orc_ctx *o);
int orc_ngg(const orc_ctx *o);
/* bv: [6][mz][my][mx] interior (rho, u, v, w, p, T).  Runs the reference initialisation sequence. */
void orc_set_state(orc_ctx *o, const double *bv);
/* Same with the species mass fractions sv: [n_spec][mz][my][mx] (mixtures). */
void orc_set_state_sv(orc_ctx *o, const double *bv, const double *sv);
/* Interior copies of cv[n_var][N], bv[6][N] and mul[N] (any pointer may be NULL); n_var = 5 + n_spec. */
void orc_get_state(const orc_ctx *o, double *cv, double *bv, double *mul);
/* Interior mass fractions sv[n_spec][N] and, when non-NULL, thermal conductivity, rho*D[n_spec][N],
 * acoustic speed and gamma (mixtures). */
void orc_get_mixture(const orc_ctx *o, double *sv, double *cond, double *rho_d, double *acoustic, double *gamma);
/* Metric (9 entries, row-major 1-based (r,c) -> (r-1)*3+c-1) and Jacobian on the interior nodes. */
void orc_get_metric(const orc_ctx *o, double *metric9, double *jac);
/* Right-hand side dq[n_var][N] of the current state.  mask: 4 = chemical source (evaluated first,
 * RK.cuh:116), 1 = inviscid (AWENO + Riemann + CDS, a primitive reconstruction + Riemann, or the
 * flux-split WENO of inviscid_scheme 51/52/71/72),
 * 2 = viscous; the reference evaluates them in that order (RK.cuh:138-139). */
void orc_rhs(orc_ctx *o, unsigned mask, double *dq);
/* n full SSP-RK3 steps (RK.cuh:85-185).  Returns the last dt. */
double orc_step(orc_ctx *o, int n);
/* n iterations of the steady driver (steady_simulation, SteadySim.cuh:65-140) */
void orc_steady(orc_ctx *o, int n);
/* n physical steps of dual time stepping; returns the inner-iteration count in force after them */
int orc_dual(orc_ctx *o, int n);
/* one single-point statistics collection added to acc (collect_single_point_basic_statistics) */
void orc_stat_collect(const orc_ctx *o, int n_rey, const int *rey_idx, int rho_p, double *acc);
/* The additional collectors on the interior nodes (SinglePointStat.cu:707-722): tke[7][N] (null: off),
 * and for the species ss_idx[0..nss) svc[3 nss][N] and sdr[5 nss][N] (null: off). */
void orc_stat_extra(const orc_ctx *o, double *tke, int nss, const int *ss_idx, double *svc, double *sdr);
double orc_time(const orc_ctx *o);
/* Local CFL time step of the current state and its minimum (TimeAdvanceFunc.cuh:28-83). */
double orc_dt(orc_ctx *o);

/* Multi-block: one context per block plus the 1:1 interfaces of the inner-face file
 * ("inner   0.txt", Mesh.cpp:812-844), each as its two lines: this block's 1-based range with the
 * reference's signs (x1 x2 y1 y2 z1 z2, seventh value unused) and the target's range + block id. */
typedef struct {
  int raw[7];
  int traw[7];
} orc_inner_in;

typedef struct orc_multi orc_multi;
/* n_inner[b] faces of block b, concatenated in `inner` in block order. */
orc_multi *orc_multi_create(int nb, const orc_case *cases, const double *const *x, const double *const *y,
                            const double *const *z, const int *n_inner, const orc_inner_in *inner);
void orc_multi_destroy(orc_multi *m);
orc_ctx *orc_multi_block(orc_multi *m, int b);
/* bv[b]: [6][N_b] interior state of block b; sv[b] its mass fractions (NULL for air). */
void orc_multi_set_state(orc_multi *m, const double *const *bv, const double *const *sv);
double orc_multi_step(orc_multi *m, int n);

#ifdef __cplusplus
}
#endif
#endif
