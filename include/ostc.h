/*
 * ostc.h -- C ABI of the B200 OpenSTC right-hand-side + SSP-RK3 library (libostc_b200.so).
 *
 * The reference solver has no plugin/FFI layer: its seam is the set of C++ template calls made by
 * RK3<mix,turb>() in RK.cuh:112-174 (compute_inviscid_flux, compute_viscous_flux, compute_source,
 * local_time_step/global_time_step, update_cv_and_bv_rk, apply_boundary_conditions,
 * data_communication, update_physical_properties) over the DZone/DParameter/Parameter data built
 * from input/setup.txt and the grid/boundary files.  Each entry point below names the reference
 * interface it replaces.  Conventions:
 *   - every function returns OSTC_OK (0) or a negative OSTC_E* code; ostc_last_error() gives text;
 *   - no exceptions cross the boundary, no torch or CUDA types appear in the signatures;
 *   - a context owns all device memory and one CUDA stream on the device given to ostc_create;
 *     one host thread uses a context at a time;
 *   - host arrays are SoA with the i index fastest: a[l][k][j][i] for l < n_var (or 6, or n_scalar),
 *     over the interior nodes of one block (mx*my*mz per variable).
 */
#ifndef OSTC_H
#define OSTC_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OSTC_OK 0
#define OSTC_EINVAL (-1)     /* bad argument or unsupported configuration */
#define OSTC_EIO (-2)        /* input file missing or malformed */
#define OSTC_ECUDA (-3)      /* CUDA runtime error */
#define OSTC_ESTATE (-4)     /* call out of order (e.g. stepping before a state was set) */
#define OSTC_ENOMEM (-5)     /* device allocation failed */
#define OSTC_ENUMERIC (-6)   /* a device error flag was raised (see ostc_error_flags) */

/* ostc_set_state / ostc_get_state / ostc_rhs pointer kinds */
#define OSTC_HOST 0
#define OSTC_DEVICE 1

/* ostc_set_precision modes */
#define OSTC_PREC_FP64 0   /* every operation in FP64, as the reference */
#define OSTC_PREC_MIXED 1  /* reconstruction, Riemann / flux splitting, viscous flux and (mixtures)
                              transport properties in FP32; RK3 state, EOS, chemistry in FP64 */

/* ostc_rhs term mask (the order of evaluation follows RK.cuh:116-139) */
#define OSTC_TERM_INVISCID 1u
#define OSTC_TERM_VISCOUS 2u
#define OSTC_TERM_SOURCE 4u
#define OSTC_TERM_ALL 7u

/* device error flags (ostc_error_flags) */
#define OSTC_FLAG_NONPOSITIVE 1u   /* rho, p or T not positive after an RK stage */
#define OSTC_FLAG_NAN 2u           /* NaN in the conservative state */

typedef struct ostc_ctx ostc_ctx;

/* Raw device views of one block, zero-copy (replaces reading DZone, Field.h:12-90).  Arrays are
 * ghost-padded SoA: element (i,j,k,l) of a field sits at base[l*plane + (k+gz)*sy*pitch +
 * (j+g)*pitch + (i+g)].  In 2-D (mz == 1) gz is 0: the reference's copied k-ghost layers
 * (eliminate_k_gradient, FieldOperation.cu:42-67) are implicit. */
typedef struct {
  int mx, my, mz, ngg, gz;
  int pitch, sy, sz;       /* padded extents in i (row pitch), j, k */
  long long plane;         /* elements per variable plane */
  double *cv, *bv, *mul;   /* current state: cv[n_var], bv[6] (rho,u,v,w,p,T), mu */
  double *metric, *jac;    /* metric[9] planes ((r-1)*3+(c-1)), Jacobian */
} ostc_zone_view;

/* Build a context from a reference-format case directory: reads <input_dir>/setup.txt (or the file
 * given by setup_txt), the binary grid "grid/grid   0.dat" and "boundary_condition/boundary   0.txt" /
 * "inner   0.txt" below input_dir, computes ghost grids, metrics and Jacobians, and allocates the
 * device state on `device`.  Replaces Parameter(&argc,&argv) + Mesh(parameter) + Driver ctor
 * (Parameter.cpp:10-23, Mesh.cpp:592-641, Driver.cu:12-113). */
int ostc_create(const char *setup_txt, const char *input_dir, int device, ostc_ctx **out);

/* Free every resource of the context. */
void ostc_destroy(ostc_ctx *ctx);

/* Text of the last error raised on this context (or of the last failed ostc_create when ctx is NULL). */
const char *ostc_last_error(const ostc_ctx *ctx);

/* Number of blocks and the size of block b: dims = {mx, my, mz, ngg}. */
int ostc_n_blocks(const ostc_ctx *ctx, int *n_block);
int ostc_block_dims(const ostc_ctx *ctx, int block, int dims[4]);
/* n_var (5 + transported scalars) and n_scalar (Parameter::deduce_sim_info, Parameter.cpp:589-653). */
int ostc_n_var(const ostc_ctx *ctx, int *n_var, int *n_scalar);

/* Arithmetic of the flux path (see OSTC_PREC_*). */
int ostc_set_precision(ostc_ctx *ctx, int mode);

/* Treatment of the finite-rate chemical source in RK3 (mixtures with reaction = 1).
 * OSTC_CHEM_EXPLICIT: the reference's RK3 path (chemSrcMethod forced to 0, Parameter.cpp:280-283).
 * OSTC_CHEM_POINT_IMPLICIT: extension -- the species part of dq is replaced by the solution of
 * (I - dt J_chem) x = dq_species per cell (EPI + solve_chem_system, FiniteRateChem.cu:197-254,
 * 302-357, with the step's global dt), batched over all cells in one launch per stage. */
#define OSTC_CHEM_EXPLICIT 0
#define OSTC_CHEM_POINT_IMPLICIT 1
int ostc_set_chem_mode(ostc_ctx *ctx, int mode);

/* Set the interior primitive state of one block: bv[6][N] (rho,u,v,w,p,T), sv[n_scalar][N] (NULL
 * when n_scalar == 0).  After the last block is set, the next ostc_rhs/ostc_rk3_step first runs
 * the reference initialisation (2-D k-copy, boundary conditions, interfaces, properties,
 * cv <- bv; Driver.cu:115-199, RK.cuh:37-45). Replaces Field::initialize_basic_variables. */
int ostc_set_state(ostc_ctx *ctx, int block, const double *bv, const double *sv, int ptr_kind);

/* Copy the interior state of one block out: cv[n_var][N], bv[6][N], sv[n_scalar][N] (any pointer
 * may be NULL).  Synchronises the context stream.  Replaces Field::copy_data_from_device. */
int ostc_get_state(ostc_ctx *ctx, int block, double *cv, double *bv, double *sv, int ptr_kind);

/* Right-hand side dq[n_var][N] of the current state for one block, terms selected by mask
 * (compute_inviscid_flux + compute_viscous_flux + compute_source, SchemeSelector.cuh:24-67,
 * SourceTerm.cuh:11-35).  dq has the reference's sign: d(cv)/dt = dq / jac. */
int ostc_rhs(ostc_ctx *ctx, int block, unsigned term_mask, double *dq, int ptr_kind);

/* Replace the interior conservative state of one block by cv[n_var][N] (the layout of dq): the
 * primitive state follows by the equation of state (mixtures: the temperature Newton iteration
 * started from each node's current T, FieldOperation.cu:3-40), then the boundary faces, interfaces
 * and (mixtures) properties, as after an RK stage.  The physical time is unchanged.  No reference
 * counterpart: it lets a caller perturb cv (finite differences, adjoint checks). */
int ostc_set_conservative(ostc_ctx *ctx, int block, const double *cv, int ptr_kind);

/* Vector-Jacobian product of ostc_rhs at the current state (no reference counterpart):
 * cv_bar = (d dq / d cv)^T dq_bar for the terms in term_mask, with cv the block's interior
 * conservative variables and every dependent quantity (primitive state by the equation of state,
 * ghost nodes by the boundary faces, transport properties) following cv as ostc_set_conservative
 * defines it.  dq_bar and cv_bar have the layout of dq.  The product is that of the FP64 right-hand
 * side.  Covers the multi-component path (species = 1; inviscid_scheme 71 / 72, viscous, explicit
 * finite-rate source) and the air path (AWENO: WENO5-Z / WENO7-Z reconstruction with AUSM+, HLLC or
 * Lax-Friedrichs, and the viscous terms) on a single block with periodic and outflow faces; anything
 * else returns OSTC_EINVAL.  Accumulation uses atomics: results agree run to run to rounding. */
int ostc_rhs_vjp(ostc_ctx *ctx, int block, unsigned term_mask, const double *dq_bar, double *cv_bar,
                 int ptr_kind);

/* Adjoint of one SSP-RK3 step (RK.cuh:85-185, stage coefficients :10-14) from the current state, with
 * the step's dt (CFL of the current state, or the fixed dt) held constant: lam_in = (d q' / d q)^T
 * lam_out, q the interior conservative state before the step and q' after it (layout of dq).  The
 * state is left as it was.  Same coverage as ostc_rhs_vjp, FP64 precision mode only. */
int ostc_rk3_step_vjp(ostc_ctx *ctx, const double *lam_out, double *lam_in, int ptr_kind);

/* Checkpointed discrete adjoint of n_steps SSP-RK3 steps from the current state: runs the steps
 * (the context ends at the final state, as after ostc_rk3_step(n_steps)), keeping a device
 * checkpoint every `every` steps and each step's dt, then sweeps backwards segment by segment,
 * recomputing a segment's states from its checkpoint: lam_initial = (d q_N / d q_0)^T lam_final.
 * Device memory: (n_steps / every + every + 1) states of (n_var + 6 + n_spec) padded planes (air:
 * n_var + 7). */
int ostc_adjoint_steps(ostc_ctx *ctx, int n_steps, int every, const double *lam_final, double *lam_initial,
                       int ptr_kind);

/* Advance n_steps full SSP-RK3 steps (the loop body of RK3<mix,turb>, RK.cuh:85-185), all stream
 * ordered and replayed from a CUDA graph.  dt_last (nullable) receives the last step's dt (CFL
 * minimum over all blocks, TimeAdvanceFunc.cu:39-64, or the fixed dt); reading it synchronises, and
 * then a raised device error flag (NaN, non-positive rho / p / T) returns OSTC_ENUMERIC. */
int ostc_rk3_step(ostc_ctx *ctx, int n_steps, double *dt_last);

/* Serving loop over independent states (ensemble members, parameter sweeps), single-block cases:
 * for each i < n, state i is set from host arrays bv_in[i] (and sv_in[i] for mixtures) exactly as
 * ostc_set_state does, advanced n_steps SSP-RK3 steps from t = 0, and its primitive state written
 * to bv_out[i] (sv_out[i]).  The host->device copy of state i + 1 and the device->host copy of state
 * i - 1 run on two copy streams while state i is computed (double-buffered device staging), so with
 * pinned host buffers the transfers hide behind the steps.  Synchronises at the end.  No reference
 * counterpart (the reference advances one case per process). */
int ostc_run_states(ostc_ctx *ctx, int n, const double *const *bv_in, const double *const *sv_in,
                    double *const *bv_out, double *const *sv_out, int n_steps);

/* Same as ostc_rk3_step without the dt read-back, bracketed by CUDA events recorded on the context
 * stream: *ms receives the device time of the n_steps steps.  Synchronises. */
int ostc_timed_steps(ostc_ctx *ctx, int n_steps, double *ms);

/* How ostc_rk3_step and ostc_timed_steps issue a step.  OSTC_LAUNCH_GRAPH (the default): one CUDA
 * graph per step, captured on first use, with the blocks' stage work forked onto side streams inside
 * it.  OSTC_LAUNCH_BLOCK_LOOP: the reference's per-block launch loop (RK.cuh:112-174) - every kernel
 * launched from the host in turn, block after block, on the context stream - for comparison and
 * debugging.  Both compute the same results bit for bit. */
#define OSTC_LAUNCH_GRAPH 0
#define OSTC_LAUNCH_BLOCK_LOOP 1
int ostc_set_launch_mode(ostc_ctx *ctx, int mode);

/* Seed of the white-noise inflow (an inflow struct with fluctuation_type 1): generator state i of the
 * face plane restarts from curand_init(seed + i, i, 0), as the reference's initialize_rng does with the
 * clock (BoundCond.cu:1384-1391, 1731-1735); ostc_create seeds it from the clock too.  A case run with
 * the seed the reference drew reproduces its inflow noise.  No effect without such a face. */
int ostc_set_inflow_seed(ostc_ctx *ctx, long long seed);

/* Number of kernels one step launches (kernel nodes of the captured step graph). */
int ostc_step_kernel_count(ostc_ctx *ctx, int *n_kernels);

/* Physical time advanced so far (RK.cuh:175-176).  Synchronises. */
int ostc_physical_time(ostc_ctx *ctx, double *t);

/* Snapshot the current state as the residual reference (store_last_step, TimeAdvanceFunc.cu:6-19). */
int ostc_store_residual_reference(ostc_ctx *ctx);
/* RMS change of rho, |V|, p, T since the snapshot (compute_residual, Residual.cuh:74-190):
 * res[l] = sqrt(sum over all interior nodes of (change)^2 / total node count). Synchronises. */
int ostc_residual(ostc_ctx *ctx, double res[4]);

/* Bounds-checked build only (libostc_b200_checked.so, compiled with -DOSTC_BOUNDS_CHECK): bit 1 = a
 * padded-plane index, bit 2 = an interior index fell outside its block since the last call (the
 * index was clamped, no access left the arrays); the call clears the flag.  ostc_bounds_checked()
 * tells whether the loaded library is that build (1) or the regular one (0, flags always 0).  No
 * reference counterpart: a device-side substitute for a memory checker. */
int ostc_bounds_flags(ostc_ctx *ctx, unsigned *flags);
int ostc_bounds_checked(void);

/* Device error flags (OSTC_FLAG_*) accumulated since the last call, then cleared.  Synchronises. */
int ostc_error_flags(ostc_ctx *ctx, unsigned *flags);

/* Zero-copy device view of block b (valid until ostc_destroy). */
int ostc_device_view(ostc_ctx *ctx, int block, ostc_zone_view *out);

/* Kernel timing for measurement: runs n_steps steps launch by launch (no graph) with CUDA events
 * around every kernel on the context stream and returns, per kernel family, the number of launches
 * and the summed device milliseconds.  names[i] points to static strings. Returns the number of
 * families written (<= max). */
int ostc_profile_steps(ostc_ctx *ctx, int n_steps, int max, const char **names, int *launches, double *ms);

/* Pin the kernel shape of one inviscid sweep (AWENO path) instead of the autotuner's choice:
 * precision 0 = FP64, 1 = mixed; dir 0/1/2 = x/y/z; variant 0.. (x: 0 only, one thread per face;
 * y/z: 0 column march, 1-3 shared-memory tiles of three shapes), or
 * -1 to return the direction to the autotuner (forgetting its cached result for these block shapes).
 * Every variant computes the same face fluxes with the same expressions; the choice changes speed,
 * not results.  Takes effect at the next step.  No reference counterpart (its sweep kernels have one
 * fixed shape). */
int ostc_set_sweep_variant(ostc_ctx *ctx, int precision, int dir, int variant);

/* What the sweep autotuner measured for one block: precision 0 = FP64, 1 = mixed; dir 0/1/2 = x/y/z.
 * chosen receives the variant the steps use (-1 before tuning); ms[v] the device milliseconds of
 * one launch of variant v as timed by the tuner (0 where it was not timed in this context, e.g. a
 * result reused from an earlier context of the same shape).  Returns the variant count of that
 * direction.  No reference counterpart: the reference has one fixed kernel shape per sweep. */
int ostc_tune_report(ostc_ctx *ctx, int block, int precision, int dir, int *chosen, float *ms, int max);

/* Number of interior nodes over all blocks (the unit of cell-steps/s). */
int ostc_total_nodes(const ostc_ctx *ctx, long long *n);

/* Host-only parse of a case directory (no device is touched): runs the setup/grid/boundary readers
 * and writes out[0..13] = ngg, inviscid_type, n_var, n_scalar, n_block, dimension, mx, my, mz of
 * block 0, number of boundary faces of block 0, reconstruction, inviscid_scheme, viscous_order,
 * number of boundary-face applications per stage.  On failure msg receives the reason
 * (Parameter::deduce_known_info / Mesh::Mesh checks, Parameter.cpp:187-437, Mesh.cpp:592-641). */
int ostc_probe_case(const char *setup_txt, const char *input_dir, int out[16], char *msg, int msg_len);

/* ---- Tecplot flow-field file (FieldIO, FieldIO.h:73-648; read_flowfield, Initialize.cuh:102-215)
 *
 * ostc_write_plt writes every block's current state as the reference's output/flowfield.plt: binary
 * Tecplot V112, one ordered zone per block with ngg_out ghost layers on each side, node-located
 * double variables x, y, z, density, u, v, w, pressure, temperature, mach, then the species mass
 * fractions (a laminar case without user-defined output); solution_time goes into every zone header.
 * ostc_read_plt restarts from such a file (written here or by the reference): the primitive
 * variables and mass fractions are found by name, their interior values set as ostc_set_state does,
 * and the physical time continues from the file's solution time (returned in *solution_time, may be
 * NULL).  Zone count and extents must match the case's blocks; float data, passive or shared
 * variables and auxiliary zone data are refused with OSTC_EIO and the reason. */
int ostc_write_plt(ostc_ctx *ctx, const char *path, int ngg_out, double solution_time);
int ostc_read_plt(ostc_ctx *ctx, const char *path, double *solution_time);

/* ---- single-point statistics (SinglePointStat, SinglePointStat.h / SinglePointStat.cu:515-706)
 *
 * Replaces the collector the reference runs after every time step past start_collect_statistics_iter
 * (RK.cuh:200-203, collect_single_point_basic_statistics SinglePointStat.cu:641-706) and its export
 * (export_statistical_data, SinglePointStat.cu:553-638).  Per block and per node, one ghost layer
 * included, sums over the collected steps of:
 *   group 0 Reynolds 1st: rho, p, then u / v / w / T as OSTC_STAT_REY_* select (stat_rey_1st)
 *   group 1 Favre 1st:    rho u, rho v, rho w, rho T, then rho Y_k for every species
 *   group 2 Reynolds 2nd: rho rho, p p, then rho p with OSTC_STAT_RHO_P (rho_p_correlation)
 *   group 3 Favre 2nd:    rho u u, rho v v, rho w w, rho u v, rho u w, rho v w, rho T T, rho Y_k Y_k
 * each group stored [n_var][mz+2][my+2][mx+2], i fastest.  With if_collect_statistics = 1 in the
 * setup (and an unsteady case) ostc_create enables collection with start_collect_statistics_iter,
 * stat_rey_1st and rho_p_correlation; steps are counted from ostc_create.  The TKE budget and the
 * species correlation / dissipation collectors (stat_lib/) are not provided. */
#define OSTC_STAT_REY_U 1u
#define OSTC_STAT_REY_V 2u
#define OSTC_STAT_REY_W 4u
#define OSTC_STAT_REY_T 8u
#define OSTC_STAT_RHO_P 16u
/* The additional collectors (collect_single_point_additional_statistics, SinglePointStat.cu:707-722),
 * over interior nodes, exported as tke_budget.bin, species_velocity_correlation.bin and
 * species_dissipation_rate.bin (stat groups 4, 5, 6; ostc_stat_get reads them too):
 *   group 4 TKE budget: tau11 tau12 tau13 tau22 tau23 tau33, tau_ij dU_i/dx_j (stat_tke_budget)
 *   group 5 per species: rho u Y, rho v Y, rho w Y (stat_species_velocity_correlation)
 *   group 6 per species: rho D |grad Y|^2, rho D dY/dx, dY/dy, dY/dz, rho D (stat_species_dissipation_rate)
 * Through ostc_stat_enable the species groups cover every species; the setup's stat_species selects. */
#define OSTC_STAT_TKE_BUDGET 32u
#define OSTC_STAT_SPECIES_VELOCITY 64u
#define OSTC_STAT_SPECIES_DISSIPATION 128u

/* Allocate and zero the accumulators of every block and collect after each later step (ostc_rk3_step,
 * ostc_timed_steps, ostc_profile_steps) whose index, counted from this call starting at 1, exceeds
 * start_step.  Calling it again restarts from zero with the new selection. */
int ostc_stat_enable(ostc_ctx *ctx, int start_step, unsigned flags);
/* Stop collecting and free the accumulators. */
int ostc_stat_disable(ostc_ctx *ctx);
/* Variables per group (n_var[4]), collections so far (the reference's per-variable counters, all
 * equal here) and steps counted since enabling.  OSTC_ESTATE when collection is off. */
int ostc_stat_info(ostc_ctx *ctx, int n_var[4], int *n_collected, long long *steps);
/* Copy group g of block b to host or device memory (ptr_kind): groups 0..3 n_var x (mx+2)(my+2)(mz+2)
 * doubles, groups 4..6 n_var x mx my mz (no ghost layer; n_var from ostc_stat_group_vars, 0 when the
 * collector is off), layout as above.  Synchronises. */
int ostc_stat_get(ostc_ctx *ctx, int block, int group, double *out, int ptr_kind);
/* Number of variables of statistics group g (0..6) in the current selection. */
int ostc_stat_group_vars(ostc_ctx *ctx, int group, int *n_var);
/* Write coll_rey_1st.bin, coll_fav_1st.bin, coll_rey_2nd.bin, coll_fav_2nd.bin into dir in the
 * reference's layout (SinglePointStat.cu:163-226, 553-638, one process): int32 n_block, n_var, ngg = 1;
 * the variable names as int32 characters, each ended by an int32 0; int32 counters[n_var]; then per
 * block int32 mx, my, mz and its n_var planes of doubles. */
int ostc_stat_export(ostc_ctx *ctx, const char *dir);
/* Read the four files back into the accumulators and counters (if_continue_collect_statistics,
 * read_previous_statistical_data): the selection must match the enabled one and the block extents
 * the case's, else OSTC_EIO with the reason.  Collection then continues from the next step. */
int ostc_stat_import(ostc_ctx *ctx, const char *dir);

/* The reference's steady driver (steady_simulation, SteadySim.cuh:15-140, as Simulate.cuh selects it for
 * steady = 1): up to max_iter iterations, each over every block and in place: dq from the chemical
 * source (with its Jacobian for chemSrcMethod 1 / 2) and the inviscid and viscous fluxes; local time
 * steps (local_time_step, TimeAdvanceFunc.cuh:28-83); implicit_treatment (ImplicitTreatmentHPP.cuh:7-54):
 * with implicit_method 0 the point-implicit chemistry (EPI / DA, FiniteRateChem.cu:233-254, 414-426),
 * with 1 DPLUR with DPLUR_inner_step inner iterations (DPLUR.cuh:14-327); update_cv_and_bv
 * (FieldOperation.cuh:189-232); boundary faces, interfaces, properties.  The settings come from the
 * setup (implicit_method, DPLUR_inner_step, chemSrcMethod, convergence_criteria, output_screen).  As the
 * reference, it computes the residual (RMS change of rho, |V|, p, T, scaled by that of the first
 * iteration) after iteration 1 and every output_screen-th and stops once its largest component falls
 * below convergence_criteria.  iters_done / err_max (nullable) receive the iterations run and the last
 * scaled residual (-1 if none was computed).  The physical time does not advance.  Synchronises. */
int ostc_steady_step(ostc_ctx *ctx, int max_iter, int *iters_done, double *err_max);

/* The reference's dual time stepping (dual_time_stepping, DualTimeStepping.cuh:32-252; temporal_scheme 2):
 * n_steps physical steps of the setup's dt, each forming q* = jac / (2 dt) (4 cv^n - cv^(n-1)) and then
 * up to inner_iteration pseudo-time iterations of the steady driver's form with dq += q* - 1.5 jac /
 * dt cv and DPLUR (DPLUR_inner_step inner sweeps, diagonal factor 1.5 / dt).  Every
 * iteration_adjust_step-th step the inner loop is monitored as the reference's inner_converged does
 * (residual scaled by the first iteration's; stop below 1e-3, the count trimmed to it; raised by 5 up
 * to max_inner_iteration when the last iteration is still above) - the monitored residual uses the
 * ostc_residual reference, which it overwrites.  inner_iters (nullable) receives the count in force
 * afterwards.  The physical time advances by dt per step; statistics collect as after an RK3 step.
 * Synchronises. */
int ostc_dual_time_step(ostc_ctx *ctx, int n_steps, int *inner_iters);

/* Limits of ostc_residual_noalloc: its static scratch holds one partial sum set per block of
 * 256 threads x 64 nodes, for at most OSTC_NOALLOC_MAX_BLOCKS blocks (128 KB of device memory). */
#define OSTC_NOALLOC_NODES_PER_THREAD 64
#define OSTC_NOALLOC_MAX_BLOCKS 4096
#define OSTC_NOALLOC_MAX_NODES (256LL * OSTC_NOALLOC_NODES_PER_THREAD * OSTC_NOALLOC_MAX_BLOCKS)

/* Residual norms without any device allocation.  No counterpart in the reference: it exists for
 * callers that cannot call cudaMalloc - hosts whose device memory is planned up front and handed out
 * by their own pool, loops that must not take an allocation's implicit synchronisation, code that
 * runs while another thread captures a CUDA graph in global mode.
 * bv_new, bv_old: caller-owned device arrays of interior primitive states, [6][n_nodes]
 * (rho,u,v,w,p,T), e.g. the output of ostc_get_state(..., OSTC_DEVICE).  res: host array that
 * receives the RMS changes of rho, |V|, p and T (the same quantities as ostc_residual).  stream:
 * cudaStream_t to run on (NULL = legacy default stream); the call synchronises it.  A caller that
 * runs while another thread captures a graph must pass a stream created with cudaStreamNonBlocking:
 * work on the legacy default stream during another thread's capture of a blocking stream
 * invalidates that capture.
 * n_nodes above OSTC_NOALLOC_MAX_NODES (67,108,864) is rejected with OSTC_EINVAL; the message is
 * available from ostc_last_error(NULL).
 * Scratch lives in one file-scope __device__ array (per GPU, held until the process exits), shared
 * by every call: calls that overlap on the GPU (different streams, or host threads on the same
 * device) race on it and must be serialised by the caller.  Each call writes every partial it
 * reads, so nothing in the array has to start at zero.  The first call on a device resolves the
 * array's device address (cudaGetSymbolAddress) and caches it with the id of the current context;
 * a later call in a new context (after cudaDeviceReset, or a primary context released and made
 * again) resolves it anew.  Make the first call on a device, and the first after such a reset,
 * before any stream capture. */
int ostc_residual_noalloc(const double *bv_new, const double *bv_old, long long n_nodes, double res[4],
                          void *stream);

#ifdef __cplusplus
}
#endif
#endif
