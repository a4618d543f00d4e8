// context.cuh -- the library context behind an ostc_ctx handle: per-block device resources
// (BlockRes), streams, captured graphs, the constant-table binding and the CK error macro.
// Part of the ostc_b200.cu translation unit (included in order; not a standalone header).
#pragma once

using namespace ostc;

struct BlockRes {
  DevBlock db{};
  double *met = nullptr, *jac = nullptr;
  float *met32 = nullptr;  // air: metric + Jacobian rounded to FP32 (DevBlock::met32)
  // state slots: 0..2 the RK3 stage buffers, 3 the step adjoint's copy of a step's output
  double *cv[4]{}, *bv[4]{}, *mul[4]{};
  double *sv[4]{}, *cond[4]{}, *rhod[4]{}, *gam[4]{}, *acs[4]{};  // mixtures only
  double *dq = nullptr;
  double *last = nullptr;
  std::vector<DevFace> faces;  // file order
  std::vector<double *> face_y;  // per face: y of its nodes (mixing-layer inflows), else null
  double *plt_xyz = nullptr;     // flow-field output: the zone's coordinates for output width plt_g
  int plt_g = -1;
  double *ycoord = nullptr;      // problem_type 1: y of every padded node (the initial profile)
  std::vector<DevInner> inner;  // interfaces of this block, file order
  int yz_var[2][2] = {{-1, -1}, {-1, -1}};  // autotuned y / z sweep variant [FP64, mixed][y, z]
  int x_var[2] = {-1, -1};                   // autotuned x sweep variant [FP64, mixed]
  float tune_ms[2][3][8] = {};               // autotuner's time per variant [precision][x, y, z][variant]
  std::vector<int> inner_target;
  double *adj = nullptr;  // node adjoint planes of ostc_rhs_vjp (allocated on first use)
  double *dqb = nullptr;  // dq_bar on the device
  // step adjoint: [lam_cv, x2_cv, x1_cv, g_cv] (n_var x N each) then [lam_T, x2_T, x1_T, g_T] (N each)
  double *adj_work = nullptr;
  double *stat = nullptr;  // single-point statistics accumulators (ostc_stat.cuh layout)
  // steady driver (ostc_steady.cuh layout, allocated on first use): local time steps, inviscid
  // spectral radii, chemical source Jacobian, DPLUR iterates
  double *dtl = nullptr, *srad = nullptr, *cj = nullptr, *dq0 = nullptr, *dqk = nullptr;
  // dual time stepping: the previous physical step's cv (padded planes) and the BDF2 source q* (interior)
  double *qn1 = nullptr, *qstar = nullptr;
  // mixtures on the primitive-reconstruction path (pv_mix.cuh): face fluxes of one sweep, entropy-fix
  // thresholds (padded)
  double *fcb = nullptr, *efd = nullptr;
};

struct ostc_ctx {
  int device = 0;
  // multi-component mixture (species = 1): tables, device copy in constant memory, n_var = 5 + n_spec
  bool mixture = false;
  bool tables = false;  // constant tables in use (mixtures, or the flux-split path's epsilon scales)
  int nv = 5;
  ChemTables chem;
  MixTables mixtab{};
  // default initialisation of every node (ghosts included) before the interior state is set
  // (Field::initialize_basic_variables with the default_init struct, Field.cu:316-345, 388-470)
  int chem_mode = OSTC_CHEM_EXPLICIT;
  bool has_init = false;
  double init_bv[6]{};
  std::vector<double> init_sv;
  cudaStream_t stream = nullptr;
  // multi-block cases: side streams on which the blocks' stage work runs concurrently (forked from
  // and joined back into `stream`, inside the captured step graph as well)
  std::vector<cudaStream_t> side;
  std::vector<cudaEvent_t> side_ev;
  cudaEvent_t fork_ev = nullptr;
  // ostc_run_states pipeline: copy streams, double-buffered device staging, hand-over events
  cudaStream_t rs_h2d = nullptr, rs_d2h = nullptr;
  double *rs_in[2]{}, *rs_out[2]{};
  cudaEvent_t rs_in_ready[2]{}, rs_in_free[2]{}, rs_out_ready[2]{}, rs_out_free[2]{};
  Setup setup;
  Derived der;
  HostMesh mesh;
  std::vector<BlockRes> blk;
  std::vector<std::pair<int, int>> order;
  int precision = OSTC_PREC_FP64;
  bool state_set = false, initialised = false;
  std::vector<char> block_set;
  unsigned long long *d_dtbits = nullptr;
  double *d_dt = nullptr, *d_time = nullptr, *d_sums = nullptr, *d_staging = nullptr;
  long long *d_step = nullptr;
  unsigned *d_flags = nullptr;
  cudaGraphExec_t graph = nullptr;
  int graph_precision = -1;
  // one steady / dual-time iteration captured as a graph: key = 2 x mixed + dual, with its physical dt
  cudaGraphExec_t steady_graph = nullptr;
  int steady_key = -1;
  double steady_dt = 0;
  int launch_mode = OSTC_LAUNCH_GRAPH;
  // white-noise inflow: one generator state per node of the largest fluctuating face plane, shared by
  // the faces as the reference shares one array (BoundCond.cu:1706-1735); seeded by ostc_set_inflow_seed
  curandState *rng = nullptr;
  long long rng_size = 0;
  // problem_type 1: the two streams of the initial mixing-layer profile
  MixingLayerStreams ml;
  // digital-filter inflow (at most one face): its buffers, block / face, the stream molecular weights,
  // a device zero (the reference's dt before the first step), and whether the boundary faces being
  // enqueued are the initial application
  DevDf df{};
  int df_block = -1, df_face = -1;
  double df_mw_up = kMwAir, df_mw_lo = kMwAir;
  double *d_zero = nullptr;
  bool bc_initial = false;
  bool tuned[2] = {false, false};  // x / y / z sweep autotuning done [FP64, mixed]
  int forced[2][3] = {{-1, -1, -1}, {-1, -1, -1}};  // sweep variants pinned by ostc_set_sweep_variant
  int graph_kernels = 0;
  // steady driver: iterations done (the reference's step counter) and the residual scales of its
  // first iteration (compute_residual, Residual.cuh:128-136)
  long long steady_iter = 0;
  double res_scale[4] = {1, 1, 1, 1};
  // dual time stepping: physical steps done, the inner-iteration count in force (adapted by
  // inner_converged, DualTimeStepping.cu:32-135) and the inner residual scales
  long long dual_step = 0;
  int dual_inner = -1;
  double res_scale_inner[4] = {1, 1, 1, 1};
  std::string err;
  int sm_count = 148;
  // timing (ostc_profile_steps)
  bool timing = false;
  struct Fam {
    const char *name;
    int launches;
    double ms;
  };
  std::vector<Fam> fams;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_pool;
  std::vector<std::pair<int, size_t>> ev_used;
  // single-point statistics: collected after every step whose index (from enabling, 1-based)
  // exceeds stat_start
  bool stat_on = false;
  int stat_start = 0;
  long long stat_steps = 0;
  int stat_count = 0;
  unsigned stat_flags = 0;
  StatSpec stat_spec{};
};

static std::string g_create_error;

// The constant-memory tables belong to one context at a time; a context (re)binds them before its
// first launch, outside any stream capture.
static const ostc_ctx *g_mix_owner = nullptr;
static int bind_tables(ostc_ctx *ctx) {
  if (!ctx->tables || g_mix_owner == ctx) return 0;
  if (g_mix_owner && cudaDeviceSynchronize() != cudaSuccess) return -1;  // the previous owner's work
  if (cudaMemcpyToSymbol(c_mix, &ctx->mixtab, sizeof(MixTables)) != cudaSuccess) return -1;
  g_mix_owner = ctx;
  return 0;
}

namespace ostc {
// Error text of the context-free entry points (ostc_create failures, ostc_residual_noalloc),
// reported by ostc_last_error(NULL).
void set_free_error(const std::string &msg) { g_create_error = msg; }
}  // namespace ostc

#define CK(call)                                                                                         \
  do {                                                                                                   \
    cudaError_t e_ = (call);                                                                             \
    if (e_ != cudaSuccess) {                                                                             \
      ctx->err = std::string(#call) + ": " + cudaGetErrorString(e_);                                      \
      return OSTC_ECUDA;                                                                                 \
    }                                                                                                    \
  } while (0)
