// api_step.cuh -- C ABI (include/ostc.h): RK3 steps from the captured step graph or the
// per-block launch loop, timing, residuals, the steady and dual-time drivers, bounds flags.
// Part of the ostc_b200.cu translation unit (included in order; not a standalone header).
#pragma once

extern "C" {

static int ensure_graph(ostc_ctx *ctx) {
  if (!ctx->graph || ctx->graph_precision != ctx->precision) {
    if (ctx->graph) {
      cudaGraphExecDestroy(ctx->graph);
      ctx->graph = nullptr;
    }
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    enqueue_step_any(ctx);
    CK(cudaStreamEndCapture(ctx->stream, &g));
    CK(cudaGraphInstantiate(&ctx->graph, g, 0));
    size_t nodes = 0;
    CK(cudaGraphGetNodes(g, nullptr, &nodes));
    std::vector<cudaGraphNode_t> nv(nodes);
    CK(cudaGraphGetNodes(g, nv.data(), &nodes));
    int nk = 0;
    for (auto nd : nv) {
      cudaGraphNodeType t;
      if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++nk;
    }
    ctx->graph_kernels = nk;
    cudaGraphDestroy(g);
    ctx->graph_precision = ctx->precision;
  }
  return OSTC_OK;
}

// One step as ostc_set_launch_mode selects: the captured graph, or every kernel launched from the
// host, block after block on the context stream.
static int launch_step(ostc_ctx *ctx) {
  if (ctx->launch_mode == OSTC_LAUNCH_BLOCK_LOOP) {
    if (int r = enqueue_step_any(ctx)) return r;
    CK(cudaGetLastError());
  } else {
    CK(cudaGraphLaunch(ctx->graph, ctx->stream));
  }
  return stat_after_step(ctx);
}

int ostc_set_launch_mode(ostc_ctx *ctx, int mode) {
  if (!ctx) return OSTC_EINVAL;
  if (mode != OSTC_LAUNCH_GRAPH && mode != OSTC_LAUNCH_BLOCK_LOOP) {
    ctx->err = "launch mode must be OSTC_LAUNCH_GRAPH (0) or OSTC_LAUNCH_BLOCK_LOOP (1)";
    return OSTC_EINVAL;
  }
  ctx->launch_mode = mode;
  return OSTC_OK;
}

int ostc_set_inflow_seed(ostc_ctx *ctx, long long seed) {
  if (!ctx) return OSTC_EINVAL;
  if (!ctx->rng && !ctx->df.rng) return OSTC_OK;
  cudaSetDevice(ctx->device);
  if (ctx->rng)
    k_rng_init<<<grid_for(ctx, ctx->rng_size, 128), 128, 0, ctx->stream>>>(ctx->rng, ctx->rng_size,
                                                                            (unsigned long long)seed);
  if (ctx->df.rng) df_start(ctx, (unsigned long long)seed);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->stream));
  return OSTC_OK;
}

int ostc_rk3_step(ostc_ctx *ctx, int n_steps, double *dt_last) {
  if (!ctx || n_steps < 0) return OSTC_EINVAL;
  cudaSetDevice(ctx->device);
  if (int r = check_ready(ctx)) return r;
  if (ctx->launch_mode == OSTC_LAUNCH_GRAPH)
    if (int r = ensure_graph(ctx)) return r;
  for (int s = 0; s < n_steps; ++s)
    if (int r = launch_step(ctx)) return r;
  if (dt_last) {
    unsigned flags = 0;
    CK(cudaMemcpyAsync(dt_last, ctx->d_dt, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(&flags, ctx->d_flags, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (flags) {
      ctx->err = (flags & OSTC_FLAG_NAN) ? "a NaN appeared in the conservative state (ostc_error_flags reads and clears it)"
                                         : "non-positive density, pressure or temperature after an RK stage "
                                           "(ostc_error_flags reads and clears it)";
      return OSTC_ENUMERIC;
    }
  }
  return OSTC_OK;
}

int ostc_timed_steps(ostc_ctx *ctx, int n_steps, double *ms) {
  if (!ctx || n_steps < 0 || !ms) return OSTC_EINVAL;
  cudaSetDevice(ctx->device);
  if (int r = check_ready(ctx)) return r;
  if (ctx->launch_mode == OSTC_LAUNCH_GRAPH)
    if (int r = ensure_graph(ctx)) return r;
  cudaEvent_t a, b;
  CK(cudaEventCreate(&a));
  CK(cudaEventCreate(&b));
  CK(cudaEventRecord(a, ctx->stream));
  for (int s = 0; s < n_steps; ++s)
    if (int r = launch_step(ctx)) return r;
  CK(cudaEventRecord(b, ctx->stream));
  CK(cudaEventSynchronize(b));
  float t = 0;
  CK(cudaEventElapsedTime(&t, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  *ms = t;
  return OSTC_OK;
}

int ostc_step_kernel_count(ostc_ctx *ctx, int *n) {
  if (!ctx || !n) return OSTC_EINVAL;
  cudaSetDevice(ctx->device);
  if (int r = check_ready(ctx)) return r;
  if (int r = ensure_graph(ctx)) return r;
  *n = ctx->graph_kernels;
  return OSTC_OK;
}

int ostc_physical_time(ostc_ctx *ctx, double *t) {
  if (!ctx || !t) return OSTC_EINVAL;
  cudaSetDevice(ctx->device);
  CK(cudaMemcpyAsync(t, ctx->d_time, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return OSTC_OK;
}

int ostc_store_residual_reference(ostc_ctx *ctx) {
  if (!ctx) return OSTC_EINVAL;
  cudaSetDevice(ctx->device);
  if (int r = check_ready(ctx)) return r;
  for (auto &B : ctx->blk)
    k_store_last<<<grid_for(ctx, B.db.n, 256), 256, 0, ctx->stream>>>(B.db, state_of(B, 0), B.last);
  CK(cudaGetLastError());
  return OSTC_OK;
}

int ostc_residual(ostc_ctx *ctx, double res[4]) {
  if (!ctx || !res) return OSTC_EINVAL;
  cudaSetDevice(ctx->device);
  if (int r = check_ready(ctx)) return r;
  CK(cudaMemsetAsync(ctx->d_sums, 0, 4 * sizeof(double), ctx->stream));
  long long tot = 0;
  for (auto &B : ctx->blk) {
    k_residual<<<grid_for(ctx, B.db.n, 256), 256, 0, ctx->stream>>>(B.db, state_of(B, 0), B.last, ctx->d_sums);
    tot += B.db.n;
  }
  CK(cudaGetLastError());
  double h[4];
  CK(cudaMemcpyAsync(h, ctx->d_sums, 4 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  for (int l = 0; l < 4; ++l) res[l] = std::sqrt(h[l] / (double)tot);
  return OSTC_OK;
}

// One steady (dt_phys = 0) or dual-time inner iteration: replayed from a captured graph (captured on
// first use per precision and physical dt), or launched kernel by kernel while timing or in the
// per-block launch mode.
static int steady_iteration(ostc_ctx *ctx, double dt_phys) {
  const bool mixed = ctx->precision == OSTC_PREC_MIXED;
  if (ctx->timing || ctx->launch_mode == OSTC_LAUNCH_BLOCK_LOOP)
    return mixed ? enqueue_steady_iteration<float>(ctx, dt_phys) : enqueue_steady_iteration<double>(ctx, dt_phys);
  const int key = (mixed ? 2 : 0) + (dt_phys > 0.0 ? 1 : 0);
  if (!ctx->steady_graph || ctx->steady_key != key || ctx->steady_dt != dt_phys) {
    if (ctx->steady_graph) {
      cudaGraphExecDestroy(ctx->steady_graph);
      ctx->steady_graph = nullptr;
    }
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    const int r = mixed ? enqueue_steady_iteration<float>(ctx, dt_phys) : enqueue_steady_iteration<double>(ctx, dt_phys);
    const cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
    if (r) return r;
    CK(e);
    const cudaError_t ei = cudaGraphInstantiate(&ctx->steady_graph, g, 0);
    cudaGraphDestroy(g);
    CK(ei);
    ctx->steady_key = key;
    ctx->steady_dt = dt_phys;
  }
  CK(cudaGraphLaunch(ctx->steady_graph, ctx->stream));
  return OSTC_OK;
}

int ostc_steady_step(ostc_ctx *ctx, int max_iter, int *iters_done, double *err_max) {
  if (!ctx || max_iter < 0) return OSTC_EINVAL;
  cudaSetDevice(ctx->device);
  if (int r = check_ready(ctx)) return r;
  if (int r = steady_alloc(ctx)) return r;
  const int screen = std::max(1, ctx->der.output_screen);
  int done = 0;
  double err = -1;
  for (int it = 0; it < max_iter; ++it) {
    const long long step = ctx->steady_iter + 1;
    const bool check = step == 1 || step % screen == 0;
    // store_last_step before the iteration whose change is measured (SteadySim.cuh:52-53, 72-76)
    if (check)
      for (auto &B : ctx->blk)
        k_store_last<<<grid_for(ctx, B.db.n, 256), 256, 0, ctx->stream>>>(B.db, state_of(B, 0), B.last);
    if (int r = steady_iteration(ctx, 0.0)) return r;
    ctx->steady_iter = step;
    ++done;
    if (check) {
      // compute_residual (Residual.cuh:74-190): RMS changes scaled by those of the first iteration
      double res[4];
      if (int rr = ostc_residual(ctx, res)) return rr;
      if (step == 1)
        for (int l = 0; l < 4; ++l) ctx->res_scale[l] = res[l] < 1e-20 ? 1e-20 : res[l];
      err = res[0] / ctx->res_scale[0];
      for (int l = 1; l < 4; ++l) err = std::max(err, res[l] / ctx->res_scale[l]);
      if (std::isnan(err)) {
        ctx->err = "the steady residual is NaN";
        if (iters_done) *iters_done = done;
        return OSTC_ENUMERIC;
      }
      if (err < ctx->der.convergence_criteria) break;
    }
  }
  CK(cudaStreamSynchronize(ctx->stream));
  if (iters_done) *iters_done = done;
  if (err_max) *err_max = err;
  return OSTC_OK;
}

int ostc_dual_time_step(ostc_ctx *ctx, int n_steps, int *inner_iters) {
  if (!ctx || n_steps < 0) return OSTC_EINVAL;
  if (!(ctx->der.dt > 0.0)) {
    ctx->err = "dual time stepping needs a positive physical step dt in the setup";
    return OSTC_EINVAL;
  }
  cudaSetDevice(ctx->device);
  if (int r = check_ready(ctx)) return r;
  if (int r = steady_alloc(ctx, true)) return r;
  const double dt = ctx->der.dt;
  const int nv = ctx->nv;
  if (ctx->dual_inner < 0) {
    // the previous physical step's state starts as the initial one (DualTimeStepping.cuh:64-72)
    for (auto &B : ctx->blk)
      CK(cudaMemcpyAsync(B.qn1, B.cv[0], (size_t)nv * B.db.plane * sizeof(double), cudaMemcpyDeviceToDevice,
                         ctx->stream));
    ctx->dual_inner = ctx->der.inner_iteration;
  }
  CK(cudaMemcpyAsync(ctx->d_dt, &dt, sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  for (int s = 0; s < n_steps; ++s) {
    const long long step = ++ctx->dual_step;
    for (auto &B : ctx->blk) {
      k_qn_star<<<grid_for(ctx, B.db.n, 128), 128, 0, ctx->stream>>>(B.db, state_of(B, 0), B.qn1, B.qstar, nv, dt);
      CK(cudaMemcpyAsync(B.qn1, B.cv[0], (size_t)nv * B.db.plane * sizeof(double), cudaMemcpyDeviceToDevice,
                         ctx->stream));
    }
    const bool monitor = ctx->der.iteration_adjust_step > 0 && step % ctx->der.iteration_adjust_step == 0;
    for (int iter = 1; iter <= ctx->dual_inner; ++iter) {
      // store_last_iter: the residual reference of ostc_residual holds the inner iterate
      if (monitor)
        for (auto &B : ctx->blk)
          k_store_last<<<grid_for(ctx, B.db.n, 256), 256, 0, ctx->stream>>>(B.db, state_of(B, 0), B.last);
      if (int r = steady_iteration(ctx, dt)) return r;
      if (monitor) {
        // inner_converged (DualTimeStepping.cu:32-135)
        double res[4];
        if (int rr = ostc_residual(ctx, res)) return rr;
        if (iter == 1)
          for (int l = 0; l < 4; ++l) ctx->res_scale_inner[l] = res[l] < 1e-20 ? 1e-20 : res[l];
        double err = res[0] / ctx->res_scale_inner[0];
        for (int l = 1; l < 4; ++l) err = std::max(err, res[l] / ctx->res_scale_inner[l]);
        if (std::isnan(err)) {
          ctx->err = "NaN in the inner iterations of dual time stepping";
          return OSTC_ENUMERIC;
        }
        if (iter == ctx->dual_inner && err > 1e-3 && ctx->dual_inner < ctx->der.max_inner_iteration)
          ctx->dual_inner = std::min(ctx->dual_inner + 5, ctx->der.max_inner_iteration);
        if (err < 1e-3) {
          if (ctx->dual_inner - iter > 0) ctx->dual_inner = iter;
          break;
        }
      }
    }
    k_step_end<<<1, 1, 0, ctx->stream>>>(ctx->d_time, ctx->d_dt, ctx->d_step);
    if (int r = stat_after_step(ctx)) return r;
  }
  CK(cudaStreamSynchronize(ctx->stream));
  if (inner_iters) *inner_iters = ctx->dual_inner;
  return OSTC_OK;
}

int ostc_bounds_flags(ostc_ctx *ctx, unsigned *flags) {
  if (!ctx || !flags) return OSTC_EINVAL;
  cudaSetDevice(ctx->device);
  CK(cudaStreamSynchronize(ctx->stream));
  CK(cudaMemcpyFromSymbol(flags, g_ostc_bounds, sizeof(unsigned)));
  const unsigned zero = 0;
  CK(cudaMemcpyToSymbol(g_ostc_bounds, &zero, sizeof(unsigned)));
  return OSTC_OK;
}

int ostc_bounds_checked(void) {
#ifdef OSTC_BOUNDS_CHECK
  return 1;
#else
  return 0;
#endif
}

}  // extern "C"
