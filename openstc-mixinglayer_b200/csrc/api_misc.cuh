// api_misc.cuh -- C ABI (include/ostc.h): device flags, zone views, case probing, sweep
// variants, the autotuner report and per-kernel-family step profiles.
// Part of the ostc_b200.cu translation unit (included in order; not a standalone header).
#pragma once

extern "C" {

int ostc_error_flags(ostc_ctx *ctx, unsigned *flags) {
  if (!ctx || !flags) return OSTC_EINVAL;
  cudaSetDevice(ctx->device);
  CK(cudaMemcpyAsync(flags, ctx->d_flags, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemsetAsync(ctx->d_flags, 0, sizeof(unsigned), ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return OSTC_OK;
}

int ostc_device_view(ostc_ctx *ctx, int block, ostc_zone_view *v) {
  if (!ctx || !v || block < 0 || block >= (int)ctx->blk.size()) return OSTC_EINVAL;
  BlockRes &B = ctx->blk[block];
  const DevBlock &b = B.db;
  v->mx = b.mx;
  v->my = b.my;
  v->mz = b.mz;
  v->ngg = b.g;
  v->gz = b.gz;
  v->pitch = b.pitch;
  v->sy = b.sy;
  v->sz = b.sz;
  v->plane = b.plane;
  v->cv = B.cv[0];
  v->bv = B.bv[0];
  v->mul = B.mul[0];
  v->metric = B.met;
  v->jac = B.jac;
  return OSTC_OK;
}

int ostc_probe_case(const char *setup_txt, const char *input_dir, int out[16], char *msg, int msg_len) {
  if (!input_dir || !out) return OSTC_EINVAL;
  Setup setup;
  setup.set_defaults();
  Derived der;
  HostMesh mesh;
  std::string err;
  const std::string dir(input_dir);
  const std::string sp = setup_txt && *setup_txt ? std::string(setup_txt) : dir + "/setup.txt";
  int rc = OSTC_OK;
  if (!setup.read_file(sp, err)) rc = OSTC_EIO;
  else if (!derive(setup, der, err)) rc = OSTC_EINVAL;
  else if (!read_mesh(dir, der, mesh, err)) rc = err.find("cannot open") != std::string::npos ? OSTC_EIO : OSTC_EINVAL;
  else if (!resolve_boundaries(setup, der, mesh, err)) rc = OSTC_EINVAL;
  ChemTables chem;
  if (rc == OSTC_OK && der.species == 1) {
    // the species count comes from the mechanism (Species ctor, ChemData.cpp:11-75)
    auto str = [&](const char *k) {
      auto it = setup.strings.find(k);
      return it == setup.strings.end() ? std::string() : it->second;
    };
    if (!read_chemistry(dir, str("mechanism_file"), str("therm_file"), str("transport_file"), der.reaction == 1, chem,
                        err)) {
      rc = err.find("cannot open") != std::string::npos ? OSTC_EIO : OSTC_EINVAL;
    } else {
      der.n_spec = der.n_scalar = chem.n_spec;
      der.n_var = 5 + chem.n_spec;
    }
  }
  // the inflow states (mixing-layer streams included) resolve on the host too
  if (rc == OSTC_OK && !resolve_inflows(setup, der.species == 1 ? &chem : nullptr, mesh, err)) rc = OSTC_EINVAL;
  if (rc != OSTC_OK) {
    if (msg && msg_len > 0) {
      std::strncpy(msg, err.c_str(), (size_t)msg_len - 1);
      msg[msg_len - 1] = 0;
    }
    return rc;
  }
  const auto order = bc_order(setup, mesh);
  const HostBlock &B = mesh.blocks[0];
  const int vals[14] = {der.ngg, der.inviscid_type, der.n_var, der.n_scalar, (int)mesh.blocks.size(), mesh.dimension,
                        B.mx, B.my, B.mz, (int)B.faces.size(), der.reconstruction, der.inviscid_scheme,
                        der.viscous_order, (int)order.size()};
  for (int i = 0; i < 14; ++i) out[i] = vals[i];
  return OSTC_OK;
}

int ostc_set_sweep_variant(ostc_ctx *ctx, int precision, int dir, int variant) {
  if (!ctx) return OSTC_EINVAL;
  if (precision < 0 || precision > 1 || dir < 0 || dir > 2) {
    ctx->err = "ostc_set_sweep_variant: precision must be 0/1 and dir 0/1/2";
    return OSTC_EINVAL;
  }
  if (variant < -1 || variant >= (dir == 0 ? kXVariants : kYzVariants)) {
    ctx->err = "ostc_set_sweep_variant: variant " + std::to_string(variant) + " outside -1.." +
               std::to_string((dir == 0 ? kXVariants : kYzVariants) - 1);
    return OSTC_EINVAL;
  }
  ctx->forced[precision][dir] = variant;
  // the next step tunes again (keeping pinned directions) and captures a new step graph
  ctx->tuned[precision] = false;
  if (ctx->graph) {
    cudaGraphExecDestroy(ctx->graph);
    ctx->graph = nullptr;
  }
  if (ctx->steady_graph) {
    cudaGraphExecDestroy(ctx->steady_graph);
    ctx->steady_graph = nullptr;
  }
  if (variant < 0) {
    std::lock_guard<std::mutex> lk(g_tune_mutex);
    for (auto &B : ctx->blk) {
      const TuneKey key{ctx->device, B.db.mx, B.db.my, B.db.mz, B.db.g, ctx->der.riemann, ctx->der.inviscid_type,
                        precision, dir};
      g_tune_cache.erase(key);
    }
  }
  return OSTC_OK;
}

int ostc_tune_report(ostc_ctx *ctx, int block, int precision, int dir, int *chosen, float *ms, int max) {
  if (!ctx || block < 0 || block >= (int)ctx->blk.size() || precision < 0 || precision > 1 || dir < 0 || dir > 2)
    return OSTC_EINVAL;
  const BlockRes &B = ctx->blk[block];
  if (chosen) *chosen = dir == 0 ? B.x_var[precision] : B.yz_var[precision][dir - 1];
  const int n = std::min(max, dir == 0 ? kXVariants : kYzVariants);
  for (int v = 0; v < n && ms; ++v) ms[v] = B.tune_ms[precision][dir][v];
  return dir == 0 ? kXVariants : kYzVariants;
}

int ostc_profile_steps(ostc_ctx *ctx, int n_steps, int max, const char **names, int *launches, double *ms) {
  if (!ctx || n_steps < 0) return OSTC_EINVAL;
  cudaSetDevice(ctx->device);
  if (int r = check_ready(ctx)) return r;
  ctx->fams.clear();
  ctx->ev_used.clear();
  ctx->timing = true;
  for (int s = 0; s < n_steps; ++s) {
    enqueue_step_any(ctx);
    if (int r = stat_after_step(ctx)) {
      ctx->timing = false;
      return r;
    }
  }
  ctx->timing = false;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->stream));
  for (auto &u : ctx->ev_used) {
    float t = 0;
    cudaEventElapsedTime(&t, ctx->ev_pool[u.second].first, ctx->ev_pool[u.second].second);
    ctx->fams[u.first].ms += t;
    ctx->fams[u.first].launches += 1;
  }
  const int n = std::min<int>(max, (int)ctx->fams.size());
  for (int i = 0; i < n; ++i) {
    if (names) names[i] = ctx->fams[i].name;
    if (launches) launches[i] = ctx->fams[i].launches;
    if (ms) ms[i] = ctx->fams[i].ms;
  }
  return n;
}

}  // extern "C"
