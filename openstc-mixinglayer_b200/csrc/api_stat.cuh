// api_stat.cuh -- C ABI (include/ostc.h): single-point statistics (SinglePointStat): group
// layout and names, accumulator set-up, collection after a step, export and import of the
// reference's coll_*.bin / tke_budget.bin / species_*.bin files.
// Part of the ostc_b200.cu translation unit (included in order; not a standalone header).
#pragma once

extern "C" {

// ---------------------------------------------------------------- single-point statistics

// Variable names of the four groups as the reference writes them (SinglePointStat.h:30-38,
// init_stat_name SinglePointStat.cu:98-147).
static std::vector<std::string> stat_names(const ostc_ctx *ctx, int g) {
  const StatSpec &sp = ctx->stat_spec;
  std::vector<std::string> v;
  if (g == 0) {
    v = {"rho", "p"};
    for (int l = 0; l < sp.n_rey; ++l) {
      const int q = sp.rey_idx[l];
      v.push_back(q == 1 ? "u" : q == 2 ? "v" : q == 3 ? "w" : "T");
    }
  } else if (g == 1) {
    v = {"rhoU", "rhoV", "rhoW", "rhoT"};
    for (int l = 0; l < sp.ns; ++l) v.push_back("rho" + ctx->chem.names[l]);
  } else if (g == 2) {
    v = {"RhoRho", "pp"};
    if (sp.rho_p) v.push_back("rhoP");
  } else if (g == 3) {
    v = {"rhoUU", "rhoVV", "rhoWW", "rhoUV", "rhoUW", "rhoVW", "rhoTT"};
    for (int l = 0; l < sp.ns; ++l) v.push_back("rho" + ctx->chem.names[l] + ctx->chem.names[l]);
  } else if (g == 4) {
    // TkeBudget::collect_name (TkeBudget.cuh:9-12)
    if (sp.tke) v = {"Tau11", "Tau12", "Tau13", "Tau22", "Tau23", "Tau33", "TauIjDUiDXj"};
  } else {
    // SpeciesVelocityCorrelation / SpeciesDissipationRate::collect_name with the species name appended,
    // species outer (create_species_collect_file, SpeciesStat.cuh:176-205)
    static const char *const kSvc[3] = {"rhoUY", "rhoVY", "rhoWY"};
    static const char *const kSdr[5] = {"rhoDdYDxdYDx", "rhoDdYDx", "rhoDdYDy", "rhoDdYDz", "rhoD"};
    if (stat_group_vars(sp, g) > 0)
      for (int q = 0; q < sp.nss; ++q)
        for (int c = 0; c < (g == 5 ? 3 : 5); ++c)
          v.push_back(std::string(g == 5 ? kSvc[c] : kSdr[c]) + ctx->chem.names[sp.ss_idx[q]]);
  }
  return v;
}

static long long stat_block_doubles(const ostc_ctx *ctx, const BlockRes &B) {
  return stat_group_offset(ctx->stat_spec, B.db, kStatGroups);
}

static void stat_free(ostc_ctx *ctx) {
  for (auto &B : ctx->blk) {
    cudaFree(B.stat);
    B.stat = nullptr;
  }
  ctx->stat_on = false;
}

// (Re)allocate and zero the accumulators for the selection rey_idx (primitive indices of the extra
// Reynolds averages, in the order given), rho_p and the additional collectors.
static int stat_setup(ostc_ctx *ctx, int start_step, const std::vector<int> &rey_idx, bool rho_p,
                      const StatExtras &ex) {
  if (start_step < 0 || rey_idx.size() > 4) {
    ctx->err = "ostc_stat_enable: start_step must be >= 0 and at most 4 extra Reynolds averages";
    return OSTC_EINVAL;
  }
  if (ex.ss_idx.size() > 16) {
    ctx->err = "ostc_stat_enable: at most 16 species for the species statistics";
    return OSTC_EINVAL;
  }
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  stat_free(ctx);
  StatSpec sp{};
  sp.n_rey = (int)rey_idx.size();
  for (int l = 0; l < sp.n_rey; ++l) sp.rey_idx[l] = rey_idx[l];
  sp.rho_p = rho_p ? 1 : 0;
  sp.ns = ctx->der.n_spec;
  sp.tke = ex.tke ? 1 : 0;
  // the species collectors need species to collect (SinglePointStat.cu:87-96)
  sp.nss = (int)ex.ss_idx.size();
  sp.svc = ex.svc && sp.nss > 0 ? 1 : 0;
  sp.sdr = ex.sdr && sp.nss > 0 ? 1 : 0;
  for (int q = 0; q < sp.nss; ++q) sp.ss_idx[q] = ex.ss_idx[q];
  ctx->stat_spec = sp;
  for (auto &B : ctx->blk)
    if (stat_points(B.db) >= (1LL << 31)) {
      ctx->err = "ostc_stat_enable: a block with 2^31 or more points (ghost layer included) is not supported";
      return OSTC_EINVAL;
    }
  for (auto &B : ctx->blk) {
    const size_t bytes = (size_t)stat_block_doubles(ctx, B) * sizeof(double);
    if (cudaMalloc(&B.stat, bytes) != cudaSuccess) {
      stat_free(ctx);
      ctx->err = "ostc_stat_enable: device allocation of the statistics accumulators failed";
      return OSTC_ENOMEM;
    }
    CK(cudaMemsetAsync(B.stat, 0, bytes, ctx->stream));
  }
  ctx->stat_on = true;
  ctx->stat_start = start_step;
  ctx->stat_steps = 0;
  ctx->stat_count = 0;
  return OSTC_OK;
}

// After one step on the context stream: count it and, past the start step, accumulate every block
// (SinglePointStat::collect_data, SinglePointStat.cu:515-551).
static int stat_after_step(ostc_ctx *ctx) {
  if (!ctx->stat_on) return OSTC_OK;
  if (++ctx->stat_steps <= ctx->stat_start) return OSTC_OK;
  const StatSpec &sp = ctx->stat_spec;
  for (auto &B : ctx->blk) {
    long tok = begin_t(ctx, "statistics");
    k_stat_collect<<<grid_for(ctx, stat_points(B.db), 256), 256, 0, ctx->stream>>>(B.db, state_of(B, 0), B.stat, sp);
    if (sp.tke || sp.svc || sp.sdr)
      k_stat_extra<<<grid_for(ctx, B.db.n, 128), 128, 0, ctx->stream>>>(B.db, state_of(B, 0),
                                                                         B.stat + stat_group_offset(sp, B.db, 4), sp);
    end_t(ctx, tok);
  }
  CK(cudaGetLastError());
  ++ctx->stat_count;
  return OSTC_OK;
}

static const char *const kStatFiles[kStatGroups] = {"coll_rey_1st.bin", "coll_fav_1st.bin", "coll_rey_2nd.bin",
                                                    "coll_fav_2nd.bin", "tke_budget.bin",
                                                    "species_velocity_correlation.bin",
                                                    "species_dissipation_rate.bin"};

int ostc_stat_enable(ostc_ctx *ctx, int start_step, unsigned flags) {
  if (!ctx) return OSTC_EINVAL;
  if (flags & ~255u) {
    ctx->err = "ostc_stat_enable: unknown flag bits";
    return OSTC_EINVAL;
  }
  cudaSetDevice(ctx->device);
  std::vector<int> idx;
  if (flags & OSTC_STAT_REY_U) idx.push_back(1);
  if (flags & OSTC_STAT_REY_V) idx.push_back(2);
  if (flags & OSTC_STAT_REY_W) idx.push_back(3);
  if (flags & OSTC_STAT_REY_T) idx.push_back(5);
  StatExtras ex;
  ex.tke = (flags & OSTC_STAT_TKE_BUDGET) != 0;
  ex.svc = (flags & OSTC_STAT_SPECIES_VELOCITY) != 0;
  ex.sdr = (flags & OSTC_STAT_SPECIES_DISSIPATION) != 0;
  for (int l = 0; l < ctx->der.n_spec; ++l) ex.ss_idx.push_back(l);  // every species ("all")
  return stat_setup(ctx, start_step, idx, (flags & OSTC_STAT_RHO_P) != 0, ex);
}

int ostc_stat_disable(ostc_ctx *ctx) {
  if (!ctx) return OSTC_EINVAL;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  stat_free(ctx);
  return OSTC_OK;
}

int ostc_stat_info(ostc_ctx *ctx, int n_var[4], int *n_collected, long long *steps) {
  if (!ctx) return OSTC_EINVAL;
  if (!ctx->stat_on) {
    ctx->err = "statistics collection is off (ostc_stat_enable, or if_collect_statistics in the setup)";
    return OSTC_ESTATE;
  }
  for (int g = 0; g < 4 && n_var; ++g) n_var[g] = stat_group_vars(ctx->stat_spec, g);
  if (n_collected) *n_collected = ctx->stat_count;
  if (steps) *steps = ctx->stat_steps;
  return OSTC_OK;
}

int ostc_stat_group_vars(ostc_ctx *ctx, int group, int *n_var) {
  if (!ctx || !n_var || group < 0 || group >= kStatGroups) return OSTC_EINVAL;
  if (!ctx->stat_on) {
    ctx->err = "statistics collection is off (ostc_stat_enable, or if_collect_statistics in the setup)";
    return OSTC_ESTATE;
  }
  *n_var = stat_group_vars(ctx->stat_spec, group);
  return OSTC_OK;
}

int ostc_stat_get(ostc_ctx *ctx, int block, int group, double *out, int ptr_kind) {
  if (!ctx || !out || block < 0 || block >= (int)ctx->blk.size() || group < 0 || group >= kStatGroups)
    return OSTC_EINVAL;
  if (!ctx->stat_on) {
    ctx->err = "statistics collection is off (ostc_stat_enable, or if_collect_statistics in the setup)";
    return OSTC_ESTATE;
  }
  cudaSetDevice(ctx->device);
  const BlockRes &B = ctx->blk[block];
  const long long off = stat_group_offset(ctx->stat_spec, B.db, group);
  const size_t bytes = (size_t)stat_group_vars(ctx->stat_spec, group) * stat_group_points(B.db, group) * sizeof(double);
  if (bytes == 0) return OSTC_OK;
  CK(cudaMemcpyAsync(out, B.stat + off, bytes, ptr_kind == OSTC_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                     ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return OSTC_OK;
}

int ostc_stat_export(ostc_ctx *ctx, const char *dir) {
  if (!ctx || !dir) return OSTC_EINVAL;
  if (!ctx->stat_on) {
    ctx->err = "statistics collection is off (ostc_stat_enable, or if_collect_statistics in the setup)";
    return OSTC_ESTATE;
  }
  cudaSetDevice(ctx->device);
  CK(cudaStreamSynchronize(ctx->stream));
  std::vector<double> host;
  for (int g = 0; g < kStatGroups; ++g) {
    const int nvar = stat_group_vars(ctx->stat_spec, g);
    if (g >= 4 && nvar == 0) continue;  // an additional collector that is off writes no file
    const std::string path = std::string(dir) + "/" + kStatFiles[g];
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) {
      ctx->err = "ostc_stat_export: cannot open " + path + " for writing";
      return OSTC_EIO;
    }
    bool ok = true;
    auto put_i = [&](int v) { ok = ok && std::fwrite(&v, 4, 1, f) == 1; };
    put_i((int)ctx->blk.size());
    put_i(nvar);
    put_i(g < 4 ? 1 : 0);  // ghost layers of the group's arrays
    for (const auto &name : stat_names(ctx, g)) {
      for (char c : name) put_i((int)c);
      put_i(0);
    }
    for (int v = 0; v < nvar; ++v) put_i(ctx->stat_count);
    for (const auto &B : ctx->blk) {
      put_i(B.db.mx);
      put_i(B.db.my);
      put_i(B.db.mz);
      const long long np = stat_group_points(B.db, g);
      host.resize((size_t)nvar * np);
      if (cudaMemcpy(host.data(), B.stat + stat_group_offset(ctx->stat_spec, B.db, g), host.size() * sizeof(double),
                     cudaMemcpyDeviceToHost) != cudaSuccess) {
        std::fclose(f);
        ctx->err = "ostc_stat_export: device copy failed";
        return OSTC_ECUDA;
      }
      ok = ok && std::fwrite(host.data(), sizeof(double), host.size(), f) == host.size();
    }
    if (std::fclose(f) != 0 || !ok) {
      ctx->err = "ostc_stat_export: write to " + path + " failed";
      return OSTC_EIO;
    }
  }
  return OSTC_OK;
}

int ostc_stat_import(ostc_ctx *ctx, const char *dir) {
  if (!ctx || !dir) return OSTC_EINVAL;
  if (!ctx->stat_on) {
    ctx->err = "statistics collection is off (ostc_stat_enable, or if_collect_statistics in the setup)";
    return OSTC_ESTATE;
  }
  cudaSetDevice(ctx->device);
  CK(cudaStreamSynchronize(ctx->stream));
  // read and check every file of the selection before touching the accumulators
  std::vector<std::vector<double>> data(kStatGroups * ctx->blk.size());
  int count = -1;
  for (int g = 0; g < kStatGroups; ++g) {
    const int nvar = stat_group_vars(ctx->stat_spec, g);
    if (g >= 4 && nvar == 0) continue;
    const std::string path = std::string(dir) + "/" + kStatFiles[g];
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) {
      ctx->err = "ostc_stat_import: cannot open " + path;
      return OSTC_EIO;
    }
    std::string why;
    auto get_i = [&](int &v) { return std::fread(&v, 4, 1, f) == 1; };
    int nb = 0, nv = 0, ngg = 0;
    if (!get_i(nb) || !get_i(nv) || !get_i(ngg)) why = "truncated header";
    else if (nb != (int)ctx->blk.size() || nv != nvar || ngg != (g < 4 ? 1 : 0))
      why = "header (n_block " + std::to_string(nb) + ", n_var " + std::to_string(nv) + ", ngg " +
            std::to_string(ngg) + ") does not match the case and the enabled selection";
    for (const auto &name : stat_names(ctx, g)) {
      if (!why.empty()) break;
      std::string got;
      int c = 0;
      while (get_i(c) && c != 0 && got.size() < 256) got.push_back((char)c);
      if (got != name) why = "variable '" + got + "' where '" + name + "' was expected";
    }
    for (int v = 0; v < nvar && why.empty(); ++v) {
      int c = 0;
      if (!get_i(c)) why = "truncated counters";
      else if (c < 0 || (count >= 0 && c != count)) why = "counters differ between variables or files";
      else count = c;
    }
    for (size_t b = 0; b < ctx->blk.size() && why.empty(); ++b) {
      const DevBlock &db = ctx->blk[b].db;
      int mx = 0, my = 0, mz = 0;
      if (!get_i(mx) || !get_i(my) || !get_i(mz)) why = "truncated block header";
      else if (mx != db.mx || my != db.my || mz != db.mz)
        why = "block " + std::to_string(b) + " extents differ from the case";
      else {
        auto &d = data[g * ctx->blk.size() + b];
        d.resize((size_t)nvar * stat_group_points(db, g));
        if (std::fread(d.data(), sizeof(double), d.size(), f) != d.size()) why = "truncated data";
      }
    }
    std::fclose(f);
    if (!why.empty()) {
      ctx->err = "ostc_stat_import: " + path + ": " + why;
      return OSTC_EIO;
    }
  }
  for (size_t b = 0; b < ctx->blk.size(); ++b)
    for (int g = 0; g < kStatGroups; ++g) {
      const auto &d = data[g * ctx->blk.size() + b];
      if (d.empty()) continue;
      CK(cudaMemcpy(ctx->blk[b].stat + stat_group_offset(ctx->stat_spec, ctx->blk[b].db, g), d.data(),
                    d.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
  ctx->stat_count = count < 0 ? 0 : count;
  // a continued collection (the reference's step index runs on across the restart): collect from the
  // next step on
  ctx->stat_steps = std::max<long long>(ctx->stat_steps, ctx->stat_start);
  return OSTC_OK;
}

}  // extern "C"
