// api_core.cuh -- C ABI (include/ostc.h): context creation and teardown, state in and out, the
// right-hand side, the adjoint entry points and the pipelined ostc_run_states.
// Part of the ostc_b200.cu translation unit (included in order; not a standalone header).
#pragma once

extern "C" {

// The additional collectors of a statistics selection: the TKE budget, and for the species ss_idx
// (indices into the mechanism) their velocity correlation and dissipation rate.
struct StatExtras {
  bool tke = false, svc = false, sdr = false;
  std::vector<int> ss_idx;
};
static int stat_setup(ostc_ctx *ctx, int start_step, const std::vector<int> &rey_idx, bool rho_p,
                      const StatExtras &ex = StatExtras());

int ostc_create(const char *setup_txt, const char *input_dir, int device, ostc_ctx **out) {
  if (!out || !input_dir) {
    g_create_error = "ostc_create: null argument";
    return OSTC_EINVAL;
  }
  *out = nullptr;
  auto ctx = std::make_unique<ostc_ctx>();
  ctx->device = device;
  ctx->setup.set_defaults();
  std::string err;
  const std::string dir(input_dir);
  const std::string sp = setup_txt && *setup_txt ? std::string(setup_txt) : dir + "/setup.txt";
  if (!ctx->setup.read_file(sp, err) || !derive(ctx->setup, ctx->der, err) ||
      !read_mesh(dir, ctx->der, ctx->mesh, err) || !resolve_boundaries(ctx->setup, ctx->der, ctx->mesh, err)) {
    g_create_error = err;
    return err.find("cannot open") != std::string::npos || err.find("grid file") != std::string::npos ||
                   err.find("file:") != std::string::npos
               ? OSTC_EIO
               : OSTC_EINVAL;
  }
  ctx->order = bc_order(ctx->setup, ctx->mesh);
  if (ctx->der.species == 1) {
    auto str = [&](const char *k) {
      auto it = ctx->setup.strings.find(k);
      return it == ctx->setup.strings.end() ? std::string() : it->second;
    };
    if (!read_chemistry(dir, str("mechanism_file"), str("therm_file"), str("transport_file"), ctx->der.reaction == 1,
                        ctx->chem, err)) {
      g_create_error = err;
      return err.find("cannot open") != std::string::npos ? OSTC_EIO : OSTC_EINVAL;
    }
    const ChemTables &c = ctx->chem;
    MixTables &m = ctx->mixtab;
    m.ns = c.n_spec;
    m.nr = c.n_reac;
    for (int i = 0; i < c.n_spec; ++i) {
      m.mw[i] = c.mw[i];
      m.imw[i] = 1.0 / c.mw[i];
      m.ru_mw[i] = kRu / c.mw[i];
      m.t_low[i] = c.t_low[i];
      m.t_mid[i] = c.t_mid[i];
      for (int q = 0; q < 7; ++q) {
        m.low[i][q] = c.low[i * 7 + q];
        m.high[i][q] = c.high[i * 7 + q];
      }
      m.lj_potent_inv[i] = c.lj_potent_inv[i];
      m.ln_lj[i] = std::log(c.lj_potent_inv[i]);
      m.vis_coeff[i] = c.vis_coeff[i];
      for (int j = 0; j < c.n_spec; ++j) {
        m.wj_div_wi_1_4[i][j] = c.wj_div_wi_1_4[i * c.n_spec + j];
        m.sqrt_wiwj_8[i][j] = c.sqrt_wiwj_8[i * c.n_spec + j];
        m.binary_diff[i][j] = c.binary_diff[i * c.n_spec + j];
        m.kb_over_eps[i][j] = c.kb_over_eps_jk[i * c.n_spec + j];
        // the diagonal (0) is never used
        m.ln_kbe[i][j] = m.kb_over_eps[i][j] > 0 ? std::log(m.kb_over_eps[i][j]) : 0.0;
      }
    }
    m.use_gibbs = 0;
    for (int r = 0; r < c.n_reac; ++r) {
      m.label[r] = c.label[r];
      m.rev_type[r] = c.rev_type[r];
      m.order[r] = c.order[r];
      if (c.label[r] != 0 && c.rev_type[r] != 1) m.use_gibbs = 1;
      m.A[r] = c.A[r];
      m.b[r] = c.b[r];
      m.Ea[r] = c.Ea[r];
      m.A2[r] = c.A2[r];
      m.b2[r] = c.b2[r];
      m.Ea2[r] = c.Ea2[r];
      m.troe_alpha[r] = c.troe_alpha[r];
      m.troe_t3[r] = c.troe_t3[r];
      m.troe_t1[r] = c.troe_t1[r];
      m.troe_t2[r] = c.troe_t2[r];
      for (int i = 0; i < c.n_spec; ++i) {
        m.stoi_f[r][i] = (signed char)c.stoi_f[r * c.n_spec + i];
        m.stoi_b[r][i] = (signed char)c.stoi_b[r * c.n_spec + i];
        m.third_body[r][i] = c.third_body[r * c.n_spec + i];
      }
    }
    ctx->mixture = true;
    ctx->nv = 5 + c.n_spec;
    ctx->der.n_spec = c.n_spec;
    ctx->der.n_scalar = c.n_spec;
    ctx->der.n_var = ctx->nv;
  }
  if (!resolve_inflows(ctx->setup, ctx->mixture ? &ctx->chem : nullptr, ctx->mesh, err)) {
    g_create_error = err;
    return OSTC_EINVAL;
  }
  if (ctx->der.inviscid_type == 3) {
    if (!reference_scales(ctx->setup, ctx->mixture ? &ctx->chem : nullptr, ctx->mixtab.weno_eps_scale,
                          ctx->mixtab.v_ref, err)) {
      g_create_error = err;
      return OSTC_EINVAL;
    }
    if (!ctx->mixture) {
      // air on the flux-split path: the tables carry only the epsilon scales
      ctx->mixtab.ns = 0;
      ctx->mixtab.nr = 0;
    }
  }
  ctx->tables = ctx->mixture || ctx->der.inviscid_type == 3;
  {
    auto di = ctx->setup.strings.find("default_init");
    if (di != ctx->setup.strings.end() && ctx->setup.structs.count(di->second)) {
      double c;
      std::string e2;
      ctx->has_init = inflow_state(ctx->setup, di->second, ctx->mixture ? &ctx->chem : nullptr, ctx->init_bv,
                                   ctx->init_sv, c, e2);
    }
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    g_create_error = "no CUDA device " + std::to_string(device) + " available";
    return OSTC_ECUDA;
  }
  if (cudaSetDevice(device) != cudaSuccess) {
    g_create_error = "cudaSetDevice failed";
    return OSTC_ECUDA;
  }
  cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device);
  if (!set_march_attrs<double>() || !set_march_attrs<float>() || !set_mix_attrs(ctx->nv)) {
    g_create_error = "cudaFuncSetAttribute (dynamic shared memory) failed";
    return OSTC_ECUDA;
  }
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
    g_create_error = "cudaStreamCreate failed";
    return OSTC_ECUDA;
  }
  if (ctx->mesh.blocks.size() > 1) {
    const size_t ns = std::min<size_t>(ctx->mesh.blocks.size(), 4);
    bool ok = cudaEventCreateWithFlags(&ctx->fork_ev, cudaEventDisableTiming) == cudaSuccess;
    for (size_t k = 0; k < ns && ok; ++k) {
      cudaStream_t st;
      cudaEvent_t ev;
      ok = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) == cudaSuccess;
      if (ok) ctx->side.push_back(st);
      ok = ok && cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) == cudaSuccess;
      if (ok) ctx->side_ev.push_back(ev);
    }
    if (!ok) {
      g_create_error = "cudaStreamCreate (block streams) failed";
      ostc_destroy(ctx.release());
      return OSTC_ECUDA;
    }
  }
  const bool is3d = ctx->mesh.dimension == 3;
  size_t max_n = 0;
  for (auto &HB : ctx->mesh.blocks) {
    BlockRes R;
    DevBlock &b = R.db;
    b.mx = HB.mx;
    b.my = HB.my;
    b.mz = HB.mz;
    b.g = HB.ngg;
    b.gz = is3d ? HB.ngg : 0;
    b.pitch = ((HB.mx + 2 * b.g) + 7) / 8 * 8;
    b.sy = HB.my + 2 * b.g;
    b.sz = HB.mz + 2 * b.gz;
    b.plane = (long long)b.pitch * b.sy * b.sz;
    b.off0 = ((long long)b.gz * b.sy + b.g) * b.pitch + b.g;
    b.n = (long long)HB.mx * HB.my * HB.mz;
    max_n = std::max<size_t>(max_n, (size_t)b.n);
    auto alloc = [&](double **p, size_t n) -> bool {
      if (cudaMalloc(p, n * sizeof(double)) != cudaSuccess) return false;
      return cudaMemset(*p, 0, n * sizeof(double)) == cudaSuccess;
    };
    const int nv = ctx->nv, ns = ctx->der.n_spec;
    bool ok = alloc(&R.met, 9 * b.plane) && alloc(&R.jac, b.plane) && alloc(&R.dq, (size_t)nv * b.n) &&
              alloc(&R.last, 4 * b.n);
    if (ok && ctx->mixture && ctx->der.inviscid_type != 3)
      ok = alloc(&R.fcb, (size_t)nv * (HB.mx + 1) * (HB.my + 1) * (HB.mz + 1)) && alloc(&R.efd, b.plane);
    for (int s = 0; s < 3 && ok; ++s) {
      ok = alloc(&R.cv[s], (size_t)nv * b.plane) && alloc(&R.bv[s], 6 * b.plane) && alloc(&R.mul[s], b.plane);
      if (ok && ctx->mixture)
        ok = alloc(&R.sv[s], (size_t)ns * b.plane) && alloc(&R.rhod[s], (size_t)ns * b.plane) &&
             alloc(&R.cond[s], b.plane) && alloc(&R.gam[s], b.plane) && alloc(&R.acs[s], b.plane);
    }
    if (!ok) {
      g_create_error = "device allocation failed";
      ctx->blk.push_back(R);
      ostc_destroy(ctx.release());
      return OSTC_ENOMEM;
    }
    // metric/Jacobian: host arrays have ngg ghosts in every direction; copy the device part
    std::vector<double> hm(9 * b.plane, 0.0), hj(b.plane, 0.0);
    const long HP = HB.padded();
    for (int k = -b.gz; k < b.mz + b.gz; ++k)
      for (int j = -b.g; j < b.my + b.g; ++j)
        for (int i = -b.g; i < b.mx + b.g; ++i) {
          const long long d = b.id(i, j, k);
          const long h = HB.gidx(i, j, k);
          hj[d] = HB.jac[h];
          for (int r = 0; r < 9; ++r) hm[r * b.plane + d] = HB.metric[r * HP + h];
        }
    cudaMemcpy(R.met, hm.data(), hm.size() * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(R.jac, hj.data(), hj.size() * sizeof(double), cudaMemcpyHostToDevice);
    b.met = R.met;
    b.jac = R.jac;
    b.met32 = nullptr;
    if (!ctx->mixture) {
      std::vector<float> h32(10 * b.plane);
      for (long long q = 0; q < 9 * b.plane; ++q) h32[q] = (float)hm[q];
      for (long long q = 0; q < b.plane; ++q) h32[9 * b.plane + q] = (float)hj[q];
      if (cudaMalloc(&R.met32, h32.size() * sizeof(float)) != cudaSuccess ||
          cudaMemcpy(R.met32, h32.data(), h32.size() * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) {
        g_create_error = "device allocation failed";
        ctx->blk.push_back(R);
        ostc_destroy(ctx.release());
        return OSTC_ENOMEM;
      }
      b.met32 = R.met32;
    }
    for (auto &hf : HB.faces) {
      DevFace f{};
      f.type = hf.type;
      f.face = hf.face;
      f.direction = hf.direction;
      for (int q = 0; q < 3; ++q) {
        f.rs[q] = hf.rs[q];
        f.re[q] = hf.re[q];
      }
      if (!is3d) {
        f.rs[2] = 0;
        f.re[2] = 0;
      }
      f.density = hf.density;
      f.u = hf.u;
      f.v = hf.v;
      f.w = hf.w;
      f.pressure = hf.pressure;
      f.temperature = hf.temperature;
      f.acoustic_speed = hf.acoustic_speed;
      f.gamma = hf.gamma;
      f.entropy = hf.entropy;
      f.mw = hf.mw;
      f.wall_adiabatic = hf.wall_adiabatic;
      for (size_t l = 0; l < hf.y.size() && l < 16; ++l) f.y[l] = hf.y[l];
      f.inflow_type = hf.inflow_type;
      f.fluct = hf.fluctuation_type;
      f.fluct_rms = hf.fluct_intensity;
      f.velocity = hf.velocity;
      f.delta_omega = hf.delta_omega;
      for (int l = 0; l < 6; ++l) f.lower[l] = hf.lower[l];
      for (size_t l = 0; l < hf.y_lower.size() && l < 16; ++l) f.y_lower[l] = hf.y_lower[l];
      f.rng_row = (f.face == 0 ? HB.my : HB.mx) + 2 * HB.ngg;
      double *fy = nullptr;
      if (hf.type == kInflow && hf.inflow_type == 2) {
        // y of every face node in k_bc_face's enumeration (tangential ranges padded by ngg)
        const int t0 = f.face == 0 ? 1 : 0, t1 = f.face == 2 ? 1 : 2;
        const int n0 = f.re[t0] - f.rs[t0] + 1, n1 = f.re[t1] - f.rs[t1] + 1;
        std::vector<double> hy((size_t)n0 * n1);
        for (int q = 0; q < n0 * n1; ++q) {
          int id3[3];
          id3[f.face] = f.rs[f.face];
          id3[t0] = f.rs[t0] + q % n0;
          id3[t1] = f.rs[t1] + q / n0;
          hy[q] = HB.y[HB.cidx(id3[0], id3[1], id3[2])];
        }
        if (cudaMalloc(&fy, hy.size() * sizeof(double)) != cudaSuccess) {
          g_create_error = "device allocation for the inflow coordinates failed";
          ctx->blk.push_back(R);
          ostc_destroy(ctx.release());
          return OSTC_ENOMEM;
        }
        cudaMemcpy(fy, hy.data(), hy.size() * sizeof(double), cudaMemcpyHostToDevice);
      }
      f.ycoord = fy;
      R.face_y.push_back(fy);
      R.faces.push_back(f);
    }
    for (auto &hi : HB.inner) {
      DevInner fi{};
      for (int q = 0; q < 3; ++q) {
        fi.rs[q] = hi.rs[q];
        fi.ts[q] = hi.ts[q];
        fi.loop_dir[q] = hi.loop_dir[q];
        fi.target_loop_dir[q] = hi.target_loop_dir[q];
        fi.src_tar[q] = hi.src_tar[q];
        fi.n_point[q] = hi.n_point[q];
      }
      fi.face = hi.face;
      fi.direction = hi.direction;
      // the coincident layer: the start of a high-side range, the end of a low-side one
      fi.face_index = hi.direction > 0 ? hi.rs[hi.face] : hi.re[hi.face];
      R.inner.push_back(fi);
      R.inner_target.push_back(hi.target_block);
    }
    ctx->blk.push_back(R);
  }
  ctx->block_set.assign(ctx->blk.size(), 0);
  bool ok = cudaMalloc(&ctx->d_dtbits, sizeof(unsigned long long)) == cudaSuccess &&
            cudaMalloc(&ctx->d_dt, sizeof(double)) == cudaSuccess && cudaMalloc(&ctx->d_time, sizeof(double)) == cudaSuccess &&
            cudaMalloc(&ctx->d_sums, 4 * sizeof(double)) == cudaSuccess &&
            cudaMalloc(&ctx->d_step, sizeof(long long)) == cudaSuccess &&
            cudaMalloc(&ctx->d_flags, sizeof(unsigned)) == cudaSuccess &&
            cudaMalloc(&ctx->d_staging, (size_t)std::max(6 + ctx->der.n_spec, ctx->nv) * max_n * sizeof(double)) == cudaSuccess;
  if (!ok) {
    g_create_error = "device allocation failed";
    ostc_destroy(ctx.release());
    return OSTC_ENOMEM;
  }
  if (ctx->der.problem_type == 1) {
    // the initial field of a mixing-layer problem is the two-stream profile at every node, ghosts
    // included (initialize_mixing_layer, Initialize.cu:228-326): y of every padded node
    std::string e2;
    if (!mixing_layer_streams(ctx->setup, ctx->mixture ? &ctx->chem : nullptr, ctx->ml, e2)) {
      g_create_error = e2;
      ostc_destroy(ctx.release());
      return OSTC_EINVAL;
    }
    for (size_t bi = 0; bi < ctx->blk.size(); ++bi) {
      BlockRes &R = ctx->blk[bi];
      const HostBlock &HB = ctx->mesh.blocks[bi];
      const DevBlock &b = R.db;
      std::vector<double> hy(b.plane, 0.0);
      for (int k = -b.gz; k < b.mz + b.gz; ++k)
        for (int j = -b.g; j < b.my + b.g; ++j)
          for (int i = -b.g; i < b.mx + b.g; ++i) hy[b.id(i, j, k)] = HB.y[HB.cidx(i, j, k)];
      if (cudaMalloc(&R.ycoord, hy.size() * sizeof(double)) != cudaSuccess) {
        g_create_error = "device allocation failed";
        ostc_destroy(ctx.release());
        return OSTC_ENOMEM;
      }
      cudaMemcpy(R.ycoord, hy.data(), hy.size() * sizeof(double), cudaMemcpyHostToDevice);
    }
  }
  {
    // white-noise inflows: generator states for the largest fluctuating face plane, ghost-padded by
    // ngg (BoundCond.cu:1706-1735), seeded from the clock as the reference does until
    // ostc_set_inflow_seed fixes the seed
    long long size = 0;
    int n_fluct = 0;
    for (size_t bi = 0; bi < ctx->blk.size(); ++bi) {
      const HostBlock &HB = ctx->mesh.blocks[bi];
      for (const auto &f : ctx->blk[bi].faces) {
        if (f.type != kInflow || f.fluct != 1) continue;
        ++n_fluct;
        const long long n1 = f.face == 0 ? HB.my : HB.mx, n2 = f.face == 2 ? HB.my : HB.mz;
        size = std::max(size, (n1 + 2 * HB.ngg) * (n2 + 2 * HB.ngg));
      }
    }
    int n_df = 0;
    for (size_t bi = 0; bi < ctx->blk.size(); ++bi)
      for (size_t fi = 0; fi < ctx->blk[bi].faces.size(); ++fi)
        if (ctx->blk[bi].faces[fi].type == kInflow && ctx->blk[bi].faces[fi].fluct == 11) {
          ++n_df;
          ctx->df_block = (int)bi;
          ctx->df_face = (int)fi;
        }
    if (n_fluct > 1 || n_df > 1 || (n_fluct && n_df)) {
      // the reference draws every white-noise face from one shared array, in face order, and supports
      // one digital-filter face; this library runs one fluctuating inflow face
      g_create_error = "more than one inflow face with fluctuation_type 1 is not provided";
      ostc_destroy(ctx.release());
      return OSTC_EINVAL;
    }
    if (n_df) {
      // DBoundCond::initialize_digital_filter (DigitalFilter.cu:8-247): buffers, the Lund matrix of the
      // Gaussian Reynolds stresses, the filter coefficients from the scaled y spacing and the mean z
      // spacing, then the first random field
      const HostBlock &HB = ctx->mesh.blocks[ctx->df_block];
      const BcFace &hf = HB.faces[ctx->df_face];
      DevDf &d = ctx->df;
      d.my = HB.my;
      d.mz = HB.mz;
      d.g = HB.ngg;
      d.wy = d.my + 2 * (kDfN + d.g);
      d.wz = d.mz + 2 * (kDfN + d.g);
      d.py = d.my + 2 * d.g;
      d.pz = d.mz + 2 * d.g;
      // DeltaU of write_reference_state (Driver.cu:252-276): the difference of the streams' speeds
      d.delta_u = std::fabs(std::sqrt(hf.u * hf.u + hf.v * hf.v + hf.w * hf.w) -
                            std::sqrt(hf.lower[1] * hf.lower[1] + hf.lower[2] * hf.lower[2] + hf.lower[3] * hf.lower[3]));
      if (ctx->mixture) {
        double a = 0, b2 = 0;
        for (int l = 0; l < ctx->der.n_spec; ++l) {
          a += hf.y[l] / ctx->chem.mw[l];
          b2 += hf.y_lower[l] / ctx->chem.mw[l];
        }
        ctx->df_mw_up = 1 / a;
        ctx->df_mw_lo = 1 / b2;
      }
      const long long ns = (long long)d.wy * d.wz * 3, nf = (long long)d.py * d.wz * 3,
                      np = (long long)d.py * d.pz;
      std::vector<double> ysc(d.py), yface((size_t)np);
      const double yref = hf.delta_omega;
      for (int j = -d.g; j < d.my + d.g; ++j) ysc[j + d.g] = HB.y[HB.cidx(0, j, 0)] / yref;
      for (int k = -d.g; k < d.mz + d.g; ++k)
        for (int j = -d.g; j < d.my + d.g; ++j) yface[(size_t)(k + d.g) * d.py + (j + d.g)] = HB.y[HB.cidx(0, j, k)];
      double dz = 0;
      for (int k = 1; k < d.mz; ++k) dz += HB.z[HB.cidx(0, 0, k)] - HB.z[HB.cidx(0, 0, k - 1)];
      dz /= d.mz - 1;
      double *ysc_d = nullptr, *yface_d = nullptr;
      bool okd = cudaMalloc(&d.rng, ns * sizeof(curandState)) == cudaSuccess &&
                 cudaMalloc(&d.r, ns * sizeof(double)) == cudaSuccess &&
                 cudaMalloc(&d.fy, nf * sizeof(double)) == cudaSuccess &&
                 cudaMalloc(&d.vnew, 3 * np * sizeof(double)) == cudaSuccess &&
                 cudaMalloc(&d.vold, 3 * np * sizeof(double)) == cudaSuccess &&
                 cudaMalloc(&d.fluc, 3 * np * sizeof(double)) == cudaSuccess &&
                 cudaMalloc(&d.lund, 6 * (size_t)d.py * sizeof(double)) == cudaSuccess &&
                 cudaMalloc(&d.by, (2 * kDfN + 1) * (size_t)d.py * sizeof(double)) == cudaSuccess &&
                 cudaMalloc(&d.bz, (2 * kDfN + 1) * (size_t)d.py * sizeof(double)) == cudaSuccess &&
                 cudaMalloc(&yface_d, np * sizeof(double)) == cudaSuccess &&
                 cudaMalloc(&ysc_d, d.py * sizeof(double)) == cudaSuccess &&
                 cudaMalloc(&ctx->d_zero, sizeof(double)) == cudaSuccess;
      d.yface = yface_d;
      if (!okd) {
        cudaFree(ysc_d);
        g_create_error = "device allocation for the digital filter failed";
        ostc_destroy(ctx.release());
        return OSTC_ENOMEM;
      }
      cudaMemset(d.r, 0, ns * sizeof(double));
      cudaMemset(d.fy, 0, nf * sizeof(double));
      cudaMemset(ctx->d_zero, 0, sizeof(double));
      cudaMemcpy(ysc_d, ysc.data(), ysc.size() * sizeof(double), cudaMemcpyHostToDevice);
      cudaMemcpy(yface_d, yface.data(), yface.size() * sizeof(double), cudaMemcpyHostToDevice);
      const auto &R = hf.df_rij;
      k_df_lund<<<(d.py + 127) / 128, 128, 0, ctx->stream>>>(d, ysc_d, R[0], R[1], R[2], R[3], R[4], R[5]);
      k_df_coeffs<<<(d.py + 127) / 128, 128, 0, ctx->stream>>>(d, ysc_d, dz / yref);
      df_start(ctx.get(), (unsigned long long)std::time(nullptr));
      cudaStreamSynchronize(ctx->stream);
      cudaFree(ysc_d);
      if (cudaGetLastError() != cudaSuccess) {
        g_create_error = "digital filter set-up failed on the device";
        ostc_destroy(ctx.release());
        return OSTC_ECUDA;
      }
    }
    if (size > 0) {
      if (cudaMalloc(&ctx->rng, size * sizeof(curandState)) != cudaSuccess) {
        g_create_error = "device allocation for the inflow random-number states failed";
        ostc_destroy(ctx.release());
        return OSTC_ENOMEM;
      }
      ctx->rng_size = size;
      for (auto &R : ctx->blk)
        for (auto &f : R.faces)
          if (f.type == kInflow && f.fluct == 1) f.rng = ctx->rng;
      k_rng_init<<<grid_for(ctx.get(), size, 128), 128, 0, ctx->stream>>>(ctx->rng, size,
                                                                     (unsigned long long)std::time(nullptr));
    }
  }
  const double dt0 = ctx->der.fixed_time_step ? ctx->der.dt : 1e6;
  cudaMemcpy(ctx->d_dt, &dt0, sizeof(double), cudaMemcpyHostToDevice);
  cudaMemset(ctx->d_time, 0, sizeof(double));
  cudaMemset(ctx->d_step, 0, sizeof(long long));
  cudaMemset(ctx->d_flags, 0, sizeof(unsigned));
  if (cudaDeviceSynchronize() != cudaSuccess) {
    g_create_error = "device set-up failed";
    ostc_destroy(ctx.release());
    return OSTC_ECUDA;
  }
  // statistics requested by the setup (Driver.cu:104: unsteady runs only; init_stat_name,
  // SinglePointStat.cu:115-146, skips unknown stat_rey_1st entries with a message)
  if (ctx->setup.get_bool("if_collect_statistics") && !ctx->der.steady) {
    std::vector<int> idx;
    auto it = ctx->setup.string_arrays.find("stat_rey_1st");
    if (it != ctx->setup.string_arrays.end())
      for (std::string v : it->second) {
        for (auto &c : v) c = (char)std::toupper((unsigned char)c);
        const int q = v == "U" ? 1 : v == "V" ? 2 : v == "W" ? 3 : v == "T" ? 5 : -1;
        if (q < 0 || idx.size() >= 4)
          std::fprintf(stderr, "ostc: variable %s for Reynolds average is not supported\n", v.c_str());
        else
          idx.push_back(q);
      }
    // the additional collectors (SinglePointStat.cu:27-96): stat_tke_budget, and for the species of
    // stat_species ("all", or names; unknown names skipped with a message) their velocity correlation
    // and dissipation rate
    StatExtras ex;
    ex.tke = ctx->setup.get_bool("stat_tke_budget");
    ex.svc = ctx->setup.get_bool("stat_species_velocity_correlation");
    ex.sdr = ctx->setup.get_bool("stat_species_dissipation_rate");
    auto ss = ctx->setup.string_arrays.find("stat_species");
    if (ctx->mixture && ss != ctx->setup.string_arrays.end()) {
      if (std::find(ss->second.begin(), ss->second.end(), "all") != ss->second.end()) {
        for (int l = 0; l < ctx->der.n_spec; ++l) ex.ss_idx.push_back(l);
      } else {
        for (const auto &name : ss->second) {
          auto f = std::find(ctx->chem.names.begin(), ctx->chem.names.end(), name);
          if (f == ctx->chem.names.end())
            std::fprintf(stderr, "ostc: species %s is not in the mechanism; its statistics are not collected\n",
                         name.c_str());
          else
            ex.ss_idx.push_back((int)(f - ctx->chem.names.begin()));
        }
      }
    }
    if (int r = stat_setup(ctx.get(), ctx->setup.get_int("start_collect_statistics_iter"), idx,
                           ctx->setup.get_bool("rho_p_correlation"), ex)) {
      g_create_error = ctx->err;
      ostc_destroy(ctx.release());
      return r;
    }
  }
  *out = ctx.release();
  return OSTC_OK;
}

void ostc_destroy(ostc_ctx *ctx) {
  if (!ctx) return;
  if (g_mix_owner == ctx) g_mix_owner = nullptr;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->graph) cudaGraphExecDestroy(ctx->graph);
  if (ctx->steady_graph) cudaGraphExecDestroy(ctx->steady_graph);
  for (auto &B : ctx->blk) {
    cudaFree(B.met);
    cudaFree(B.jac);
    cudaFree(B.met32);
    cudaFree(B.dq);
    cudaFree(B.last);
    cudaFree(B.adj);
    cudaFree(B.dqb);
    cudaFree(B.adj_work);
    cudaFree(B.stat);
    cudaFree(B.dtl);
    cudaFree(B.srad);
    cudaFree(B.cj);
    cudaFree(B.dq0);
    cudaFree(B.dqk);
    cudaFree(B.qn1);
    cudaFree(B.qstar);
    cudaFree(B.fcb);
    cudaFree(B.efd);
    cudaFree(B.ycoord);
    cudaFree(B.plt_xyz);
    for (double *p : B.face_y) cudaFree(p);
    for (int s = 0; s < 4; ++s) {
      cudaFree(B.cv[s]);
      cudaFree(B.bv[s]);
      cudaFree(B.mul[s]);
      cudaFree(B.sv[s]);
      cudaFree(B.cond[s]);
      cudaFree(B.rhod[s]);
      cudaFree(B.gam[s]);
      cudaFree(B.acs[s]);
    }
  }
  cudaFree(ctx->rng);
  for (void *p : {(void *)ctx->df.rng, (void *)ctx->df.r, (void *)ctx->df.fy, (void *)ctx->df.vnew,
                  (void *)ctx->df.vold, (void *)ctx->df.fluc, (void *)ctx->df.lund, (void *)ctx->df.by,
                  (void *)ctx->df.bz, (void *)ctx->df.yface, (void *)ctx->d_zero})
    cudaFree(p);
  cudaFree(ctx->d_dtbits);
  cudaFree(ctx->d_dt);
  cudaFree(ctx->d_time);
  cudaFree(ctx->d_sums);
  cudaFree(ctx->d_step);
  cudaFree(ctx->d_flags);
  cudaFree(ctx->d_staging);
  for (auto &e : ctx->ev_pool) {
    cudaEventDestroy(e.first);
    cudaEventDestroy(e.second);
  }
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  for (auto st : ctx->side) cudaStreamDestroy(st);
  if (ctx->rs_h2d) cudaStreamDestroy(ctx->rs_h2d);
  if (ctx->rs_d2h) cudaStreamDestroy(ctx->rs_d2h);
  for (int b = 0; b < 2; ++b) {
    cudaFree(ctx->rs_in[b]);
    cudaFree(ctx->rs_out[b]);
    for (cudaEvent_t e : {ctx->rs_in_ready[b], ctx->rs_in_free[b], ctx->rs_out_ready[b], ctx->rs_out_free[b]})
      if (e) cudaEventDestroy(e);
  }
  for (auto ev : ctx->side_ev) cudaEventDestroy(ev);
  if (ctx->fork_ev) cudaEventDestroy(ctx->fork_ev);
  delete ctx;
}

const char *ostc_last_error(const ostc_ctx *ctx) { return ctx ? ctx->err.c_str() : g_create_error.c_str(); }

int ostc_n_blocks(const ostc_ctx *ctx, int *n) {
  if (!ctx || !n) return OSTC_EINVAL;
  *n = (int)ctx->blk.size();
  return OSTC_OK;
}

int ostc_block_dims(const ostc_ctx *ctx, int block, int dims[4]) {
  if (!ctx || !dims || block < 0 || block >= (int)ctx->blk.size()) return OSTC_EINVAL;
  const DevBlock &b = ctx->blk[block].db;
  dims[0] = b.mx;
  dims[1] = b.my;
  dims[2] = b.mz;
  dims[3] = b.g;
  return OSTC_OK;
}

int ostc_n_var(const ostc_ctx *ctx, int *n_var, int *n_scalar) {
  if (!ctx) return OSTC_EINVAL;
  if (n_var) *n_var = ctx->der.n_var;
  if (n_scalar) *n_scalar = ctx->der.n_scalar;
  return OSTC_OK;
}

int ostc_total_nodes(const ostc_ctx *ctx, long long *n) {
  if (!ctx || !n) return OSTC_EINVAL;
  long long t = 0;
  for (auto &B : ctx->blk) t += B.db.n;
  *n = t;
  return OSTC_OK;
}

int ostc_set_precision(ostc_ctx *ctx, int mode) {
  if (!ctx) return OSTC_EINVAL;
  if (mode != OSTC_PREC_FP64 && mode != OSTC_PREC_MIXED) {
    ctx->err = "unknown precision mode";
    return OSTC_EINVAL;
  }
  ctx->precision = mode;
  return OSTC_OK;
}

int ostc_set_chem_mode(ostc_ctx *ctx, int mode) {
  if (!ctx) return OSTC_EINVAL;
  if (mode != OSTC_CHEM_EXPLICIT && mode != OSTC_CHEM_POINT_IMPLICIT) {
    ctx->err = "unknown chemistry mode";
    return OSTC_EINVAL;
  }
  if (mode == OSTC_CHEM_POINT_IMPLICIT && !(ctx->mixture && ctx->der.reaction == 1)) {
    ctx->err = "point-implicit chemistry needs a finite-rate mixture (species = 1, reaction = 1)";
    return OSTC_EINVAL;
  }
  if (ctx->graph && ctx->chem_mode != mode) {
    cudaGraphExecDestroy(ctx->graph);
    ctx->graph = nullptr;
  }
  ctx->chem_mode = mode;
  return OSTC_OK;
}

int ostc_set_state(ostc_ctx *ctx, int block, const double *bv, const double *sv, int ptr_kind) {
  if (!ctx || !bv || block < 0 || block >= (int)ctx->blk.size()) return OSTC_EINVAL;
  if (ctx->mixture && !sv) {
    ctx->err = "ostc_set_state: a mixture case needs the mass fractions sv[n_spec][N]";
    return OSTC_EINVAL;
  }
  cudaSetDevice(ctx->device);
  BlockRes &B = ctx->blk[block];
  const auto kind = ptr_kind == OSTC_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  const size_t bytes = 6 * (size_t)B.db.n * sizeof(double);
  CK(cudaMemcpyAsync(ctx->d_staging, bv, bytes, kind, ctx->stream));
  if (ctx->mixture) {
    CK(cudaMemcpyAsync(ctx->d_staging + 6 * B.db.n, sv, (size_t)ctx->der.n_spec * B.db.n * sizeof(double), kind,
                       ctx->stream));
  }
  enqueue_set_state(ctx, B, ctx->d_staging, ctx->d_staging + 6 * B.db.n);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->block_set[block] = 1;
  ctx->state_set = true;
  ctx->initialised = false;
  CK(cudaMemsetAsync(ctx->d_time, 0, sizeof(double), ctx->stream));
  return OSTC_OK;
}

int ostc_get_state(ostc_ctx *ctx, int block, double *cv, double *bv, double *sv, int ptr_kind) {
  if (!ctx || block < 0 || block >= (int)ctx->blk.size()) return OSTC_EINVAL;
  cudaSetDevice(ctx->device);
  if (int r = check_ready(ctx)) return r;
  BlockRes &B = ctx->blk[block];
  const auto kind = ptr_kind == OSTC_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  const int nv = ctx->nv;
  if (cv) {
    k_gather<<<grid_for(ctx, nv * B.db.n, 256), 256, 0, ctx->stream>>>(B.db, B.cv[0], ctx->d_staging, nv);
    CK(cudaMemcpyAsync(cv, ctx->d_staging, (size_t)nv * B.db.n * sizeof(double), kind, ctx->stream));
  }
  if (sv && ctx->mixture) {
    const int ns = ctx->der.n_spec;
    CK(cudaStreamSynchronize(ctx->stream));
    k_gather<<<grid_for(ctx, ns * B.db.n, 256), 256, 0, ctx->stream>>>(B.db, B.sv[0], ctx->d_staging, ns);
    CK(cudaMemcpyAsync(sv, ctx->d_staging, (size_t)ns * B.db.n * sizeof(double), kind, ctx->stream));
  }
  if (bv) {
    k_gather<<<grid_for(ctx, 6 * B.db.n, 256), 256, 0, ctx->stream>>>(B.db, B.bv[0], ctx->d_staging, 6);
    CK(cudaMemcpyAsync(bv, ctx->d_staging, 6 * B.db.n * sizeof(double), kind, ctx->stream));
  }
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->stream));
  return OSTC_OK;
}

int ostc_rhs(ostc_ctx *ctx, int block, unsigned mask, double *dq, int ptr_kind) {
  if (!ctx || !dq || block < 0 || block >= (int)ctx->blk.size()) return OSTC_EINVAL;
  cudaSetDevice(ctx->device);
  if (int r = check_ready(ctx)) return r;
  BlockRes &B = ctx->blk[block];
  const int nv = ctx->nv;
  CK(cudaMemsetAsync(B.dq, 0, (size_t)nv * B.db.n * sizeof(double), ctx->stream));
  if (ctx->mixture) {
    // source (dq initialised by it, RK.cuh:116), flux-split WENO7, viscous
    const DevState in = state_of(B, 0);
    const bool chem = (mask & OSTC_TERM_SOURCE) && ctx->der.reaction == 1;
    const bool implicit = chem && ctx->chem_mode == OSTC_CHEM_POINT_IMPLICIT;
    launch_mix_source(ctx, B, in, chem && !implicit);
    if (mask & OSTC_TERM_INVISCID) launch_mix_inviscid(ctx, B, in);
    if ((mask & OSTC_TERM_VISCOUS) && ctx->der.viscous_order != 0) launch_mix_visc(ctx, B, in);
    if (implicit) launch_chem_epi(ctx, B, in);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(dq, B.dq, (size_t)nv * B.db.n * sizeof(double),
                       ptr_kind == OSTC_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return OSTC_OK;
  }
  const bool mixed = ctx->precision == OSTC_PREC_MIXED;
  if (mask & OSTC_TERM_INVISCID) {
    if (mixed) launch_flux<float>(ctx, B, state_of(B, 0));
    else launch_flux<double>(ctx, B, state_of(B, 0));
  }
  if ((mask & OSTC_TERM_VISCOUS) && ctx->der.viscous_order != 0) {
    StageArgs a{};
    a.in = state_of(B, 0);
    a.qn = a.in;
    a.out = a.in;
    a.prandtl = ctx->der.prandtl;
    a.viscous = 1;
    a.update = 0;
    a.flags = ctx->d_flags;
    a.dt = ctx->d_dt;
    if (mixed) launch_visc<float>(ctx, B, a);
    else launch_visc<double>(ctx, B, a);
  }
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(dq, B.dq, 5 * B.db.n * sizeof(double),
                     ptr_kind == OSTC_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return OSTC_OK;
}

int ostc_set_conservative(ostc_ctx *ctx, int block, const double *cv, int ptr_kind) {
  if (!ctx || !cv || block < 0 || block >= (int)ctx->blk.size()) return OSTC_EINVAL;
  cudaSetDevice(ctx->device);
  if (int r = check_ready(ctx)) return r;
  BlockRes &B = ctx->blk[block];
  const int nv = ctx->nv;
  const auto kind = ptr_kind == OSTC_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  CK(cudaMemcpyAsync(ctx->d_staging, cv, (size_t)nv * B.db.n * sizeof(double), kind, ctx->stream));
  DevState st = state_of(B, 0);
  k_scatter<<<grid_for(ctx, nv * B.db.n, 256), 256, 0, ctx->stream>>>(B.db, ctx->d_staging, st.cv, nv);
  const int g = grid_for(ctx, B.db.n, 128);
  if (ctx->mixture && ctx->der.n_spec == kFixedNS)
    k_state_from_cv<kFixedNS><<<g, 128, 0, ctx->stream>>>(B.db, st, 1, ctx->d_flags);
  else
    k_state_from_cv<0><<<g, 128, 0, ctx->stream>>>(B.db, st, ctx->mixture ? 1 : 0, ctx->d_flags);
  launch_bcs(ctx, block, st);
  launch_interfaces(ctx, 0);
  if (ctx->mixture)
    for (auto &Bk : ctx->blk) launch_mix_props(ctx, Bk, state_of(Bk, 0));
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->stream));
  return OSTC_OK;
}

int ostc_rhs_vjp(ostc_ctx *ctx, int block, unsigned mask, const double *dq_bar, double *cv_bar, int ptr_kind) {
  if (!ctx || !dq_bar || !cv_bar || block < 0 || block >= (int)ctx->blk.size()) return OSTC_EINVAL;
  if (int r = adjoint_check(ctx, mask)) return r;
  cudaSetDevice(ctx->device);
  if (int r = check_ready(ctx)) return r;
  BlockRes &B = ctx->blk[block];
  if (int r = adjoint_alloc(ctx, B)) return r;
  const size_t bytes = (size_t)ctx->nv * B.db.n * sizeof(double);
  CK(cudaMemcpyAsync(B.dqb, dq_bar, bytes, ptr_kind == OSTC_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                     ctx->stream));
  if (int r = vjp_core(ctx, block, 0, mask, B.dq)) return r;
  CK(cudaMemcpyAsync(cv_bar, B.dq, bytes, ptr_kind == OSTC_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                     ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return OSTC_OK;
}

int ostc_rk3_step_vjp(ostc_ctx *ctx, const double *lam_out, double *lam_in, int ptr_kind) {
  if (!ctx || !lam_out || !lam_in) return OSTC_EINVAL;
  if (int r = adjoint_check(ctx, OSTC_TERM_ALL, true)) return r;
  if (ctx->precision != OSTC_PREC_FP64) {
    ctx->err = "the step adjoint is that of the FP64 step: set OSTC_PREC_FP64";
    return OSTC_EINVAL;
  }
  cudaSetDevice(ctx->device);
  if (int r = check_ready(ctx)) return r;
  BlockRes &B = ctx->blk[0];
  if (int r = adjoint_alloc(ctx, B)) return r;
  const size_t bytes = (size_t)ctx->nv * B.db.n * sizeof(double);
  CK(cudaMemcpyAsync(B.adj_work, lam_out, bytes,
                     ptr_kind == OSTC_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemsetAsync(B.adj_work + 4 * (size_t)ctx->nv * B.db.n, 0, B.db.n * sizeof(double), ctx->stream));
  if (!ctx->der.fixed_time_step) enqueue_cfl_dt(ctx);
  if (int r = step_vjp(ctx)) return r;
  if (ctx->mixture)
    if (int r = adjoint_t_to_cv(ctx)) return r;
  CK(cudaMemcpyAsync(lam_in, B.adj_work, bytes,
                     ptr_kind == OSTC_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return OSTC_OK;
}

int ostc_adjoint_steps(ostc_ctx *ctx, int n_steps, int every, const double *lam_final, double *lam_initial,
                       int ptr_kind) {
  if (!ctx || !lam_final || !lam_initial || n_steps < 1 || every < 1) return OSTC_EINVAL;
  if (int r = adjoint_check(ctx, OSTC_TERM_ALL, true)) return r;
  if (ctx->precision != OSTC_PREC_FP64) {
    ctx->err = "the step adjoint is that of the FP64 step: set OSTC_PREC_FP64";
    return OSTC_EINVAL;
  }
  cudaSetDevice(ctx->device);
  if (int r = check_ready(ctx)) return r;
  BlockRes &B = ctx->blk[0];
  if (int r = adjoint_alloc(ctx, B)) return r;
  const int nv = ctx->nv, ns = ctx->der.n_spec;
  const long long P = B.db.plane;
  // a saved state: cv, bv and (mixtures) the mass fractions or (air) the viscosity
  const int nx = ctx->mixture ? ns : 1;
  double *const xs = ctx->mixture ? B.sv[0] : B.mul[0];
  const size_t state_doubles = (size_t)(nv + 6 + nx) * P;
  const int ncp = (n_steps + every - 1) / every;
  // device checkpoints (every `every` steps), one segment of step-start states, the final state
  double *cps = nullptr, *seg = nullptr, *fin = nullptr;
  auto release = [&]() {
    cudaFree(cps);
    cudaFree(seg);
    cudaFree(fin);
  };
  if (cudaMalloc(&cps, (size_t)ncp * state_doubles * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&seg, (size_t)every * state_doubles * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&fin, state_doubles * sizeof(double)) != cudaSuccess) {
    release();
    ctx->err = "ostc_adjoint_steps: device memory for the checkpoints";
    return OSTC_ECUDA;
  }
  auto save = [&](double *dst) {
    cudaMemcpyAsync(dst, B.cv[0], (size_t)nv * P * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream);
    cudaMemcpyAsync(dst + (size_t)nv * P, B.bv[0], 6 * P * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream);
    cudaMemcpyAsync(dst + (size_t)(nv + 6) * P, xs, (size_t)nx * P * sizeof(double), cudaMemcpyDeviceToDevice,
                    ctx->stream);
  };
  auto restore = [&](const double *src) {
    cudaMemcpyAsync(B.cv[0], src, (size_t)nv * P * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream);
    cudaMemcpyAsync(B.bv[0], src + (size_t)nv * P, 6 * P * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream);
    cudaMemcpyAsync(xs, src + (size_t)(nv + 6) * P, (size_t)nx * P * sizeof(double), cudaMemcpyDeviceToDevice,
                    ctx->stream);
    if (ctx->mixture) launch_mix_props(ctx, B, state_of(B, 0));
  };
  auto stages = [&]() {
    for (int rk = 0; rk < 3; ++rk) {
      if (ctx->mixture) enqueue_mix_stage(ctx, rk);
      else enqueue_air_stage<double>(ctx, rk);
    }
  };
  // forward sweep: checkpoints and the dt of every step
  std::vector<double> dts(n_steps);
  for (int n = 0; n < n_steps; ++n) {
    if (n % every == 0) save(cps + (size_t)(n / every) * state_doubles);
    if (!ctx->der.fixed_time_step) enqueue_cfl_dt(ctx);
    stages();
    k_step_end<<<1, 1, 0, ctx->stream>>>(ctx->d_time, ctx->d_dt, ctx->d_step);
    if (cudaMemcpyAsync(&dts[n], ctx->d_dt, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess ||
        cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
      release();
      ctx->err = "ostc_adjoint_steps: forward sweep failed";
      return OSTC_ECUDA;
    }
  }
  save(fin);
  // reverse sweep, one segment at a time: recompute the segment's step-start states from its
  // checkpoint, then run the step adjoints backwards through them
  const size_t bytes = (size_t)nv * B.db.n * sizeof(double);
  cudaMemcpyAsync(B.adj_work, lam_final, bytes, ptr_kind == OSTC_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                  ctx->stream);
  cudaMemsetAsync(B.adj_work + 4 * (size_t)nv * B.db.n, 0, B.db.n * sizeof(double), ctx->stream);
  int rc = OSTC_OK;
  for (int sgi = ncp - 1; sgi >= 0 && rc == OSTC_OK; --sgi) {
    const int a = sgi * every, b = std::min(a + every, n_steps);
    restore(cps + (size_t)sgi * state_doubles);
    for (int n = a; n < b; ++n) {
      save(seg + (size_t)(n - a) * state_doubles);
      if (n + 1 < b) {
        cudaMemcpyAsync(ctx->d_dt, &dts[n], sizeof(double), cudaMemcpyHostToDevice, ctx->stream);
        stages();
      }
    }
    for (int n = b - 1; n >= a && rc == OSTC_OK; --n) {
      restore(seg + (size_t)(n - a) * state_doubles);
      cudaMemcpyAsync(ctx->d_dt, &dts[n], sizeof(double), cudaMemcpyHostToDevice, ctx->stream);
      rc = step_vjp(ctx);
    }
  }
  // the first checkpoint is the caller's state, whose T is the equation-of-state root of its cv
  if (rc == OSTC_OK && ctx->mixture) {
    restore(cps);
    rc = adjoint_t_to_cv(ctx);
  }
  restore(fin);
  cudaMemcpyAsync(ctx->d_dt, &dts[n_steps - 1], sizeof(double), cudaMemcpyHostToDevice, ctx->stream);
  if (rc == OSTC_OK)
    cudaMemcpyAsync(lam_initial, B.adj_work, bytes,
                    ptr_kind == OSTC_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, ctx->stream);
  const bool ok = cudaGetLastError() == cudaSuccess && cudaStreamSynchronize(ctx->stream) == cudaSuccess;
  release();
  if (rc != OSTC_OK) return rc;
  if (!ok) {
    ctx->err = "ostc_adjoint_steps: CUDA error";
    return OSTC_ECUDA;
  }
  return OSTC_OK;
}

static int ensure_graph(ostc_ctx *ctx);

int ostc_run_states(ostc_ctx *ctx, int n, const double *const *bv_in, const double *const *sv_in,
                    double *const *bv_out, double *const *sv_out, int n_steps) {
  if (!ctx || n < 0 || n_steps < 0 || (n > 0 && (!bv_in || !bv_out))) return OSTC_EINVAL;
  if (ctx->blk.size() != 1) {
    ctx->err = "ostc_run_states: single-block cases";
    return OSTC_EINVAL;
  }
  if (ctx->mixture && n > 0 && (!sv_in || !sv_out)) {
    ctx->err = "ostc_run_states: a mixture case needs sv_in and sv_out";
    return OSTC_EINVAL;
  }
  cudaSetDevice(ctx->device);
  BlockRes &B = ctx->blk[0];
  const long long N = B.db.n;
  const int ns = ctx->mixture ? ctx->der.n_spec : 0;
  const size_t vals = (size_t)(6 + ns) * N;
  if (!ctx->rs_h2d) {
    CK(cudaStreamCreateWithFlags(&ctx->rs_h2d, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&ctx->rs_d2h, cudaStreamNonBlocking));
    for (int b = 0; b < 2; ++b) {
      CK(cudaMalloc(&ctx->rs_in[b], vals * sizeof(double)));
      CK(cudaMalloc(&ctx->rs_out[b], vals * sizeof(double)));
      for (cudaEvent_t *e : {&ctx->rs_in_ready[b], &ctx->rs_in_free[b], &ctx->rs_out_ready[b], &ctx->rs_out_free[b]})
        CK(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    }
  }
  // the step graph is captured once, from the first state
  for (int i = 0; i < n; ++i) {
    const int b = i & 1;
    // host -> device of state i (overlaps the computation of state i - 1)
    CK(cudaStreamWaitEvent(ctx->rs_h2d, ctx->rs_in_free[b], 0));
    CK(cudaMemcpyAsync(ctx->rs_in[b], bv_in[i], 6 * N * sizeof(double), cudaMemcpyHostToDevice, ctx->rs_h2d));
    if (ns)
      CK(cudaMemcpyAsync(ctx->rs_in[b] + 6 * N, sv_in[i], (size_t)ns * N * sizeof(double), cudaMemcpyHostToDevice,
                         ctx->rs_h2d));
    CK(cudaEventRecord(ctx->rs_in_ready[b], ctx->rs_h2d));
    // compute state i: set, initialise, n_steps steps
    CK(cudaStreamWaitEvent(ctx->stream, ctx->rs_in_ready[b], 0));
    enqueue_set_state(ctx, B, ctx->rs_in[b], ctx->rs_in[b] + 6 * N);
    CK(cudaEventRecord(ctx->rs_in_free[b], ctx->stream));
    CK(cudaMemsetAsync(ctx->d_time, 0, sizeof(double), ctx->stream));
    ctx->block_set[0] = 1;
    ctx->state_set = true;
    ctx->initialised = false;
    if (int r = check_ready(ctx)) return r;
    if (n_steps > 0) {
      if (int r = ensure_graph(ctx)) return r;
      for (int st = 0; st < n_steps; ++st) CK(cudaGraphLaunch(ctx->graph, ctx->stream));
    }
    CK(cudaStreamWaitEvent(ctx->stream, ctx->rs_out_free[b], 0));
    k_gather<<<grid_for(ctx, 6 * N, 256), 256, 0, ctx->stream>>>(B.db, B.bv[0], ctx->rs_out[b], 6);
    if (ns)
      k_gather<<<grid_for(ctx, ns * N, 256), 256, 0, ctx->stream>>>(B.db, B.sv[0], ctx->rs_out[b] + 6 * N, ns);
    CK(cudaGetLastError());
    CK(cudaEventRecord(ctx->rs_out_ready[b], ctx->stream));
    // device -> host of state i (overlaps the computation of state i + 1)
    CK(cudaStreamWaitEvent(ctx->rs_d2h, ctx->rs_out_ready[b], 0));
    CK(cudaMemcpyAsync(bv_out[i], ctx->rs_out[b], 6 * N * sizeof(double), cudaMemcpyDeviceToHost, ctx->rs_d2h));
    if (ns)
      CK(cudaMemcpyAsync(sv_out[i], ctx->rs_out[b] + 6 * N, (size_t)ns * N * sizeof(double), cudaMemcpyDeviceToHost,
                         ctx->rs_d2h));
    CK(cudaEventRecord(ctx->rs_out_free[b], ctx->rs_d2h));
  }
  CK(cudaStreamSynchronize(ctx->rs_d2h));
  CK(cudaStreamSynchronize(ctx->stream));
  return OSTC_OK;
}

}  // extern "C"
