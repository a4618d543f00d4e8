// enqueue.cuh -- host-side launch machinery: per-kernel launch helpers, the stage / step / steady /
// dual-time / adjoint enqueue functions, the y/z sweep autotuner and the context initialisation.
// Part of the ostc_b200.cu translation unit (included in order; not a standalone header).
#pragma once

namespace {

int fam_index(ostc_ctx *ctx, const char *name) {
  for (size_t i = 0; i < ctx->fams.size(); ++i)
    if (std::strcmp(ctx->fams[i].name, name) == 0) return (int)i;
  ctx->fams.push_back({name, 0, 0.0});
  return (int)ctx->fams.size() - 1;
}

// Records a begin event for a kernel family when timing is on; returns a token for end_t.
// Per-kernel-family timing of ostc_profile_steps: CUDA events on the context stream around each
// launch group, and an NVTX range of the same name (visible to nsys / ncu range filters).
long begin_t(ostc_ctx *ctx, const char *name) {
  if (!ctx->timing) return -1;
  nvtxRangePushA(name);
  const size_t slot = ctx->ev_used.size();
  if (slot >= ctx->ev_pool.size()) {
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    ctx->ev_pool.emplace_back(a, b);
  }
  ctx->ev_used.emplace_back(fam_index(ctx, name), slot);
  cudaEventRecord(ctx->ev_pool[slot].first, ctx->stream);
  return (long)slot;
}
void end_t(ostc_ctx *ctx, long tok) {
  if (tok < 0) return;
  nvtxRangePop();
  cudaEventRecord(ctx->ev_pool[tok].second, ctx->stream);
}

int grid_for(ostc_ctx *ctx, long long n, int tpb) {
  long long g = (n + tpb - 1) / tpb;
  const long long cap = (long long)ctx->sm_count * 16;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}

// inviscid sweeps of one block with a primitive reconstruction (inviscid_type 0: MUSCL/NND/1st order
// + LF/AUSM+/HLLC, InviscidScheme.cu:12-50; inviscid_type 2: Roe, :369-415)
template <int RS, typename T>
void launch_flux_pv_rs(ostc_ctx *ctx, BlockRes &B, DevState in) {
  const DevBlock &b = B.db;
  const bool is3d = b.mz > 1;
  const PvArgs a{ctx->der.reconstruction, ctx->der.entropy_fix_factor, is3d ? 1 : 0};
  {
    dim3 grid((b.mx + 123) / 124, b.my, b.mz);
    long tok = begin_t(ctx, "flux_x");
    k_flux_pv_x<RS, T><<<grid, 128, 0, ctx->stream>>>(b, in, a, B.dq);
    end_t(ctx, tok);
  }
  for (int dir = 1; dir <= (is3d ? 2 : 1); ++dir) {
    const int n_dir = dir == 1 ? b.my : b.mz, n_o = dir == 1 ? b.mz : b.my;
    const long long cols = (long long)((b.mx + 127) / 128) * n_o;
    int nseg = (int)std::max<long long>(1, (ctx->sm_count * 16 + cols - 1) / cols);
    int seg = std::max(8, (n_dir + nseg - 1) / nseg);
    nseg = (n_dir + seg - 1) / seg;
    dim3 grid((b.mx + 127) / 128, n_o, nseg);
    long tok = begin_t(ctx, dir == 1 ? "flux_y" : "flux_z");
    if (dir == 1) k_flux_pv_march<1, RS, T><<<grid, 128, 0, ctx->stream>>>(b, in, a, B.dq, seg);
    else k_flux_pv_march<2, RS, T><<<grid, 128, 0, ctx->stream>>>(b, in, a, B.dq, seg);
    end_t(ctx, tok);
  }
}

template <typename T>
void launch_flux_pv(ostc_ctx *ctx, BlockRes &B, DevState in) {
  switch (ctx->der.riemann) {
    case 1: launch_flux_pv_rs<1, T>(ctx, B, in); break;
    case 2: launch_flux_pv_rs<2, T>(ctx, B, in); break;
    case 4: launch_flux_pv_rs<4, T>(ctx, B, in); break;
    default: launch_flux_pv_rs<3, T>(ctx, B, in); break;
  }
}

// flux-split WENO7 sweeps (inviscid_type 3, schemes 71 / 72), accumulating into dq
template <int NS, typename T>
void launch_fvs_t(ostc_ctx *ctx, BlockRes &B, DevState in) {
  const DevBlock &b = B.db;
  const int nv = ctx->nv, sch = ctx->der.inviscid_scheme;
  {
    long tok = begin_t(ctx, "flux_x");
    dim3 grid((b.mx + FvsTile<0>::TD - 2) / (FvsTile<0>::TD - 1), b.my, b.mz);
    k_fvs<0, NS, T><<<grid, FvsTile<0>::TD, fvs_smem_bytes<0, T>(nv), ctx->stream>>>(b, in, B.dq, nv, sch);
    end_t(ctx, tok);
  }
  {
    long tok = begin_t(ctx, "flux_y");
    dim3 grid((b.mx + FvsTile<1>::TXL - 1) / FvsTile<1>::TXL, (b.my + FvsTile<1>::TD - 2) / (FvsTile<1>::TD - 1), b.mz);
    k_fvs<1, NS, T><<<grid, dim3(FvsTile<1>::TXL, FvsTile<1>::TD), fvs_smem_bytes<1, T>(nv), ctx->stream>>>(b, in, B.dq, nv, sch);
    end_t(ctx, tok);
  }
  if (b.mz > 1) {
    long tok = begin_t(ctx, "flux_z");
    dim3 grid((b.mx + FvsTile<2>::TXL - 1) / FvsTile<2>::TXL, (b.mz + FvsTile<2>::TD - 2) / (FvsTile<2>::TD - 1), b.my);
    k_fvs<2, NS, T><<<grid, dim3(FvsTile<2>::TXL, FvsTile<2>::TD), fvs_smem_bytes<2, T>(nv), ctx->stream>>>(b, in, B.dq, nv, sch);
    end_t(ctx, tok);
  }
}

// mixture viscous sweeps, accumulating into dq
template <int NS, typename T>
void launch_mix_visc_t(ostc_ctx *ctx, BlockRes &B, DevState in) {
  const DevBlock &b = B.db;
  const int nv = ctx->nv;
  const bool is3d = b.mz > 1;
  long tok = begin_t(ctx, "visc");
  {
    dim3 grid((b.mx + FvsTile<0>::TD - 2) / (FvsTile<0>::TD - 1), b.my, b.mz);
    const size_t sm = (size_t)FvsTile<0>::TD * nv * sizeof(T);
    if (is3d) k_mix_visc<0, true, NS, T><<<grid, FvsTile<0>::TD, sm, ctx->stream>>>(b, in, B.dq, nv);
    else k_mix_visc<0, false, NS, T><<<grid, FvsTile<0>::TD, sm, ctx->stream>>>(b, in, B.dq, nv);
  }
  {
    dim3 grid((b.mx + FvsTile<1>::TXL - 1) / FvsTile<1>::TXL, (b.my + FvsTile<1>::TD - 2) / (FvsTile<1>::TD - 1), b.mz);
    const size_t sm = (size_t)FvsTile<1>::TD * FvsTile<1>::TXL * nv * sizeof(T);
    dim3 blk(FvsTile<1>::TXL, FvsTile<1>::TD);
    if (is3d) k_mix_visc<1, true, NS, T><<<grid, blk, sm, ctx->stream>>>(b, in, B.dq, nv);
    else k_mix_visc<1, false, NS, T><<<grid, blk, sm, ctx->stream>>>(b, in, B.dq, nv);
  }
  if (is3d) {
    dim3 grid((b.mx + FvsTile<2>::TXL - 1) / FvsTile<2>::TXL, (b.mz + FvsTile<2>::TD - 2) / (FvsTile<2>::TD - 1), b.my);
    const size_t sm = (size_t)FvsTile<2>::TD * FvsTile<2>::TXL * nv * sizeof(T);
    k_mix_visc<2, true, NS, T><<<grid, dim3(FvsTile<2>::TXL, FvsTile<2>::TD), sm, ctx->stream>>>(b, in, B.dq, nv);
  }
  end_t(ctx, tok);
}

// The H2/air mechanism's 9 species get a dedicated instantiation; other counts the generic one.
// In the mixed precision mode the flux-split, viscous and property kernels run in FP32.
constexpr int kFixedNS = 9;
void launch_fvs(ostc_ctx *ctx, BlockRes &B, DevState in) {
  const bool f32 = ctx->precision == OSTC_PREC_MIXED;
  if (ctx->der.n_spec == kFixedNS) f32 ? launch_fvs_t<kFixedNS, float>(ctx, B, in) : launch_fvs_t<kFixedNS, double>(ctx, B, in);
  else f32 ? launch_fvs_t<0, float>(ctx, B, in) : launch_fvs_t<0, double>(ctx, B, in);
}
void launch_mix_visc(ostc_ctx *ctx, BlockRes &B, DevState in) {
  const bool f32 = ctx->precision == OSTC_PREC_MIXED;
  if (ctx->der.n_spec == kFixedNS)
    f32 ? launch_mix_visc_t<kFixedNS, float>(ctx, B, in) : launch_mix_visc_t<kFixedNS, double>(ctx, B, in);
  else f32 ? launch_mix_visc_t<0, float>(ctx, B, in) : launch_mix_visc_t<0, double>(ctx, B, in);
}

// Inviscid sweeps of a mixture: flux-split WENO (inviscid_scheme 71 / 72) or the primitive
// reconstruction with AUSM+ / HLLC / Roe (pv_mix.cuh), accumulated into dq.
template <int NS>
void launch_pv_mix_t(ostc_ctx *ctx, BlockRes &B, DevState in) {
  const DevBlock &b = B.db;
  const int nv = ctx->nv, recon = ctx->der.reconstruction, rs = ctx->der.riemann;
  if (rs == 2) {
    const long long pts = (long long)(b.mx + 2) * (b.my + 2) * (b.mz > 1 ? b.mz + 2 : 1);
    k_efix_mix<<<grid_for(ctx, pts, 128), 128, 0, ctx->stream>>>(b, in, ctx->der.entropy_fix_factor, B.efd);
  }
  const int gn = grid_for(ctx, b.n, 128);
#define OSTC_PVM(D)                                                                                                 \
  k_pv_mix_face<NS, D><<<grid_for(ctx, pv_face_count<D>(b), 128), 128, 0, ctx->stream>>>(b, in, nv, recon, rs, B.efd, \
                                                                                        B.fcb);                     \
  k_pv_mix_diff<D><<<gn, 128, 0, ctx->stream>>>(b, nv, B.fcb, B.dq);
  OSTC_PVM(0)
  OSTC_PVM(1)
  if (b.mz > 1) {
    OSTC_PVM(2)
  }
#undef OSTC_PVM
}

void launch_mix_inviscid(ostc_ctx *ctx, BlockRes &B, DevState in) {
  if (ctx->der.inviscid_type == 3) {
    launch_fvs(ctx, B, in);
    return;
  }
  long tok = begin_t(ctx, "pv_mix");
  if (ctx->der.n_spec == kFixedNS) launch_pv_mix_t<kFixedNS>(ctx, B, in);
  else launch_pv_mix_t<0>(ctx, B, in);
  end_t(ctx, tok);
}
template <int NS>
void launch_mix_source_t(ostc_ctx *ctx, BlockRes &B, DevState in, bool chem) {
  k_mix_source<NS><<<grid_for(ctx, B.db.n, 128), 128, 0, ctx->stream>>>(B.db, in, B.dq, ctx->nv, chem ? 1 : 0);
}
void launch_mix_source(ostc_ctx *ctx, BlockRes &B, DevState in, bool chem) {
  if (ctx->der.n_spec == kFixedNS) launch_mix_source_t<kFixedNS>(ctx, B, in, chem);
  else launch_mix_source_t<0>(ctx, B, in, chem);
}
void launch_chem_epi(ostc_ctx *ctx, BlockRes &B, DevState in) {
  long tok = begin_t(ctx, "chem_implicit");
  if (ctx->der.n_spec == kFixedNS)
    k_mix_chem_epi<kFixedNS><<<grid_for(ctx, B.db.n, 128), 128, 0, ctx->stream>>>(B.db, in, B.dq, ctx->d_dt);
  else
    k_mix_chem_epi<0><<<grid_for(ctx, B.db.n, 128), 128, 0, ctx->stream>>>(B.db, in, B.dq, ctx->d_dt);
  end_t(ctx, tok);
}

void launch_mix_props(ostc_ctx *ctx, BlockRes &B, DevState st) {
  const int g = grid_for(ctx, B.db.plane, 128);
  const bool f32 = ctx->precision == OSTC_PREC_MIXED;
  if (ctx->der.n_spec == kFixedNS) {
    if (f32) k_mix_props<kFixedNS, float><<<g, 128, 0, ctx->stream>>>(B.db, st);
    else k_mix_props<kFixedNS, double><<<g, 128, 0, ctx->stream>>>(B.db, st);
  } else {
    if (f32) k_mix_props<0, float><<<g, 128, 0, ctx->stream>>>(B.db, st);
    else k_mix_props<0, double><<<g, 128, 0, ctx->stream>>>(B.db, st);
  }
}

DevState state_of(BlockRes &B, int s);

// ---- adjoint of the multi-component right-hand side (ostc_rhs_vjp)
template <int NS>
void launch_adjoint_t(ostc_ctx *ctx, BlockRes &B, DevState in, unsigned mask, const DevAdj &A) {
  const DevBlock &b = B.db;
  const int nv = ctx->nv, sch = ctx->der.inviscid_scheme;
  const bool is3d = b.mz > 1;
  if (mask & OSTC_TERM_INVISCID) {
    dim3 g0((b.mx + FvsTile<0>::TD - 2) / (FvsTile<0>::TD - 1), b.my, b.mz);
    k_adj_fvs<0, NS><<<g0, FvsTile<0>::TD, adj_fvs_smem_bytes<0>(nv), ctx->stream>>>(b, in, B.dqb, nv, sch, A);
    dim3 g1((b.mx + FvsTile<1>::TXL - 1) / FvsTile<1>::TXL, (b.my + FvsTile<1>::TD - 2) / (FvsTile<1>::TD - 1), b.mz);
    k_adj_fvs<1, NS><<<g1, dim3(FvsTile<1>::TXL, FvsTile<1>::TD), adj_fvs_smem_bytes<1>(nv), ctx->stream>>>(
        b, in, B.dqb, nv, sch, A);
    if (is3d) {
      dim3 g2((b.mx + FvsTile<2>::TXL - 1) / FvsTile<2>::TXL, (b.mz + FvsTile<2>::TD - 2) / (FvsTile<2>::TD - 1), b.my);
      k_adj_fvs<2, NS><<<g2, dim3(FvsTile<2>::TXL, FvsTile<2>::TD), adj_fvs_smem_bytes<2>(nv), ctx->stream>>>(
          b, in, B.dqb, nv, sch, A);
    }
  }
  if ((mask & OSTC_TERM_VISCOUS) && ctx->der.viscous_order != 0) {
    dim3 g0((b.mx + FvsTile<0>::TD - 2) / (FvsTile<0>::TD - 1), b.my, b.mz);
    dim3 g1((b.mx + FvsTile<1>::TXL - 1) / FvsTile<1>::TXL, (b.my + FvsTile<1>::TD - 2) / (FvsTile<1>::TD - 1), b.mz);
    dim3 blk(FvsTile<1>::TXL, FvsTile<1>::TD);
    if (is3d) {
      k_adj_visc<0, true, NS><<<g0, FvsTile<0>::TD, 0, ctx->stream>>>(b, in, B.dqb, nv, A);
      k_adj_visc<1, true, NS><<<g1, blk, 0, ctx->stream>>>(b, in, B.dqb, nv, A);
      dim3 g2((b.mx + FvsTile<2>::TXL - 1) / FvsTile<2>::TXL, (b.mz + FvsTile<2>::TD - 2) / (FvsTile<2>::TD - 1), b.my);
      k_adj_visc<2, true, NS><<<g2, dim3(FvsTile<2>::TXL, FvsTile<2>::TD), 0, ctx->stream>>>(b, in, B.dqb, nv, A);
    } else {
      k_adj_visc<0, false, NS><<<g0, FvsTile<0>::TD, 0, ctx->stream>>>(b, in, B.dqb, nv, A);
      k_adj_visc<1, false, NS><<<g1, blk, 0, ctx->stream>>>(b, in, B.dqb, nv, A);
    }
  }
  if ((mask & OSTC_TERM_SOURCE) && ctx->der.reaction == 1)
    k_adj_source<NS><<<grid_for(ctx, b.n, 128), 128, 0, ctx->stream>>>(b, in, B.dqb, A);
  k_adj_props<NS><<<grid_for(ctx, b.plane, 128), 128, 0, ctx->stream>>>(b, in, A);
  k_adj_ghost_cv<NS><<<grid_for(ctx, b.plane, 128), 128, 0, ctx->stream>>>(b, in, A, nv);
}

// y / z sweep variants: 0 = column march, 1..3 = tiles of the shapes below (per precision: rows
// of 128 bytes, and a block small enough for the register budget of the FP64 face arithmetic).
template <typename T> struct YzShapes;
// {lanes, threads along the sweep, faces per thread} of tile variants 1..3
template <> struct YzShapes<float> {
  static constexpr int X1 = 32, D1 = 16, F1 = 1, X2 = 32, D2 = 8, F2 = 2, X3 = 32, D3 = 4, F3 = 4;
};
template <> struct YzShapes<double> {
  static constexpr int X1 = 16, D1 = 16, F1 = 1, X2 = 16, D2 = 8, F2 = 2, X3 = 32, D3 = 4, F3 = 4;
};
constexpr int kYzVariants = 4;

template <typename T, int D, int N, int R>
void launch_yz_v(ostc_ctx *ctx, BlockRes &B, DevState in, int variant) {
  const DevBlock &b = B.db;
  const int n_dir = D == 1 ? b.my : b.mz, n_o = D == 1 ? b.mz : b.my;
  if (variant >= 1 && variant <= 3) {
    using S = YzShapes<T>;
#define OSTC_TILE(X, DD, F)                                                                             \
  {                                                                                                   \
    constexpr int TF = DD * F;                                                                        \
    dim3 grid((b.mx + X - 1) / X, (n_dir + TF - 2) / (TF - 1), n_o);                                   \
    k_flux_tile<D, N, R, T, X, DD, F><<<grid, dim3(X, DD), tile_smem_bytes<N, X, TF, T>(), ctx->stream>>>( \
        b, in, B.dq);                                                                                 \
  }
    if (variant == 1) OSTC_TILE(S::X1, S::D1, S::F1)
    else if (variant == 2) OSTC_TILE(S::X2, S::D2, S::F2)
    else OSTC_TILE(S::X3, S::D3, S::F3)
#undef OSTC_TILE
    return;
  }
  // split columns into segments so that the grid fills the GPU at least ~4 waves deep
  const long long cols = (long long)((b.mx + 31) / 32) * ((n_o + 1) / 2);
  int nseg = (int)std::max<long long>(1, (ctx->sm_count * 12 + cols - 1) / cols);
  int seg = std::max(2 * N, (n_dir + nseg - 1) / nseg);
  nseg = (n_dir + seg - 1) / seg;
  dim3 grid((b.mx + 31) / 32, (n_o + 1) / 2, nseg);
  k_flux_march<D, N, R, T><<<grid, dim3(32, 2, 1), march_smem_bytes<T>(N), ctx->stream>>>(b, in, B.dq, seg);
}

// x sweep variants: 0 = one thread per face (k_flux_x) is the only shape; splitting each face over
// two warps (by side or by characteristic field) was measured 1.3-1.7x slower at 512x256x128 (more
// shared-memory reads, repeated Roe averages, spills at the register budget of twice the warps).
constexpr int kXVariants = 1;

template <typename T, int N, int R>
void launch_x_v(ostc_ctx *ctx, BlockRes &B, DevState in, int variant) {
  (void)variant;
  const DevBlock &b = B.db;
  k_flux_x<N, R, T><<<dim3((b.mx + 126) / 127, b.my, b.mz), 128, 0, ctx->stream>>>(b, in, B.dq);
}

template <typename T>
void launch_x(ostc_ctx *ctx, BlockRes &B, DevState in, int variant) {
  const int ng = ctx->der.ngg, rs = ctx->der.riemann;
  if (ng == 3) {
    if (rs == 4) launch_x_v<T, 3, 4>(ctx, B, in, variant);
    else if (rs == 1) launch_x_v<T, 3, 1>(ctx, B, in, variant);
    else launch_x_v<T, 3, 3>(ctx, B, in, variant);
  } else {
    if (rs == 4) launch_x_v<T, 4, 4>(ctx, B, in, variant);
    else if (rs == 1) launch_x_v<T, 4, 1>(ctx, B, in, variant);
    else launch_x_v<T, 4, 3>(ctx, B, in, variant);
  }
}

template <typename T, int D>
void launch_yz(ostc_ctx *ctx, BlockRes &B, DevState in, int variant) {
  const int ng = ctx->der.ngg, rs = ctx->der.riemann;
  if (ng == 3) {
    if (rs == 4) launch_yz_v<T, D, 3, 4>(ctx, B, in, variant);
    else if (rs == 1) launch_yz_v<T, D, 3, 1>(ctx, B, in, variant);
    else launch_yz_v<T, D, 3, 3>(ctx, B, in, variant);
  } else {
    if (rs == 4) launch_yz_v<T, D, 4, 4>(ctx, B, in, variant);
    else if (rs == 1) launch_yz_v<T, D, 4, 1>(ctx, B, in, variant);
    else launch_yz_v<T, D, 4, 3>(ctx, B, in, variant);
  }
}

// Autotuner of the x, y and z sweeps: on the context's current state (the sweeps only read the state
// and write or accumulate into the dq scratch), time every variant for each block, direction and the active
// precision with CUDA events on the library stream, and keep the fastest.  Runs once per precision,
// outside any stream capture, before the step graph is built.  Results are cached in the process by
// (device, block extents, ngg, scheme, precision, direction), so further contexts of the same shape
// (other blocks of the same extents, a second solver on the same case) reuse them.
using TuneKey = std::tuple<int, int, int, int, int, int, int, int, int>;
std::map<TuneKey, int> g_tune_cache;
std::mutex g_tune_mutex;

template <typename T>
int autotune_yz(ostc_ctx *ctx) {
  const int pi = std::is_same_v<T, float> ? 1 : 0;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  for (auto &B : ctx->blk) {
    const DevState in = state_of(B, 0);
    for (int dir = 0; dir <= (B.db.mz > 1 ? 2 : 1); ++dir) {
      const TuneKey key{ctx->device, B.db.mx, B.db.my, B.db.mz, B.db.g, ctx->der.riemann, ctx->der.inviscid_type, pi, dir};
      int &slot = dir == 0 ? B.x_var[pi] : B.yz_var[pi][dir - 1];
      if (ctx->forced[pi][dir] >= 0) {
        slot = ctx->forced[pi][dir];
        continue;
      }
      {
        std::lock_guard<std::mutex> lk(g_tune_mutex);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
          slot = it->second;
          continue;
        }
      }
      float best = 1e30f;
      int bv = 0;
      for (int v = 0; v < (dir == 0 ? kXVariants : kYzVariants); ++v) {
        auto run = [&]() {
          if (dir == 0) launch_x<T>(ctx, B, in, v);
          else if (dir == 1) launch_yz<T, 1>(ctx, B, in, v);
          else launch_yz<T, 2>(ctx, B, in, v);
        };
        run();  // warm-up
        CK(cudaEventRecord(e0, ctx->stream));
        for (int r = 0; r < 3; ++r) run();
        CK(cudaEventRecord(e1, ctx->stream));
        CK(cudaEventSynchronize(e1));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        B.tune_ms[pi][dir][v] = ms / 3;
        if (ms < best) {
          best = ms;
          bv = v;
        }
      }
      slot = bv;
      std::lock_guard<std::mutex> lk(g_tune_mutex);
      g_tune_cache[key] = bv;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  CK(cudaGetLastError());
  return OSTC_OK;
}

// inviscid sweep of one block
template <typename T>
int launch_flux(ostc_ctx *ctx, BlockRes &B, DevState in) {
  if (ctx->der.inviscid_type == 3) {
    // the flux-split sweeps accumulate: the air path starts dq from zero here (mixtures start it with
    // the chemical source)
    if (!ctx->mixture) cudaMemsetAsync(B.dq, 0, (size_t)ctx->nv * B.db.n * sizeof(double), ctx->stream);
    launch_fvs(ctx, B, in);
    return OSTC_OK;
  }
  if (ctx->der.inviscid_type != 1) {
    launch_flux_pv<T>(ctx, B, in);
    return OSTC_OK;
  }
  const DevBlock &b = B.db;
  const int ng = ctx->der.ngg, rs = ctx->der.riemann;
  const bool is3d = b.mz > 1;
  // x: the variant the autotuner chose for this block and precision
  {
    (void)ng;
    (void)rs;
    long tok = begin_t(ctx, "flux_x");
    const int v = B.x_var[ctx->precision == OSTC_PREC_MIXED];
    launch_x<T>(ctx, B, in, v < 0 ? 0 : v);
    end_t(ctx, tok);
  }
  // y and z: the variant the autotuner chose for this block and precision (column march by default)
  for (int dir = 1; dir <= (is3d ? 2 : 1); ++dir) {
    const int v = B.yz_var[ctx->precision == OSTC_PREC_MIXED][dir - 1];
    long tok = begin_t(ctx, dir == 1 ? "flux_y" : "flux_z");
    if (dir == 1) launch_yz<T, 1>(ctx, B, in, v < 0 ? 0 : v);
    else launch_yz<T, 2>(ctx, B, in, v < 0 ? 0 : v);
    end_t(ctx, tok);
  }
  return OSTC_OK;
}

template <typename T>
void launch_visc(ostc_ctx *ctx, BlockRes &B, const StageArgs &a) {
  const DevBlock &b = B.db;
  long tok = begin_t(ctx, "visc_update");
  if (b.mz > 1) {
    constexpr int TX = 32, TY = 4;
    const long long cols = (long long)((b.mx + TX - 1) / TX) * ((b.my + TY - 1) / TY);
    int nseg = (int)std::max<long long>(1, (ctx->sm_count * 8 + cols - 1) / cols);
    int kseg = std::max(4, (b.mz + nseg - 1) / nseg);
    nseg = (b.mz + kseg - 1) / kseg;
    dim3 grid((b.mx + TX - 1) / TX, (b.my + TY - 1) / TY, nseg);
    k_visc_update<T, true, TX, TY>
        <<<grid, dim3(TX, TY, 1), visc_smem_bytes<T, true, TX, TY>(), ctx->stream>>>(b, a, B.dq, kseg);
  } else {
    constexpr int TX = 32, TY = 4;
    dim3 grid((b.mx + TX - 1) / TX, (b.my + TY - 1) / TY, 1);
    k_visc_update<T, false, TX, TY>
        <<<grid, dim3(TX, TY, 1), visc_smem_bytes<T, false, TX, TY>(), ctx->stream>>>(b, a, B.dq, 1);
  }
  end_t(ctx, tok);
}

void launch_carry(ostc_ctx *ctx, BlockRes &B, DevState in, DevState out) {
  for (const auto &fi : B.inner) {
    const long long tot = (long long)fi.n_point[0] * fi.n_point[1] * fi.n_point[2];
    k_inner_carry<<<grid_for(ctx, tot, 128), 128, 0, ctx->stream>>>(B.db, in, out, fi);
  }
}

// generate_random_numbers + apply_convolution (DigitalFilter.cu:367-397) and compute_fluctuations
// (:399-407) of the filter, dtp the device dt the time correlation uses.
void enqueue_df_fluctuations(ostc_ctx *ctx, const double *dtp, const DevFace &f) {
  const DevDf &d = ctx->df;
  const cudaStream_t st = ctx->stream;
  k_df_generate<<<grid_for(ctx, (long long)d.wy * d.wz * 3, 128), 128, 0, st>>>(d);
  k_df_remove_mean<<<(d.wy + 127) / 128, 128, 0, st>>>(d);
  k_df_periodic<<<grid_for(ctx, (long long)d.wy * (kDfN + d.g), 128), 128, 0, st>>>(d);
  k_df_conv_y<<<grid_for(ctx, (long long)d.py * d.wz, 128), 128, 0, st>>>(d);
  k_df_conv_z<<<grid_for(ctx, (long long)d.py * d.pz, 128), 128, 0, st>>>(d);
  k_df_correlate<<<grid_for(ctx, (long long)d.py * d.pz, 128), 128, 0, st>>>(d, dtp, f.u, f.lower[1], f.delta_omega);
}

// The filter's start (DigitalFilter.cu:226-247): generator states from seed, one random field and its
// convolutions taken as the previous field, and the first fluctuations from it.
void df_start(ostc_ctx *ctx, unsigned long long seed) {
  const DevDf &d = ctx->df;
  const cudaStream_t st = ctx->stream;
  const long long ns = (long long)d.wy * d.wz * 3, np = (long long)d.py * d.pz;
  k_df_rng_init<<<grid_for(ctx, ns, 128), 128, 0, st>>>(d.rng, ns, seed);
  k_df_generate<<<grid_for(ctx, ns, 128), 128, 0, st>>>(d);
  k_df_remove_mean<<<(d.wy + 127) / 128, 128, 0, st>>>(d);
  k_df_periodic<<<grid_for(ctx, (long long)d.wy * (kDfN + d.g), 128), 128, 0, st>>>(d);
  k_df_conv_y<<<grid_for(ctx, (long long)d.py * d.wz, 128), 128, 0, st>>>(d);
  k_df_conv_z<<<grid_for(ctx, np, 128), 128, 0, st>>>(d);
  cudaMemcpyAsync(d.vold, d.vnew, 3 * np * sizeof(double), cudaMemcpyDeviceToDevice, st);
  k_df_first<<<grid_for(ctx, np, 128), 128, 0, st>>>(d);
}

// gam_prev: where a mixture far-field face reads the gamma of its face node - the properties of the
// stage input (the reference's in-place state holds the last properties sweep there); null = out's.
void launch_bcs(ostc_ctx *ctx, int block, DevState out, const double *gam_prev = nullptr) {
  for (const auto &bf : ctx->order) {
    if (bf.first != block) continue;
    BlockRes &B = ctx->blk[block];
    const DevFace &f = B.faces[bf.second];
    const int t0 = f.face == 0 ? 1 : 0, t1 = f.face == 2 ? 1 : 2;
    const long long nn = (long long)(f.re[t0] - f.rs[t0] + 1) * (f.re[t1] - f.rs[t1] + 1);
    long tok = begin_t(ctx, "bc_face");
    if (f.type == kInflow && f.fluct == 11) {
      // the digital filter (BoundCond.cuh:1561-1573): new random field, its convolutions, the time
      // correlation with the current dt (zero at the initial application unless dt is fixed), then the
      // inflow plane
      enqueue_df_fluctuations(ctx, ctx->bc_initial && !ctx->der.fixed_time_step ? ctx->d_zero : ctx->d_dt, f);
      const long long np = (long long)ctx->df.py * ctx->df.pz;
      k_df_apply<<<grid_for(ctx, np, 128), 128, 0, ctx->stream>>>(B.db, out, f, ctx->df, ctx->df_mw_up,
                                                                   ctx->df_mw_lo);
    } else {
      k_bc_face<<<grid_for(ctx, nn, 128), 128, 0, ctx->stream>>>(B.db, out, f, gam_prev ? gam_prev : out.gam);
    }
    end_t(ctx, tok);
  }
}

DevState state_of(BlockRes &B, int s);

// data_communication (DataCommunication.cuh:29-58): every interface of every block in file order.
void launch_interfaces(ostc_ctx *ctx, int slot) {
  for (auto &B : ctx->blk)
    for (size_t f = 0; f < B.inner.size(); ++f) {
      BlockRes &T = ctx->blk[B.inner_target[f]];
      const DevInner &fi = B.inner[f];
      const long long tot = (long long)fi.n_point[0] * fi.n_point[1] * fi.n_point[2];
      long tok = begin_t(ctx, "interface");
      k_inner_face<<<grid_for(ctx, tot, 128), 128, 0, ctx->stream>>>(B.db, state_of(B, slot), T.db, state_of(T, slot), fi);
      end_t(ctx, tok);
    }
}

DevState state_of(BlockRes &B, int s) {
  DevState d{B.cv[s], B.bv[s], B.mul[s]};
  d.sv = B.sv[s];
  d.cond = B.cond[s];
  d.rhod = B.rhod[s];
  d.gam = B.gam[s];
  d.acs = B.acs[s];
  return d;
}

// The march kernels stage 2*ngg+1 nodes x 11 values x 64 threads (plus the FP32 prefetch buffers)
// in dynamic shared memory (up to 51 KB); raise the per-kernel limit once, outside any stream capture.
template <typename T>
bool set_march_attrs() {
  bool ok = true;
  auto set = [&](const void *fn, int ng) {
    const int bytes = (int)march_smem_bytes<T>(ng);
    ok = ok && cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) == cudaSuccess;
  };
  set((const void *)k_flux_march<1, 3, 1, T>, 3);
  set((const void *)k_flux_march<1, 3, 3, T>, 3);
  set((const void *)k_flux_march<1, 3, 4, T>, 3);
  set((const void *)k_flux_march<1, 4, 1, T>, 4);
  set((const void *)k_flux_march<1, 4, 3, T>, 4);
  set((const void *)k_flux_march<1, 4, 4, T>, 4);
  set((const void *)k_flux_march<2, 3, 1, T>, 3);
  set((const void *)k_flux_march<2, 3, 3, T>, 3);
  set((const void *)k_flux_march<2, 3, 4, T>, 3);
  set((const void *)k_flux_march<2, 4, 1, T>, 4);
  set((const void *)k_flux_march<2, 4, 3, T>, 4);
  set((const void *)k_flux_march<2, 4, 4, T>, 4);
  auto tset = [&](const void *fn, size_t bytes) {
    ok = ok && cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) == cudaSuccess;
  };
  using S = YzShapes<T>;
#define OSTC_TSET(D, N, R)                                                                                      \
  tset((const void *)k_flux_tile<D, N, R, T, S::X1, S::D1, S::F1>, tile_smem_bytes<N, S::X1, S::D1 * S::F1, T>()); \
  tset((const void *)k_flux_tile<D, N, R, T, S::X2, S::D2, S::F2>, tile_smem_bytes<N, S::X2, S::D2 * S::F2, T>()); \
  tset((const void *)k_flux_tile<D, N, R, T, S::X3, S::D3, S::F3>, tile_smem_bytes<N, S::X3, S::D3 * S::F3, T>());
  OSTC_TSET(1, 3, 1) OSTC_TSET(1, 3, 3) OSTC_TSET(1, 3, 4) OSTC_TSET(1, 4, 1) OSTC_TSET(1, 4, 3) OSTC_TSET(1, 4, 4)
  OSTC_TSET(2, 3, 1) OSTC_TSET(2, 3, 3) OSTC_TSET(2, 3, 4) OSTC_TSET(2, 4, 1) OSTC_TSET(2, 4, 3) OSTC_TSET(2, 4, 4)
#undef OSTC_TSET
  ok = ok && cudaFuncSetAttribute((const void *)k_visc_update<T, true, 32, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)visc_smem_bytes<T, true, 32, 4>()) == cudaSuccess;
  ok = ok && cudaFuncSetAttribute((const void *)k_visc_update<T, false, 32, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)visc_smem_bytes<T, false, 32, 4>()) == cudaSuccess;
  return ok;
}

// dynamic shared memory of the flux-split and mixture viscous sweeps (up to ~45 KB at n_var 14)
bool set_mix_attrs(int nv) {
  bool ok = true;
  auto set = [&](const void *fn, size_t bytes) {
    ok = ok && cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) == cudaSuccess;
  };
#define OSTC_FSET(T)                                                      \
  set((const void *)k_fvs<0, 0, T>, fvs_smem_bytes<0, T>(nv));            \
  set((const void *)k_fvs<1, 0, T>, fvs_smem_bytes<1, T>(nv));            \
  set((const void *)k_fvs<2, 0, T>, fvs_smem_bytes<2, T>(nv));            \
  set((const void *)k_fvs<0, kFixedNS, T>, fvs_smem_bytes<0, T>(nv));     \
  set((const void *)k_fvs<1, kFixedNS, T>, fvs_smem_bytes<1, T>(nv));     \
  set((const void *)k_fvs<2, kFixedNS, T>, fvs_smem_bytes<2, T>(nv));
  OSTC_FSET(double)
  OSTC_FSET(float)
#undef OSTC_FSET
  set((const void *)k_adj_fvs<0, 0>, adj_fvs_smem_bytes<0>(nv));
  set((const void *)k_adj_fvs<1, 0>, adj_fvs_smem_bytes<1>(nv));
  set((const void *)k_adj_fvs<2, 0>, adj_fvs_smem_bytes<2>(nv));
  set((const void *)k_adj_fvs<0, kFixedNS>, adj_fvs_smem_bytes<0>(nv));
  set((const void *)k_adj_fvs<1, kFixedNS>, adj_fvs_smem_bytes<1>(nv));
  set((const void *)k_adj_fvs<2, kFixedNS>, adj_fvs_smem_bytes<2>(nv));
  return ok;
}

int initialise(ostc_ctx *ctx) {
  // Driver::initialize_computation (Driver.cu:115-199): BCs, properties, then cv <- bv (RK.cuh:37-45)
  ctx->bc_initial = true;
  for (size_t b = 0; b < ctx->blk.size(); ++b) launch_bcs(ctx, (int)b, state_of(ctx->blk[b], 0));
  ctx->bc_initial = false;
  launch_interfaces(ctx, 0);
  for (auto &B : ctx->blk) {
    if (ctx->mixture) {
      launch_mix_props(ctx, B, state_of(B, 0));
      k_mix_init_cv<0><<<grid_for(ctx, B.db.plane, 128), 128, 0, ctx->stream>>>(B.db, state_of(B, 0));
    } else {
      k_init_fields<<<grid_for(ctx, B.db.plane, 256), 256, 0, ctx->stream>>>(B.db, state_of(B, 0));
    }
  }
  CK(cudaGetLastError());
  ctx->initialised = true;
  return OSTC_OK;
}

// Run f(b) for every block.  Multi-block steps fork the blocks onto the side streams (block b on
// side[b % n]) and join them back before returning, so independent blocks' sweeps fill the GPU
// together; with per-kernel timing on (ostc_profile_steps) the blocks run one after another.
template <class F>
void for_blocks(ostc_ctx *ctx, F f) {
  const size_t nb = ctx->blk.size();
  if (nb == 1 || ctx->timing || ctx->side.empty() || ctx->launch_mode == OSTC_LAUNCH_BLOCK_LOOP) {
    for (size_t b = 0; b < nb; ++b) f((int)b);
    return;
  }
  cudaStream_t main = ctx->stream;
  cudaEventRecord(ctx->fork_ev, main);
  const size_t ns = ctx->side.size();
  for (size_t k = 0; k < ns; ++k) cudaStreamWaitEvent(ctx->side[k], ctx->fork_ev, 0);
  for (size_t b = 0; b < nb; ++b) {
    ctx->stream = ctx->side[b % ns];
    f((int)b);
  }
  ctx->stream = main;
  for (size_t k = 0; k < ns; ++k) {
    cudaEventRecord(ctx->side_ev[k], ctx->side[k]);
    cudaStreamWaitEvent(main, ctx->side_ev[k], 0);
  }
}

// One SSP-RK3 step over all blocks (RK.cuh:85-185).
// CFL time step of the current state (slot 0) into d_dt (local_time_step + global_time_step)
void enqueue_cfl_dt(ostc_ctx *ctx) {
  long tok = begin_t(ctx, "cfl_dt");
  k_dt_reset<<<1, 1, 0, ctx->stream>>>(ctx->d_dtbits);
  for (auto &B : ctx->blk)
    k_cfl_dt<<<grid_for(ctx, B.db.n, 256), 256, 0, ctx->stream>>>(B.db, state_of(B, 0), ctx->der.cfl,
                                                                 ctx->der.prandtl, B.db.mz > 1, ctx->d_dtbits);
  k_dt_decode<<<1, 1, 0, ctx->stream>>>(ctx->d_dtbits, ctx->d_dt);
  end_t(ctx, tok);
}

// Stage rk (0..2) of an air SSP-RK3 step: state slot rk -> slot (rk + 1) % 3 (or sout_override), with
// slot 0 the step's start state and d_dt the step's dt.
template <typename T>
void enqueue_air_stage(ostc_ctx *ctx, int rk, int sout_override = -1) {
  static const double A[3] = {1.0, 0.75, 1.0 / 3.0}, Bc[3] = {0.0, 0.25, 2.0 / 3.0}, C[3] = {1.0, 0.25, 2.0 / 3.0};
  const int sin = rk, sout = sout_override >= 0 ? sout_override : (rk + 1) % 3;
  for_blocks(ctx, [&](int bi) {
    BlockRes &B = ctx->blk[bi];
    launch_flux<T>(ctx, B, state_of(B, sin));
    StageArgs a{};
    a.in = state_of(B, sin);
    a.qn = state_of(B, 0);
    a.out = state_of(B, sout);
    a.a = A[rk];
    a.bcoef = Bc[rk];
    a.c = C[rk];
    a.dt = ctx->d_dt;
    a.prandtl = ctx->der.prandtl;
    a.viscous = ctx->der.viscous_order != 0;
    a.update = 1;
    a.flags = ctx->d_flags;
    launch_visc<T>(ctx, B, a);
    launch_carry(ctx, B, state_of(B, sin), state_of(B, sout));
    launch_bcs(ctx, bi, state_of(B, sout), state_of(B, sin).gam);
  });
  launch_interfaces(ctx, sout);
}

// One SSP-RK3 step of the air path: CFL dt from slot 0, then the three stages (A -> B -> C -> A).
template <typename T>
int enqueue_step(ostc_ctx *ctx) {
  if (!ctx->der.fixed_time_step) enqueue_cfl_dt(ctx);
  for (int rk = 0; rk < 3; ++rk) enqueue_air_stage<T>(ctx, rk);
  k_step_end<<<1, 1, 0, ctx->stream>>>(ctx->d_time, ctx->d_dt, ctx->d_step);
  return OSTC_OK;
}

// Stage rk (0..2) of a mixture SSP-RK3 step: state slot rk -> slot (rk + 1) % 3, with slot 0 the
// step's start state and d_dt the step's dt.
void enqueue_mix_stage(ostc_ctx *ctx, int rk, int sout_override = -1) {
  static const double A[3] = {1.0, 0.75, 1.0 / 3.0}, Bc[3] = {0.0, 0.25, 2.0 / 3.0}, C[3] = {1.0, 0.25, 2.0 / 3.0};
  const int nv = ctx->nv;
  const int sin = rk, sout = sout_override >= 0 ? sout_override : (rk + 1) % 3;
  for_blocks(ctx, [&](int bi) {
    BlockRes &B = ctx->blk[bi];
    const DevState in = state_of(B, sin);
    const bool chem = ctx->der.reaction == 1, implicit = chem && ctx->chem_mode == OSTC_CHEM_POINT_IMPLICIT;
    {
      long tok = begin_t(ctx, "source");
      launch_mix_source(ctx, B, in, chem && !implicit);
      end_t(ctx, tok);
    }
    launch_mix_inviscid(ctx, B, in);
    if (ctx->der.viscous_order != 0) launch_mix_visc(ctx, B, in);
    if (implicit) launch_chem_epi(ctx, B, in);
    {
      long tok = begin_t(ctx, "update");
      if (ctx->der.n_spec == kFixedNS)
        k_mix_update<kFixedNS><<<grid_for(ctx, B.db.n, 128), 128, 0, ctx->stream>>>(
            B.db, in, state_of(B, 0), state_of(B, sout), B.dq, ctx->d_dt, A[rk], Bc[rk], C[rk], nv, ctx->d_flags);
      else
        k_mix_update<0><<<grid_for(ctx, B.db.n, 128), 128, 0, ctx->stream>>>(
            B.db, in, state_of(B, 0), state_of(B, sout), B.dq, ctx->d_dt, A[rk], Bc[rk], C[rk], nv, ctx->d_flags);
      end_t(ctx, tok);
    }
    launch_carry(ctx, B, in, state_of(B, sout));
    launch_bcs(ctx, bi, state_of(B, sout), in.gam);
  });
  launch_interfaces(ctx, sout);
  for_blocks(ctx, [&](int bi) {
    long tok = begin_t(ctx, "properties");
    launch_mix_props(ctx, ctx->blk[bi], state_of(ctx->blk[bi], sout));
    end_t(ctx, tok);
  });
}

// One SSP-RK3 step of a mixture (RK.cuh:85-185 with MixtureModel Mixture / FR): source, flux-split
// WENO7, viscous, update + temperature Newton, boundary faces, properties, per stage.
int enqueue_step_mix(ostc_ctx *ctx) {
  if (!ctx->der.fixed_time_step) enqueue_cfl_dt(ctx);
  for (int rk = 0; rk < 3; ++rk) enqueue_mix_stage(ctx, rk);
  k_step_end<<<1, 1, 0, ctx->stream>>>(ctx->d_time, ctx->d_dt, ctx->d_step);
  return OSTC_OK;
}

// ---- adjoint entry points' shared pieces

// what the adjoint covers: the multi-component path, explicit chemistry, one block, periodic and
// outflow faces
// step: the step adjoint (ostc_rk3_step_vjp, ostc_adjoint_steps) rather than ostc_rhs_vjp (the same
// coverage today)
int adjoint_check(ostc_ctx *ctx, unsigned mask, bool step = false) {
  (void)step;
  if (!ctx->mixture) {
    if ((mask & OSTC_TERM_INVISCID) && ctx->der.inviscid_type != 1) {
      ctx->err = "the air adjoint's inviscid term is the AWENO path (WENO5-Z / WENO7-Z with a Riemann solver)";
      return OSTC_EINVAL;
    }
  }
  if (ctx->mixture && (mask & OSTC_TERM_INVISCID) && ctx->der.inviscid_type != 3) {
    ctx->err = "the adjoint's inviscid term is the flux-split WENO (inviscid_scheme 71 / 72)";
    return OSTC_EINVAL;
  }
  if ((mask & OSTC_TERM_SOURCE) && ctx->der.reaction == 1 && ctx->chem_mode == OSTC_CHEM_POINT_IMPLICIT) {
    ctx->err = "the point-implicit chemistry mode has no adjoint; use the explicit source";
    return OSTC_EINVAL;
  }
  if (ctx->blk.size() > 1 || !ctx->blk[0].inner.empty()) {
    ctx->err = "the adjoint covers single-block cases (interfaces couple the blocks' right-hand sides)";
    return OSTC_EINVAL;
  }
  for (const auto &f : ctx->blk[0].faces)
    if (f.type != kPeriodic && f.type != kOutflow) {
      ctx->err = "the adjoint covers periodic and outflow boundary faces";
      return OSTC_EINVAL;
    }
  return OSTC_OK;
}

int adjoint_alloc(ostc_ctx *ctx, BlockRes &B) {
  if (B.adj) return OSTC_OK;
  const int nv = ctx->nv, ns = ctx->der.n_spec;
  const long long P = B.db.plane;
  CK(cudaMalloc(&B.adj, (size_t)(nv + 9 + 2 * ns) * P * sizeof(double)));
  CK(cudaMalloc(&B.dqb, (size_t)nv * B.db.n * sizeof(double)));
  CK(cudaMalloc(&B.adj_work, (size_t)4 * (nv + 1) * B.db.n * sizeof(double)));
  if (!ctx->mixture) return OSTC_OK;  // air: the step adjoint needs no fourth state slot
  // state slot 3 (zeroed: its padding columns must read as empty nodes)
  auto alloc = [&](double **p, size_t n) -> int {
    if (cudaMalloc(p, n * sizeof(double)) != cudaSuccess || cudaMemset(*p, 0, n * sizeof(double)) != cudaSuccess)
      return OSTC_ENOMEM;
    return OSTC_OK;
  };
  int r = alloc(&B.cv[3], (size_t)nv * P);
  if (!r) r = alloc(&B.bv[3], 6 * P);
  if (!r) r = alloc(&B.mul[3], P);
  if (!r) r = alloc(&B.sv[3], (size_t)ns * P);
  if (!r) r = alloc(&B.rhod[3], (size_t)ns * P);
  if (!r) r = alloc(&B.cond[3], P);
  if (!r) r = alloc(&B.gam[3], P);
  if (!r) r = alloc(&B.acs[3], P);
  if (r) ctx->err = "device allocation for the adjoint failed";
  return r;
}

// out (device, n_var x N) = (d dq / d cv)^T B.dqb at the state in `slot` of block `block`.  With
// out_t null the state's T is the equation-of-state root of its cv (its adjoint goes to cv); else T
// is a state variable and out_t (device, N) receives (d dq / d T)^T B.dqb.
template <int NG, int RS>
void launch_adjoint_air_inviscid(ostc_ctx *ctx, BlockRes &B, DevState in, double *acv) {
  const DevBlock &b = B.db;
  const long long fx = (long long)(b.mx + 1) * b.my * b.mz, fy = (long long)b.mx * (b.my + 1) * b.mz;
  const long long cx = (long long)(b.mx + 2 * NG) * b.my * b.mz, cy = (long long)b.mx * (b.my + 2 * NG) * b.mz;
  k_adj_air_face<0, NG, RS><<<grid_for(ctx, fx, 128), 128, 0, ctx->stream>>>(b, in, B.dqb, acv);
  k_adj_air_cds<0, NG><<<grid_for(ctx, cx, 128), 128, 0, ctx->stream>>>(b, in, B.dqb, acv);
  k_adj_air_face<1, NG, RS><<<grid_for(ctx, fy, 128), 128, 0, ctx->stream>>>(b, in, B.dqb, acv);
  k_adj_air_cds<1, NG><<<grid_for(ctx, cy, 128), 128, 0, ctx->stream>>>(b, in, B.dqb, acv);
  if (b.mz > 1) {
    const long long fz = (long long)b.mx * b.my * (b.mz + 1), cz = (long long)b.mx * b.my * (b.mz + 2 * NG);
    k_adj_air_face<2, NG, RS><<<grid_for(ctx, fz, 128), 128, 0, ctx->stream>>>(b, in, B.dqb, acv);
    k_adj_air_cds<2, NG><<<grid_for(ctx, cz, 128), 128, 0, ctx->stream>>>(b, in, B.dqb, acv);
  }
}

// (d dq / d cv)^T B.dqb of the air path (ostc_adj_air.cuh) at the state in `slot`: cv adjoint planes
// from the face, central-correction and viscous terms, ghost folds in the reverse of the face order,
// interior gathered into out.
int vjp_air(ostc_ctx *ctx, int block, int slot, unsigned mask, double *out) {
  BlockRes &B = ctx->blk[block];
  const DevBlock &b = B.db;
  const long long P = b.plane;
  double *acv = B.adj;
  CK(cudaMemsetAsync(acv, 0, (size_t)5 * P * sizeof(double), ctx->stream));
  const DevState in = state_of(B, slot);
  if (mask & OSTC_TERM_INVISCID) {
    const int ng = ctx->der.ngg, rs = ctx->der.riemann;
    if (ng == 3) {
      if (rs == 4) launch_adjoint_air_inviscid<3, 4>(ctx, B, in, acv);
      else if (rs == 1) launch_adjoint_air_inviscid<3, 1>(ctx, B, in, acv);
      else launch_adjoint_air_inviscid<3, 3>(ctx, B, in, acv);
    } else {
      if (rs == 4) launch_adjoint_air_inviscid<4, 4>(ctx, B, in, acv);
      else if (rs == 1) launch_adjoint_air_inviscid<4, 1>(ctx, B, in, acv);
      else launch_adjoint_air_inviscid<4, 3>(ctx, B, in, acv);
    }
  }
  if ((mask & OSTC_TERM_VISCOUS) && ctx->der.viscous_order != 0) {
    const double pr = ctx->der.prandtl;
    const long long fx = (long long)(b.mx + 1) * b.my * b.mz, fy = (long long)b.mx * (b.my + 1) * b.mz;
    if (b.mz > 1) {
      const long long fz = (long long)b.mx * b.my * (b.mz + 1);
      k_adj_air_visc<0, true><<<grid_for(ctx, fx, 128), 128, 0, ctx->stream>>>(b, in, B.dqb, pr, acv);
      k_adj_air_visc<1, true><<<grid_for(ctx, fy, 128), 128, 0, ctx->stream>>>(b, in, B.dqb, pr, acv);
      k_adj_air_visc<2, true><<<grid_for(ctx, fz, 128), 128, 0, ctx->stream>>>(b, in, B.dqb, pr, acv);
    } else {
      k_adj_air_visc<0, false><<<grid_for(ctx, fx, 128), 128, 0, ctx->stream>>>(b, in, B.dqb, pr, acv);
      k_adj_air_visc<1, false><<<grid_for(ctx, fy, 128), 128, 0, ctx->stream>>>(b, in, B.dqb, pr, acv);
    }
  }
  for (auto it = ctx->order.rbegin(); it != ctx->order.rend(); ++it) {
    if (it->first != block) continue;
    const DevFace &f = B.faces[it->second];
    const int t0 = f.face == 0 ? 1 : 0, t1 = f.face == 2 ? 1 : 2;
    const long long nn = (long long)(f.re[t0] - f.rs[t0] + 1) * (f.re[t1] - f.rs[t1] + 1);
    k_adj_air_bc_face<<<grid_for(ctx, nn, 128), 128, 0, ctx->stream>>>(b, acv, f);
  }
  k_adj_gather<<<grid_for(ctx, b.n, 128), 128, 0, ctx->stream>>>(b, acv, 5, out);
  CK(cudaGetLastError());
  return OSTC_OK;
}

int vjp_core(ostc_ctx *ctx, int block, int slot, unsigned mask, double *out, double *out_t = nullptr) {
  if (!ctx->mixture) return vjp_air(ctx, block, slot, mask, out);
  BlockRes &B = ctx->blk[block];
  const int nv = ctx->nv, ns = ctx->der.n_spec;
  const long long P = B.db.plane;
  CK(cudaMemsetAsync(B.adj, 0, (size_t)(nv + 9 + 2 * ns) * P * sizeof(double), ctx->stream));
  DevAdj A;
  A.cv = B.adj;
  A.p = A.cv + nv * P;
  A.c = A.p + P;
  A.rho = A.c + P;
  A.vel = A.rho + P;
  A.T = A.vel + 3 * P;
  A.Y = A.T + P;
  A.mu = A.Y + ns * P;
  A.lam = A.mu + P;
  A.rhod = A.lam + P;
  const DevState in = state_of(B, slot);
  if (ns == kFixedNS) launch_adjoint_t<kFixedNS>(ctx, B, in, mask, A);
  else launch_adjoint_t<0>(ctx, B, in, mask, A);
  for (auto it = ctx->order.rbegin(); it != ctx->order.rend(); ++it) {
    if (it->first != block) continue;
    const DevFace &f = B.faces[it->second];
    const int t0 = f.face == 0 ? 1 : 0, t1 = f.face == 2 ? 1 : 2;
    const long long nn = (long long)(f.re[t0] - f.rs[t0] + 1) * (f.re[t1] - f.rs[t1] + 1);
    k_adj_bc_face<<<grid_for(ctx, nn, 128), 128, 0, ctx->stream>>>(B.db, A, ns, f);
  }
  if (ns == kFixedNS)
    k_adj_eos<kFixedNS><<<grid_for(ctx, B.db.n, 128), 128, 0, ctx->stream>>>(B.db, in, A, out_t ? 0 : 1);
  else
    k_adj_eos<0><<<grid_for(ctx, B.db.n, 128), 128, 0, ctx->stream>>>(B.db, in, A, out_t ? 0 : 1);
  k_adj_gather<<<grid_for(ctx, B.db.n, 128), 128, 0, ctx->stream>>>(B.db, A.cv, nv, out);
  if (out_t) k_adj_gather<<<grid_for(ctx, B.db.n, 128), 128, 0, ctx->stream>>>(B.db, A.T, 1, out_t);
  CK(cudaGetLastError());
  return OSTC_OK;
}

// Adjoint of one SSP-RK3 step from the state in slot 0 with the dt in d_dt.  The step's state is
// (cv, T): every stage's T is the temperature Newton iterate started from the stage input's T
// (k_mix_update), so T carries an adjoint of its own.  On entry the work buffers hold lam_cv' and
// lam_T' of the step's output, on return lam_cv and lam_T of slot 0.  With
// S1 = q + dt/J R(q), S2 = 3/4 q + 1/4 S1 + 1/4 dt/J R(S1), q' = 1/3 q + 2/3 S2 + 2/3 dt/J R(S2)
// (RK.cuh:10-14) and T_s = N(T_{s-1}; cv_s):
//   stage 3: lam_cv' += N'^T lam_T';  x2 = 2/3 lam_cv' + R'(S2)^T (2/3 dt/J lam_cv'),
//            x2_T = R'_T(S2)^T (...) + dN/dT_start lam_T'
//   stage 2: likewise from (x2, x2_T) to (x1, x1_T) with 1/4, stage 1 to q with 1;
//   lam_cv = 1/3 lam_cv' + 3/4 x2 + x1 + R'(q)^T (dt/J x1),  lam_T = R'_T(q)^T (...) + dN/dT_start x1_T.
// The air step: every stage's primitive state is the equation of state of its cv, so the state is cv
// alone and the stage adjoints chain through the right-hand-side VJPs (stage 3's output is not needed).
int step_vjp_air(ostc_ctx *ctx) {
  BlockRes &B = ctx->blk[0];
  const int nv = 5;
  const long long N = B.db.n, nt = (long long)nv * N;
  double *Lc = B.adj_work, *X2c = Lc + nt, *X1c = X2c + nt, *Gc = X1c + nt;
  const int g = grid_for(ctx, N, 128), gt = grid_for(ctx, nt, 256);
  enqueue_air_stage<double>(ctx, 0);  // S1 -> slot 1
  enqueue_air_stage<double>(ctx, 1);  // S2 -> slot 2
  k_adj_stage_seed<<<g, 128, 0, ctx->stream>>>(B.db, Lc, 2.0 / 3.0, ctx->d_dt, B.dqb, nv);
  if (int r = vjp_air(ctx, 0, 2, OSTC_TERM_ALL, X2c)) return r;
  k_axpby<<<gt, 256, 0, ctx->stream>>>(nt, 2.0 / 3.0, Lc, 1.0, X2c);
  k_adj_stage_seed<<<g, 128, 0, ctx->stream>>>(B.db, X2c, 0.25, ctx->d_dt, B.dqb, nv);
  if (int r = vjp_air(ctx, 0, 1, OSTC_TERM_ALL, X1c)) return r;
  k_axpby<<<gt, 256, 0, ctx->stream>>>(nt, 0.25, X2c, 1.0, X1c);
  k_adj_stage_seed<<<g, 128, 0, ctx->stream>>>(B.db, X1c, 1.0, ctx->d_dt, B.dqb, nv);
  if (int r = vjp_air(ctx, 0, 0, OSTC_TERM_ALL, Gc)) return r;
  k_axpby<<<gt, 256, 0, ctx->stream>>>(nt, 0.75, X2c, 1.0 / 3.0, Lc);
  k_axpby<<<gt, 256, 0, ctx->stream>>>(nt, 1.0, X1c, 1.0, Lc);
  k_axpby<<<gt, 256, 0, ctx->stream>>>(nt, 1.0, Gc, 1.0, Lc);
  CK(cudaGetLastError());
  return OSTC_OK;
}

int step_vjp(ostc_ctx *ctx) {
  if (!ctx->mixture) return step_vjp_air(ctx);
  BlockRes &B = ctx->blk[0];
  const int nv = ctx->nv;
  const long long N = B.db.n, nt = (long long)nv * N;
  double *Lc = B.adj_work, *X2c = Lc + nt, *X1c = X2c + nt, *Gc = X1c + nt;
  double *LT = Gc + nt, *X2T = LT + N, *X1T = X2T + N, *GT = X1T + N;
  const int g = grid_for(ctx, N, 128), gt = grid_for(ctx, nt, 256), g1 = grid_for(ctx, N, 256);
  auto newton = [&](int sin, int sout, const double *lt, double *lc, double *lts) {
    if (ctx->der.n_spec == kFixedNS)
      k_adj_newton<kFixedNS><<<g, 128, 0, ctx->stream>>>(B.db, state_of(B, sin), state_of(B, sout), lt, lc, lts);
    else
      k_adj_newton<0><<<g, 128, 0, ctx->stream>>>(B.db, state_of(B, sin), state_of(B, sout), lt, lc, lts);
  };
  enqueue_mix_stage(ctx, 0);     // S1 -> slot 1
  enqueue_mix_stage(ctx, 1);     // S2 -> slot 2
  enqueue_mix_stage(ctx, 2, 3);  // q' -> slot 3 (slot 0 keeps q)
  // stage 3
  CK(cudaMemsetAsync(X2T, 0, N * sizeof(double), ctx->stream));
  newton(2, 3, LT, Lc, X2T);
  k_adj_stage_seed<<<g, 128, 0, ctx->stream>>>(B.db, Lc, 2.0 / 3.0, ctx->d_dt, B.dqb, nv);
  if (int r = vjp_core(ctx, 0, 2, OSTC_TERM_ALL, X2c, GT)) return r;
  k_axpby<<<gt, 256, 0, ctx->stream>>>(nt, 2.0 / 3.0, Lc, 1.0, X2c);
  k_axpby<<<g1, 256, 0, ctx->stream>>>(N, 1.0, GT, 1.0, X2T);
  // stage 2
  CK(cudaMemsetAsync(X1T, 0, N * sizeof(double), ctx->stream));
  newton(1, 2, X2T, X2c, X1T);
  k_adj_stage_seed<<<g, 128, 0, ctx->stream>>>(B.db, X2c, 0.25, ctx->d_dt, B.dqb, nv);
  if (int r = vjp_core(ctx, 0, 1, OSTC_TERM_ALL, X1c, GT)) return r;
  k_axpby<<<gt, 256, 0, ctx->stream>>>(nt, 0.25, X2c, 1.0, X1c);
  k_axpby<<<g1, 256, 0, ctx->stream>>>(N, 1.0, GT, 1.0, X1T);
  // stage 1
  CK(cudaMemsetAsync(LT, 0, N * sizeof(double), ctx->stream));
  newton(0, 1, X1T, X1c, LT);
  k_adj_stage_seed<<<g, 128, 0, ctx->stream>>>(B.db, X1c, 1.0, ctx->d_dt, B.dqb, nv);
  if (int r = vjp_core(ctx, 0, 0, OSTC_TERM_ALL, Gc, GT)) return r;
  k_axpby<<<gt, 256, 0, ctx->stream>>>(nt, 0.75, X2c, 1.0 / 3.0, Lc);
  k_axpby<<<gt, 256, 0, ctx->stream>>>(nt, 1.0, X1c, 1.0, Lc);
  k_axpby<<<gt, 256, 0, ctx->stream>>>(nt, 1.0, Gc, 1.0, Lc);
  k_axpby<<<g1, 256, 0, ctx->stream>>>(N, 1.0, GT, 1.0, LT);
  CK(cudaGetLastError());
  return OSTC_OK;
}

// lam_cv += (dT / dcv)^T lam_T at slot 0, T the equation-of-state root of cv (the start of a
// trajectory set by ostc_set_state or ostc_set_conservative), then lam_T = 0
int adjoint_t_to_cv(ostc_ctx *ctx) {
  BlockRes &B = ctx->blk[0];
  const long long N = B.db.n, nt = (long long)ctx->nv * N;
  double *Lc = B.adj_work, *LT = Lc + 4 * nt;
  const int g = grid_for(ctx, N, 128);
  if (ctx->der.n_spec == kFixedNS)
    k_adj_t_to_cv<kFixedNS><<<g, 128, 0, ctx->stream>>>(B.db, state_of(B, 0), LT, Lc);
  else
    k_adj_t_to_cv<0><<<g, 128, 0, ctx->stream>>>(B.db, state_of(B, 0), LT, Lc);
  CK(cudaMemsetAsync(LT, 0, N * sizeof(double), ctx->stream));
  CK(cudaGetLastError());
  return OSTC_OK;
}

int enqueue_step_any(ostc_ctx *ctx) {
  if (ctx->mixture) return enqueue_step_mix(ctx);
  return ctx->precision == OSTC_PREC_MIXED ? enqueue_step<float>(ctx) : enqueue_step<double>(ctx);
}

// The device part of ostc_set_state: buffer A of block B takes the primitive state from device
// arrays bv[6][N] (and sv[n_spec][N]); ghost nodes start from the default initialisation (or zero)
// and are rewritten by the boundary faces and interfaces when the context next initialises.
void enqueue_set_state(ostc_ctx *ctx, BlockRes &B, const double *bv, const double *sv) {
  const bool ml = ctx->der.problem_type == 1 && B.ycoord;
  if (ml) {
    MlVals m{};
    for (int l = 0; l < 6; ++l) {
      m.upper[l] = ctx->ml.upper[l];
      m.lower[l] = ctx->ml.lower[l];
    }
    for (size_t l = 0; l < ctx->ml.y_upper.size() && l < 16; ++l) {
      m.y_upper[l] = ctx->ml.y_upper[l];
      m.y_lower[l] = ctx->ml.y_lower[l];
    }
    m.delta_omega = ctx->ml.delta_omega;
    k_fill_mixing_layer<<<grid_for(ctx, B.db.plane, 256), 256, 0, ctx->stream>>>(
        B.db.plane, B.ycoord, B.bv[0], ctx->mixture ? B.sv[0] : nullptr, ctx->mixture ? ctx->der.n_spec : 0, m);
  } else if (ctx->has_init) {
    FillVals fv{};
    for (int l = 0; l < 6; ++l) fv.val[l] = ctx->init_bv[l];
    k_fill_planes<<<grid_for(ctx, 6 * B.db.plane, 256), 256, 0, ctx->stream>>>(B.db.plane, B.bv[0], 6, fv);
  } else {
    cudaMemsetAsync(B.bv[0], 0, 6 * B.db.plane * sizeof(double), ctx->stream);
  }
  cudaMemsetAsync(B.cv[0], 0, (size_t)ctx->nv * B.db.plane * sizeof(double), ctx->stream);
  cudaMemsetAsync(B.mul[0], 0, B.db.plane * sizeof(double), ctx->stream);
  k_scatter<<<grid_for(ctx, 6 * B.db.n, 256), 256, 0, ctx->stream>>>(B.db, bv, B.bv[0], 6);
  if (ctx->mixture) {
    const int ns = ctx->der.n_spec;
    if (ml) {
      // filled with the profile above
    } else if (ctx->has_init && (int)ctx->init_sv.size() == ns && ns <= 16) {
      FillVals fv{};
      for (int l = 0; l < ns; ++l) fv.val[l] = ctx->init_sv[l];
      k_fill_planes<<<grid_for(ctx, ns * B.db.plane, 256), 256, 0, ctx->stream>>>(B.db.plane, B.sv[0], ns, fv);
    } else {
      cudaMemsetAsync(B.sv[0], 0, (size_t)ns * B.db.plane * sizeof(double), ctx->stream);
    }
    k_scatter<<<grid_for(ctx, ns * B.db.n, 256), 256, 0, ctx->stream>>>(B.db, sv, B.sv[0], ns);
    // the properties start from zero, as the reference's freshly allocated arrays do: its first
    // boundary faces (initialize_computation, Driver.cu:145-147) run before any properties sweep, and
    // a mixture far-field face reads gamma there (BoundCond.cuh:788)
    cudaMemsetAsync(B.gam[0], 0, B.db.plane * sizeof(double), ctx->stream);
    cudaMemsetAsync(B.acs[0], 0, B.db.plane * sizeof(double), ctx->stream);
    cudaMemsetAsync(B.cond[0], 0, B.db.plane * sizeof(double), ctx->stream);
    cudaMemsetAsync(B.rhod[0], 0, (size_t)ns * B.db.plane * sizeof(double), ctx->stream);
  }
}

int check_ready(ostc_ctx *ctx) {
  if (!ctx->state_set) {
    ctx->err = "no state: call ostc_set_state for every block first";
    return OSTC_ESTATE;
  }
  for (char c : ctx->block_set)
    if (!c) {
      ctx->err = "ostc_set_state was not called for every block";
      return OSTC_ESTATE;
    }
  if (bind_tables(ctx) != 0) {
    ctx->err = "upload of the species / reaction tables to constant memory failed";
    return OSTC_ECUDA;
  }
  if (!ctx->initialised) {
    if (int r = initialise(ctx)) return r;
  }
  const int pi = ctx->precision == OSTC_PREC_MIXED ? 1 : 0;
  if (ctx->der.inviscid_type == 1 && !ctx->tuned[pi]) {
    if (int r = pi ? autotune_yz<float>(ctx) : autotune_yz<double>(ctx)) return r;
    ctx->tuned[pi] = true;
  }
  return OSTC_OK;
}

// ---- steady driver (steady_simulation, SteadySim.cuh:15-140)

int steady_alloc(ostc_ctx *ctx, bool dual = false) {
  const bool fr = ctx->mixture && ctx->der.reaction == 1;
  const int ns = ctx->der.n_spec, csm = fr ? ctx->der.chem_src_method : 0;
  for (auto &B : ctx->blk) {
    const size_t N = (size_t)B.db.n;
    if (!B.dtl) CK(cudaMalloc(&B.dtl, N * sizeof(double)));
    if (!B.srad) CK(cudaMalloc(&B.srad, 3 * N * sizeof(double)));
    if (csm && !B.cj) CK(cudaMalloc(&B.cj, N * (size_t)(csm == 1 ? ns * ns : ns) * sizeof(double)));
    if ((ctx->der.implicit_method == 1 || dual) && !B.dq0) {
      CK(cudaMalloc(&B.dq0, N * ctx->nv * sizeof(double)));
      CK(cudaMalloc(&B.dqk, N * ctx->nv * sizeof(double)));
    }
    if (dual && !B.qn1) {
      CK(cudaMalloc(&B.qn1, (size_t)ctx->nv * B.db.plane * sizeof(double)));
      CK(cudaMalloc(&B.qstar, N * ctx->nv * sizeof(double)));
    }
  }
  return OSTC_OK;
}

template <int NS>
void launch_steady_chem(ostc_ctx *ctx, BlockRes &B, DevState st, int method) {
  k_mix_source_jac<NS><<<grid_for(ctx, B.db.n, 128), 128, 0, ctx->stream>>>(B.db, st, B.dq, method, B.cj);
}

template <int NS>
void launch_steady_implicit(ostc_ctx *ctx, BlockRes &B, DevState st, int csm, bool fr, bool dplur,
                            double diag_factor) {
  const DevBlock &b = B.db;
  const int g = grid_for(ctx, b.n, 128);
  if (dplur) {
    // DPLUR (DPLUR.cuh:282-322)
    DplurArgs a{B.dtl, B.srad, B.cj, B.dq, B.dq0, B.dqk, ctx->nv, fr ? csm + 1 : 0, diag_factor};
    k_dplur_dq0<NS><<<g, 128, 0, ctx->stream>>>(b, a);
    const size_t bytes = (size_t)ctx->nv * b.n * sizeof(double);
    cudaMemcpyAsync(B.dq0, B.dq, bytes, cudaMemcpyDeviceToDevice, ctx->stream);
    for (int it = 0; it < ctx->der.dplur_inner; ++it) {
      for (const DevFace &f : B.faces)
        if (f.type == kWall)
          k_wall_dq_zero<<<grid_for(ctx, (long long)b.mx * b.my * b.mz / 4 + 1, 128), 128, 0, ctx->stream>>>(
              b, f, B.dq, ctx->nv);
      k_dplur_inner<NS><<<g, 128, 0, ctx->stream>>>(b, st, a);
      cudaMemcpyAsync(B.dq, B.dqk, bytes, cudaMemcpyDeviceToDevice, ctx->stream);
    }
    k_dplur_back<<<g, 128, 0, ctx->stream>>>(b, B.dq, B.dtl, ctx->nv);
  } else if (fr && csm) {
    k_point_implicit<NS><<<g, 128, 0, ctx->stream>>>(b, B.dq, B.dtl, B.cj, csm);
  }
}

// One iteration of the steady driver over every block, in place on state slot 0: dq from zero, the
// chemical source first (with its Jacobian for chemSrcMethod 1 / 2), inviscid and viscous fluxes,
// local_time_step, implicit_treatment (ImplicitTreatmentHPP.cuh:7-54), update_cv_and_bv, the block's
// boundary faces; then the interfaces and (mixtures) the properties.  With dt_phys > 0 it is one
// pseudo-time iteration of dual time stepping (DualTimeStepping.cuh:126-165): the BDF2 terms join dq
// (compute_modified_rhs) and DPLUR runs with diag_factor 1.5 / dt_phys.
template <typename T>
int enqueue_steady_iteration(ostc_ctx *ctx, double dt_phys = 0.0) {
  const bool dual = dt_phys > 0.0;
  const bool fr = ctx->mixture && ctx->der.reaction == 1;
  const int csm = fr ? ctx->der.chem_src_method : 0;
  const bool fixed = ctx->der.n_spec == kFixedNS;
  for (size_t bi = 0; bi < ctx->blk.size(); ++bi) {
    BlockRes &B = ctx->blk[bi];
    const DevState st = state_of(B, 0);
    const DevBlock &b = B.db;
    {
      long tok = begin_t(ctx, "rhs");
      if (ctx->mixture) {
        if (csm) {
          if (fixed) launch_steady_chem<kFixedNS>(ctx, B, st, csm);
          else launch_steady_chem<0>(ctx, B, st, csm);
        } else {
          launch_mix_source(ctx, B, st, fr);
        }
        launch_mix_inviscid(ctx, B, st);
        if (ctx->der.viscous_order != 0) launch_mix_visc(ctx, B, st);
      } else {
        launch_flux<T>(ctx, B, st);
        StageArgs a{};
        a.in = st;
        a.qn = st;
        a.out = st;
        a.prandtl = ctx->der.prandtl;
        a.viscous = ctx->der.viscous_order != 0;
        a.update = 0;
        a.flags = ctx->d_flags;
        launch_visc<T>(ctx, B, a);
      }
      end_t(ctx, tok);
    }
    {
      long tok = begin_t(ctx, "local_dt");
      k_local_dt<<<grid_for(ctx, b.n, 256), 256, 0, ctx->stream>>>(b, st, ctx->der.cfl, ctx->der.prandtl, b.mz > 1,
                                                                   B.dtl, B.srad);
      end_t(ctx, tok);
    }
    if (dual)
      k_modified_rhs<<<grid_for(ctx, b.n, 128), 128, 0, ctx->stream>>>(b, st, B.qstar, B.dq, ctx->nv, dt_phys);
    {
      long tok = begin_t(ctx, "implicit");
      const bool dplur = dual || ctx->der.implicit_method == 1;
      const double df = dual ? 1.5 / dt_phys : 0.0;
      if (fixed) launch_steady_implicit<kFixedNS>(ctx, B, st, csm, fr, dplur, df);
      else launch_steady_implicit<0>(ctx, B, st, csm, fr, dplur, df);
      end_t(ctx, tok);
    }
    {
      long tok = begin_t(ctx, "update");
      if (ctx->mixture) {
        if (fixed)
          k_mix_update<kFixedNS><<<grid_for(ctx, b.n, 128), 128, 0, ctx->stream>>>(
              b, st, st, st, B.dq, ctx->d_dt, 0.0, 1.0, 1.0, ctx->nv, ctx->d_flags, B.dtl);
        else
          k_mix_update<0><<<grid_for(ctx, b.n, 128), 128, 0, ctx->stream>>>(b, st, st, st, B.dq, ctx->d_dt, 0.0, 1.0,
                                                                            1.0, ctx->nv, ctx->d_flags, B.dtl);
      } else {
        k_steady_update_air<<<grid_for(ctx, b.n, 256), 256, 0, ctx->stream>>>(b, st, B.dq, B.dtl, ctx->d_flags);
      }
      end_t(ctx, tok);
    }
    launch_bcs(ctx, (int)bi, st);
  }
  launch_interfaces(ctx, 0);
  if (ctx->mixture)
    for (auto &B : ctx->blk) {
      long tok = begin_t(ctx, "properties");
      launch_mix_props(ctx, B, state_of(B, 0));
      end_t(ctx, tok);
    }
  CK(cudaGetLastError());
  return OSTC_OK;
}

}  // namespace
