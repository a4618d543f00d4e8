// air_kernels.cuh -- sm_100a kernels of the calorically-perfect-air RHS + SSP-RK3 path, the boundary
// faces, block interfaces and set-up kernels shared with the mixture path.
//
// Per RK stage the device work is (reference order in brackets, RK.cuh:112-174):
//   k_cfl_dt           [local_time_step + min_of_arr x2 + D2H + update_dt_global] first stage only:
//                      spectral radius, warp-shuffle min, one 64-bit atomicMin into a device scalar
//   k_flux_x           [compute_convective_term_aweno_1D + CDSPart1D, x]: staged row tile, one face per thread
//   k_flux_march<1|2>  [same, y and z]: each thread marches one column, coalesced across i, with a
//                      per-thread ring of 2*ngg+1 nodes in shared memory (no halo re-reads)
//   k_visc_update      [viscous_flux_fv/gv/hv + update_cv_and_bv_rk + update_physical_properties]
//                      3-D tile, face fluxes staged in shared memory, RK combine and EOS fused
//   k_bc_face          [apply_farfield/outflow/symmetry/periodic, in the reference priority order]
// The three RK stages ping-pong over three state buffers (A -> B -> C -> A) so no stage overwrites
// data another block still reads; buffer A doubles as q^n (RK.cuh:99-102 needs no copy).
// Part of the ostc_b200.cu translation unit (included in order; not a standalone header).
#pragma once

namespace ostc {

// ------------------------------------------------------------------------------ time step

__global__ void k_dt_reset(unsigned long long *dtbits) { *dtbits = (unsigned long long)__double_as_longlong(1e6); }

// local_time_step<Air, Laminar> (TimeAdvanceFunc.cuh:28-83) fused with the global minimum of
// global_time_step (TimeAdvanceFunc.cu:39-64).  Positive doubles order like their bit patterns, so
// the minimum is one 64-bit atomicMin per block after a warp-shuffle reduction.
__global__ void __launch_bounds__(256) k_cfl_dt(DevBlock b, DevState s, double cfl, double prandtl, int dim3,
                                                unsigned long long *dtbits) {
  double local = 1e6;
  const long long P = b.plane;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < b.n; n += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(n % b.mx);
    const long long r = n / b.mx;
    const int j = (int)(r % b.my), k = (int)(r / b.my);
    const long long p = b.id(i, j, k);
    double m[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) m[q] = b.met[q * P + p];
    const double gx = sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
    const double ge = sqrt(m[3] * m[3] + m[4] * m[4] + m[5] * m[5]);
    const double gz = sqrt(m[6] * m[6] + m[7] * m[7] + m[8] * m[8]);
    const double u = s.bv[P + p], v = s.bv[2 * P + p], w = s.bv[3 * P + p];
    const double U = u * m[0] + v * m[1] + w * m[2];
    const double V = u * m[3] + v * m[4] + w * m[5];
    const double W = u * m[6] + v * m[7] + w * m[8];
    const double a = s.acs ? s.acs[p] : sqrt(kGamma * kRuD * s.bv[5 * P + p] / kMwD);
    const double s0 = fabs(U) + a * gx, s1 = fabs(V) + a * ge;
    const double s2 = dim3 ? fabs(W) + a * gz : 0.0;
    const double sinv = s0 + s1 + s2;
    const double c1 = fmax(s.gam ? s.gam[p] : kGamma, 4.0 / 3.0) / s.bv[p];
    const double c2 = s.mul[p] / prandtl;
    double sv = gx * gx + ge * ge;
    if (dim3) sv += gz * gz;
    sv *= c1 * c2;
    local = fmin(local, cfl / (sinv + sv));
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) local = fmin(local, __shfl_xor_sync(0xffffffffu, local, off));
  __shared__ double wmin[8];
  if ((threadIdx.x & 31) == 0) wmin[threadIdx.x >> 5] = local;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = wmin[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmin(m, wmin[w]);
    atomicMin(dtbits, (unsigned long long)__double_as_longlong(m));
  }
}

// ------------------------------------------------------------------------------ inviscid flux

// Resident blocks per SM the x sweep is compiled for (register budget 65536 / (128 * this)).
template <typename T> struct FluxXOcc { static constexpr int blocks = 3; };
template <> struct FluxXOcc<float> { static constexpr int blocks = 5; };

// x sweep.  A block of 128 threads stages 127 + 2*NG nodes of one (j,k) row in shared memory
// (coalesced along i), computes the 128 faces i0-1/2 .. i0+126+1/2 (one per thread) and finalises
// the 127 nodes between them: dq = -(fc(i+1/2) - fc(i-1/2)) + central correction.
template <int NG, int RS, typename T>
__global__ void __launch_bounds__(128, FluxXOcc<T>::blocks) k_flux_x(DevBlock b, DevState s, double *__restrict__ dq) {
  constexpr int L = 127;
  constexpr int NP = L + 2 * NG;
  __shared__ T sq[6][NP];
  __shared__ T sf[5][NP];
  __shared__ T sm[4][NP];
  __shared__ T sfc[5][128];
  const int t = threadIdx.x;
  const int i0 = blockIdx.x * L;
  const int j = blockIdx.y, k = blockIdx.z;
  const long long P = b.plane;
  const long long base = b.id(0, j, k);
  for (int n = t; n < NP; n += 128) {
    const int i = i0 - NG + n;
    if (i < b.mx + NG) {
      const long long p = base + i;
      T bb[5], kk[3];
#pragma unroll
      for (int l = 0; l < 5; ++l) {
        sq[l][n] = (T)s.cv[l * P + p];
        bb[l] = (T)s.bv[l * P + p];
      }
      sq[5][n] = bb[4];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        kk[c] = (T)b.met[c * P + p];
        sm[c][n] = kk[c];
      }
      const T jj = (T)b.jac[p];
      sm[3][n] = jj;
      T f[5];
      node_flux<T>(bb, (T)s.cv[4 * P + p], kk, jj, f);
#pragma unroll
      for (int l = 0; l < 5; ++l) sf[l][n] = f[l];
    }
  }
  __syncthreads();
  const int face = i0 - 1 + t;
  if (face < b.mx) {
    auto q = [&](int st, int v) -> T { return sq[v][t + st]; };
    const T mt0[3] = {sm[0][t + NG - 1], sm[1][t + NG - 1], sm[2][t + NG - 1]};
    const T mt1[3] = {sm[0][t + NG], sm[1][t + NG], sm[2][t + NG]};
    T fc[5];
    aweno_face_flux<NG, RS, T>(q, mt0, mt1, sm[3][t + NG - 1], sm[3][t + NG], fc);
#pragma unroll
    for (int l = 0; l < 5; ++l) sfc[l][t] = fc[l];
  }
  __syncthreads();
  const int i = i0 - 1 + t;
  if (t >= 1 && i < b.mx) {
    const long long qi = b.iq(i, j, k);
    const int c = t - 1 + NG;  // staged index of node i
    auto f = [&](int m, int l) -> T { return sf[l][c + m]; };
    const bool cds = i < b.mx - 2 * NG;
#pragma unroll
    for (int l = 0; l < 5; ++l) {
      double d = 0.0;
      d -= (double)(sfc[l][t] - sfc[l][t - 1]);
      if (cds) d += (double)cds_correction<NG, T>(f, l);
      dq[l * b.n + qi] = d;
    }
  }
}

// Asynchronous global -> shared copies (cp.async, Ampere and later, plain non-bulk form).
__device__ __forceinline__ void cp_async8(void *smem_dst, const void *gsrc) {
  const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Resident 64-thread blocks per SM the march kernel is compiled for.
template <typename T> struct MarchOcc { static constexpr int blocks = 4; };
template <> struct MarchOcc<float> { static constexpr int blocks = 6; };

// y (DIR = 1) or z (DIR = 2) sweep.  Thread (i, o) marches nodes c = s0..s1-1 of its column (o is
// k for y, j for z); warps are contiguous in i, so every load of a new node is coalesced.  A
// per-thread ring in shared memory keeps the last 2*NG+1 nodes' cv(5), p and node flux(5); the
// metric row and Jacobian of the face's two nodes travel in registers.
// FP32 instantiation: the raw FP64 data of the next node (cv 5, rho/u/v/w/p 5, metric row 3,
// Jacobian 1) and the metric row + Jacobian of the face's right node are prefetched with cp.async
// one iteration ahead (double-buffered) so their latency hides behind the face computation
// (measured 1.18x).  FP64 instantiation: plain loads - the prefetch buffers would cut it from 4 to 3
// resident blocks, which costs more than the latency it hides (measured 0.79x).  Segments of `seg`
// nodes split long columns across blocks.
template <int DIR, int NG, int RS, typename T>
__global__ void __launch_bounds__(64, MarchOcc<T>::blocks) k_flux_march(DevBlock b, DevState s,
                                                                         double *__restrict__ dq, int seg) {
  constexpr int W = 2 * NG + 1;
  constexpr int NV = 11;
  constexpr int NRAW = 14;
  constexpr bool PIPE = std::is_same_v<T, float>;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int nthr = blockDim.x * blockDim.y;
  T *ring = reinterpret_cast<T *>(smraw);
  // prefetch buffers (FP32 only): raw [2][NRAW][nthr], metric [2][4][nthr], 16-byte aligned
  double *raw = reinterpret_cast<double *>(
      (reinterpret_cast<size_t>(smraw) + (size_t)W * NV * nthr * sizeof(T) + 15) & ~(size_t)15);
  double *mraw = raw + 2 * NRAW * nthr;
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int o = blockIdx.y * blockDim.y + threadIdx.y;
  const int n_dir = DIR == 1 ? b.my : b.mz;
  const int n_o = DIR == 1 ? b.mz : b.my;
  if (i >= b.mx || o >= n_o) return;
  const int s0 = blockIdx.z * seg;
  if (s0 >= n_dir) return;
  const int s1 = min(s0 + seg, n_dir);
  const long long P = b.plane;
  const long long stride = DIR == 1 ? (long long)b.pitch : (long long)b.pitch * b.sy;
  const long long base = DIR == 1 ? b.id(i, 0, o) : b.id(i, o, 0);
  const double *__restrict__ mrow = b.met + (long long)DIR * 3 * P;
  auto R = [&](int slot, int v) -> T & { return ring[(slot * NV + v) * nthr + tid]; };
  auto Raw = [&](int sl, int v) -> double & { return raw[(sl * NRAW + v) * nthr + tid]; };
  auto Mraw = [&](int sl, int v) -> double & { return mraw[(sl * 4 + v) * nthr + tid]; };
  auto prefetch_node = [&](int n, int sl) {
    const long long p = b.chk(base + (long long)n * stride);
#pragma unroll
    for (int l = 0; l < 5; ++l) cp_async8(&Raw(sl, l), s.cv + l * P + p);
#pragma unroll
    for (int l = 0; l < 5; ++l) cp_async8(&Raw(sl, 5 + l), s.bv + l * P + p);
#pragma unroll
    for (int c = 0; c < 3; ++c) cp_async8(&Raw(sl, 10 + c), mrow + c * P + p);
    cp_async8(&Raw(sl, 13), b.jac + p);
  };
  auto prefetch_metric = [&](int n, int sl) {
    const long long p = b.chk(base + (long long)n * stride);
#pragma unroll
    for (int c = 0; c < 3; ++c) cp_async8(&Mraw(sl, c), mrow + c * P + p);
    cp_async8(&Mraw(sl, 3), b.jac + p);
  };
  // node n from its raw FP64 values into the ring
  auto commit_node = [&](int n, const double *cv, const double *bv, const double *km, double jac) {
    const int slot = (n + NG) % W;
    T bb[5], kk[3];
#pragma unroll
    for (int l = 0; l < 5; ++l) {
      R(slot, l) = (T)cv[l];
      bb[l] = (T)bv[l];
    }
    R(slot, 5) = bb[4];
#pragma unroll
    for (int c = 0; c < 3; ++c) kk[c] = (T)km[c];
    T f[5];
    node_flux<T>(bb, (T)cv[4], kk, (T)jac, f);
#pragma unroll
    for (int l = 0; l < 5; ++l) R(slot, 6 + l) = f[l];
  };
  auto load_direct = [&](int n) {
    const long long p = b.chk(base + (long long)n * stride);
    double cv[5], bv[5], km[3];
#pragma unroll
    for (int l = 0; l < 5; ++l) {
      cv[l] = s.cv[l * P + p];
      bv[l] = s.bv[l * P + p];
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) km[c] = mrow[c * P + p];
    commit_node(n, cv, bv, km, b.jac[p]);
  };
  for (int n = s0 - NG; n <= s0 + NG - 2; ++n) load_direct(n);
  if constexpr (PIPE) {
    // first stage: node s0-1+NG and the right-node metric of face s0-1/2 (node s0)
    prefetch_node(s0 - 1 + NG, 0);
    prefetch_metric(s0, 0);
    cp_async_commit();
  }
  T fprev[5] = {T(0), T(0), T(0), T(0), T(0)};
  long long pc = b.chk(base + (long long)(s0 - 1) * stride);
  T mt0[3] = {(T)mrow[pc], (T)mrow[P + pc], (T)mrow[2 * P + pc]};
  T j0 = (T)b.jac[pc];
  for (int c = s0 - 1; c < s1; ++c) {
    T mt1[3], j1;
    if constexpr (PIPE) {
      cp_async_wait_all();
      // both prefetch buffers alternate slots, so a copy never targets the slot just read
      const int ms = (c - s0 + 1) & 1;
      double cv[5], bv[5], km[3];
#pragma unroll
      for (int l = 0; l < 5; ++l) {
        cv[l] = Raw(ms, l);
        bv[l] = Raw(ms, 5 + l);
      }
#pragma unroll
      for (int q3 = 0; q3 < 3; ++q3) km[q3] = Raw(ms, 10 + q3);
      commit_node(c + NG, cv, bv, km, Raw(ms, 13));
#pragma unroll
      for (int q3 = 0; q3 < 3; ++q3) mt1[q3] = (T)Mraw(ms, q3);
      j1 = (T)Mraw(ms, 3);
      if (c + 1 < s1) {
        prefetch_node(c + 1 + NG, ms ^ 1);
        prefetch_metric(c + 2, ms ^ 1);
        cp_async_commit();
      }
    } else {
      load_direct(c + NG);
      const long long pn = b.chk(pc + stride);
#pragma unroll
      for (int q3 = 0; q3 < 3; ++q3) mt1[q3] = (T)mrow[q3 * P + pn];
      j1 = (T)b.jac[pn];
      pc = pn;
    }
    const int b0 = (c + 1) % W;
    auto q = [&](int st, int v) -> T {
      int sl = b0 + st;
      sl = sl >= W ? sl - W : sl;
      return R(sl, v);
    };
    T fc[5];
    aweno_face_flux<NG, RS, T>(q, mt0, mt1, j0, j1, fc);
    if (c >= s0) {
      const long long qi = DIR == 1 ? b.iq(i, c, o) : b.iq(i, o, c);
      const bool cds = c < n_dir - 2 * NG;
      const int bc = c % W;  // slot of node c - NG
      auto f = [&](int m, int l) -> T {
        int sl = bc + NG + m;
        sl = sl >= W ? sl - W : sl;
        return R(sl, 6 + l);
      };
#pragma unroll
      for (int l = 0; l < 5; ++l) {
        double d = dq[l * b.n + qi];
        d -= (double)(fc[l] - fprev[l]);
        if (cds) d += (double)cds_correction<NG, T>(f, l);
        dq[l * b.n + qi] = d;
      }
    }
#pragma unroll
    for (int l = 0; l < 5; ++l) fprev[l] = fc[l];
#pragma unroll
    for (int q3 = 0; q3 < 3; ++q3) mt0[q3] = mt1[q3];
    j0 = j1;
  }
  if constexpr (PIPE) cp_async_wait_all();
}

// y / z sweep as a tile: a block of TXL consecutive i (coalesced rows) x TD threads along the sweep
// direction stages TF - 1 + 2*NG nodes per lane in shared memory (cv, p, node flux, metric row,
// Jacobian), computes FPT faces per thread and finalises TF - 1 nodes per lane, as the x sweep does
// for rows.  Against the column march it trades (TF - 1 + 2 NG) / (TF - 1) node loads per node for
// independent faces with no serial dependence along the column; the autotuner picks between them.
// TF = TD * FPT faces per tile along the sweep (TF - 1 nodes finalised), FPT faces per thread.
template <int NG, int TXL, int TF, typename T>
constexpr size_t tile_smem_bytes() {
  return (size_t)(15 * (TF - 1 + 2 * NG) + 5 * TF) * TXL * sizeof(T);
}

// Resident blocks per SM a tile variant is compiled for: FP32 variants at 128 registers per thread,
// but three 256-thread blocks (80 registers, measured faster despite small spills); FP64 16-lane
// variants (half the shared memory of the 32-lane ones) at three 128-thread or two 256-thread
// blocks; the FP64 32-lane variant is shared-memory limited to two blocks anyway.
template <typename T, int TXL, int NT>
__host__ __device__ constexpr int tile_min_blocks() {
  return sizeof(T) == 4 ? (NT == 256 ? 3 : 65536 / (NT * 128)) : (TXL == 16 ? (NT == 128 ? 3 : 2) : 2);
}

template <int DIR, int NG, int RS, typename T, int TXL, int TD, int FPT>
__global__ void __launch_bounds__(TXL * TD, tile_min_blocks<T, TXL, TXL * TD>())
    k_flux_tile(DevBlock b, DevState s, double *__restrict__ dq) {
  constexpr int TF = TD * FPT;
  constexpr int L = TF - 1;
  constexpr int NP = L + 2 * NG;
  extern __shared__ __align__(16) unsigned char smraw[];
  T *sq = reinterpret_cast<T *>(smraw);  // [6][NP][TXL]  cv 0..4, p
  T *sf = sq + 6 * NP * TXL;             // [5][NP][TXL]  node flux
  T *smt = sf + 5 * NP * TXL;            // [4][NP][TXL]  metric row, Jacobian
  T *sfc = smt + 4 * NP * TXL;           // [5][TF][TXL]  face flux
  const int lane = threadIdx.x;
  const int i = blockIdx.x * TXL + lane;
  const int d0 = blockIdx.y * L;
  const int o = blockIdx.z;
  const int nd = DIR == 1 ? b.my : b.mz;
  const bool lane_ok = i < b.mx;
  const long long P = b.plane;
  const long long stride = DIR == 1 ? (long long)b.pitch : (long long)b.pitch * b.sy;
  const long long base = DIR == 1 ? b.id(i < b.mx ? i : 0, 0, o) : b.id(i < b.mx ? i : 0, o, 0);
  const double *__restrict__ mrow = b.met + (long long)DIR * 3 * P;
  auto at = [&](T *a, int v, int n) -> T & { return a[(v * NP + n) * TXL + lane]; };
  if (lane_ok) {
    for (int n = threadIdx.y; n < NP; n += TD) {
      const int d = d0 - NG + n;
      if (d >= nd + NG) continue;
      const long long p = b.chk(base + (long long)d * stride);
      T bb[5], kk[3];
#pragma unroll
      for (int l = 0; l < 5; ++l) {
        at(sq, l, n) = (T)s.cv[l * P + p];
        bb[l] = (T)s.bv[l * P + p];
      }
      at(sq, 5, n) = bb[4];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        kk[c] = (T)mrow[c * P + p];
        at(smt, c, n) = kk[c];
      }
      const T jj = (T)b.jac[p];
      at(smt, 3, n) = jj;
      T f[5];
      node_flux<T>(bb, (T)s.cv[4 * P + p], kk, jj, f);
#pragma unroll
      for (int l = 0; l < 5; ++l) at(sf, l, n) = f[l];
    }
  }
  __syncthreads();
  for (int r = 0; r < FPT; ++r) {
    const int t = threadIdx.y + r * TD;
    const int face = d0 - 1 + t;  // left node of this face
    if (lane_ok && face < nd) {
      auto q = [&](int st, int v) -> T { return at(sq, v, t + st); };
      const T mt0[3] = {at(smt, 0, t + NG - 1), at(smt, 1, t + NG - 1), at(smt, 2, t + NG - 1)};
      const T mt1[3] = {at(smt, 0, t + NG), at(smt, 1, t + NG), at(smt, 2, t + NG)};
      T fc[5];
      aweno_face_flux<NG, RS, T>(q, mt0, mt1, at(smt, 3, t + NG - 1), at(smt, 3, t + NG), fc);
#pragma unroll
      for (int l = 0; l < 5; ++l) sfc[(l * TF + t) * TXL + lane] = fc[l];
    }
  }
  __syncthreads();
  for (int r = 0; r < FPT; ++r) {
    const int t = threadIdx.y + r * TD;
    const int d = d0 - 1 + t;
    if (lane_ok && t >= 1 && d < nd) {
      const long long qi = DIR == 1 ? b.iq(i, d, o) : b.iq(i, o, d);
      const int c = t - 1 + NG;
      auto f = [&](int m, int l) -> T { return at(sf, l, c + m); };
      const bool cds = d < nd - 2 * NG;
#pragma unroll
      for (int l = 0; l < 5; ++l) {
        double v = dq[l * b.n + qi];
        v -= (double)(sfc[(l * TF + t) * TXL + lane] - sfc[(l * TF + t - 1) * TXL + lane]);
        if (cds) v += (double)cds_correction<NG, T>(f, l);
        dq[l * b.n + qi] = v;
      }
    }
  }
}

// Dynamic shared memory of one 64-thread march block: the ring, plus the prefetch buffers in FP32.
template <typename T>
constexpr size_t march_smem_bytes(int ng) {
  return (size_t)(2 * ng + 1) * 11 * 64 * sizeof(T) +
         (std::is_same_v<T, float> ? 16 + (2 * 14 + 8) * 64 * sizeof(double) : 0);
}

// ------------------------------------------------------- primitive reconstruction + Riemann

// Scheme constants of the primitive-reconstruction sweeps (inviscid_type 0 and 2).
struct PvArgs {
  int recon;       // 1 first order, 2 MUSCL, 3 NND2
  double efix;     // entropy_fix_factor (Roe)
  int is3d;
};

// Face flux between nodes n and n+1 of one sweep.  v(m, l): primitive l (rho,u,v,w,p) of node n+m,
// m = -1..2; mt0/mt1, j0/j1: metric row and Jacobian of nodes n, n+1; d0/d1: their entropy-fix
// thresholds (Roe only).
template <int RS, typename T, class V>
__device__ __forceinline__ void pv_face_flux(const V &v, int recon, const T *mt0, const T *mt1, T j0, T j1, T d0,
                                             T d1, T *fc) {
  T pl[6], pr[6];
  pv_reconstruct<T>(v, recon, pl, pr);
  if constexpr (RS == 2) roe<T>(pl, pr, mt0, mt1, j0, j1, d0, d1, fc);
  else if constexpr (RS == 1) lax_friedrichs<T>(pl, pr, mt0, mt1, j0, j1, fc);
  else if constexpr (RS == 4) hllc<T>(pl, pr, mt0, mt1, j0, j1, fc);
  else ausm_plus<T>(pl, pr, mt0, mt1, j0, j1, fc);
}

template <typename T>
__device__ __forceinline__ T node_efix(const DevBlock &b, const DevState &s, long long p, T factor, bool dim3) {
  const long long P = b.plane;
  T m[9], bb[5];
#pragma unroll
  for (int r = 0; r < 9; ++r) m[r] = (T)__ldg(b.met + r * P + p);
#pragma unroll
  for (int l = 0; l < 5; ++l) bb[l] = (T)__ldg(s.bv + l * P + p);
  return entropy_fix_delta<T>(m, bb, factor, dim3);
}

// x sweep of the primitive-reconstruction schemes (compute_convective_term_pv_1D and
// Roe_compute_inviscid_flux_1D, InviscidScheme.cu:52-161, 459-548).  Each warp owns 31 nodes of one
// (j,k) row: lane l computes the face between nodes i0-1+l and i0+l from its 4-node stencil (read
// through the read-only cache, neighbouring lanes share lines), and lanes 1..31 finalise node
// i0-1+l with the left face taken from lane l-1 by a shuffle.  dq is written (first sweep).
template <int RS, typename T>
__global__ void __launch_bounds__(128) k_flux_pv_x(DevBlock b, DevState s, PvArgs a, double *__restrict__ dq) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int i0 = (blockIdx.x * 4 + warp) * 31;
  const int j = blockIdx.y, k = blockIdx.z;
  const int n = i0 - 1 + lane;  // left node of this lane's face
  const long long P = b.plane;
  T fc[5] = {T(0), T(0), T(0), T(0), T(0)};
  if (n < b.mx) {
    const long long p = b.id(n, j, k);
    T st[4][5];
#pragma unroll
    for (int m = 0; m < 4; ++m)
#pragma unroll
      for (int l = 0; l < 5; ++l) st[m][l] = (T)__ldg(s.bv + l * P + p + m - 1);
    T mt0[3], mt1[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      mt0[c] = (T)__ldg(b.met + c * P + p);
      mt1[c] = (T)__ldg(b.met + c * P + p + 1);
    }
    const T j0 = (T)__ldg(b.jac + p), j1 = (T)__ldg(b.jac + p + 1);
    T d0 = T(0), d1 = T(0);
    if constexpr (RS == 2) {
      d0 = node_efix<T>(b, s, p, (T)a.efix, a.is3d);
      d1 = node_efix<T>(b, s, p + 1, (T)a.efix, a.is3d);
    }
    auto v = [&](int m, int l) -> T { return st[m + 1][l]; };
    pv_face_flux<RS, T>(v, a.recon, mt0, mt1, j0, j1, d0, d1, fc);
  }
  T left[5];
#pragma unroll
  for (int l = 0; l < 5; ++l) left[l] = __shfl_up_sync(0xffffffffu, fc[l], 1);
  const int i = n;  // node finalised by this lane: between faces (lane-1) and (lane)
  if (lane >= 1 && i < b.mx) {
    const long long q = b.iq(i, j, k);
#pragma unroll
    for (int l = 0; l < 5; ++l) dq[l * b.n + q] = -(double)(fc[l] - left[l]);
  }
}

// y / z sweep of the primitive-reconstruction schemes: each thread marches one column over a
// segment [d0, d1) of the sweep direction, keeping the 4-node stencil, the two face nodes' metric
// rows, Jacobians and entropy-fix thresholds in registers, so every node is read once per segment
// and every face flux is computed once.  Consecutive threads are consecutive i (coalesced).
template <int DIR, int RS, typename T>
__global__ void __launch_bounds__(128) k_flux_pv_march(DevBlock b, DevState s, PvArgs a, double *__restrict__ dq,
                                                        int seg) {
  const int i = blockIdx.x * 128 + threadIdx.x;
  const int o = blockIdx.y;  // k for the y sweep, j for the z sweep
  const int nd = DIR == 1 ? b.my : b.mz;
  const int d0 = blockIdx.z * seg;
  const int d1 = min(d0 + seg, nd);
  if (i >= b.mx || d0 >= nd) return;
  const long long P = b.plane;
  auto pid = [&](int d) -> long long { return DIR == 1 ? b.id(i, d, o) : b.id(i, o, d); };
  T st[4][5];
  auto load_node = [&](int slot, int d) {
    const long long p = pid(d);
#pragma unroll
    for (int l = 0; l < 5; ++l) st[slot][l] = (T)__ldg(s.bv + l * P + p);
  };
  T mt0[3], mt1[3], j0, j1, e0 = T(0), e1 = T(0);
  auto load_face_node = [&](T *mt, T &jj, T &ee, int d) {
    const long long p = pid(d);
#pragma unroll
    for (int c = 0; c < 3; ++c) mt[c] = (T)__ldg(b.met + (DIR * 3 + c) * P + p);
    jj = (T)__ldg(b.jac + p);
    if constexpr (RS == 2) ee = node_efix<T>(b, s, p, (T)a.efix, a.is3d);
  };
  // stencil of the face (d0-1, d0): nodes d0-2 .. d0+1
#pragma unroll
  for (int m = 0; m < 4; ++m) load_node(m, d0 - 2 + m);
  load_face_node(mt0, j0, e0, d0 - 1);
  load_face_node(mt1, j1, e1, d0);
  auto v = [&](int m, int l) -> T { return st[m + 1][l]; };
  T fl[5];
  pv_face_flux<RS, T>(v, a.recon, mt0, mt1, j0, j1, e0, e1, fl);
  for (int d = d0; d < d1; ++d) {
    // shift the stencil to nodes d-1 .. d+2 and the face nodes to d, d+1
#pragma unroll
    for (int m = 0; m < 3; ++m)
#pragma unroll
      for (int l = 0; l < 5; ++l) st[m][l] = st[m + 1][l];
    load_node(3, d + 2);
#pragma unroll
    for (int c = 0; c < 3; ++c) mt0[c] = mt1[c];
    j0 = j1;
    e0 = e1;
    load_face_node(mt1, j1, e1, d + 1);
    T fr[5];
    pv_face_flux<RS, T>(v, a.recon, mt0, mt1, j0, j1, e0, e1, fr);
    const long long q = DIR == 1 ? b.iq(i, d, o) : b.iq(i, o, d);
#pragma unroll
    for (int l = 0; l < 5; ++l) {
      dq[l * b.n + q] -= (double)(fr[l] - fl[l]);
      fl[l] = fr[l];
    }
  }
}

// ------------------------------------------------------------------------------ viscous + update

// compute_fv/gv/hv_2nd_order<Air, Laminar> (ViscousScheme.cuh:24-911): viscous flux through the face
// between a node and its neighbour in direction d; fv[0..3] = flux components 1..4 (component 0 is 0).
// V(q, di, dj, dk): q = u, v, w, T, mu of the node at offset (di,dj,dk) from the face's first node,
// u, v, w, T possibly as deviations from a reference whose velocity part is vref (0 in FP64);
// Mt(r, s): metric entry r (0..8, (row-1)*3+col-1) or Jacobian (r = 9) of face node s (0 or 1).
template <typename T, bool DIM3, class VA, class MA>
__device__ __forceinline__ void viscous_face(int d, const VA &V, const MA &Mt, T iprandtl, const T *vref, T *fv) {
  const int e[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  T m[9];
#pragma unroll
  for (int r = 0; r < 9; ++r) m[r] = T(0.5) * (Mt(r, 0) + Mt(r, 1));
  T gx[4], gy[4], gz[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    T g[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if (c == d) {
        g[c] = V(q, e[d][0], e[d][1], e[d][2]) - V(q, 0, 0, 0);
      } else if (c == 2 && !DIM3) {
        g[c] = T(0);
      } else {
        const int a0 = e[c][0], a1 = e[c][1], a2 = e[c][2];
        g[c] = T(0.25) * (V(q, a0, a1, a2) - V(q, -a0, -a1, -a2) + V(q, e[d][0] + a0, e[d][1] + a1, e[d][2] + a2) -
                          V(q, e[d][0] - a0, e[d][1] - a1, e[d][2] - a2));
      }
    }
    gx[q] = g[0] * m[0] + g[1] * m[3] + g[2] * m[6];
    gy[q] = g[0] * m[1] + g[1] * m[4] + g[2] * m[7];
    gz[q] = g[0] * m[2] + g[1] * m[5] + g[2] * m[8];
  }
  const T u_x = gx[0], u_y = gy[0], u_z = gz[0];
  const T v_x = gx[1], v_y = gy[1], v_z = gz[1];
  const T w_x = gx[2], w_y = gy[2], w_z = gz[2];
  const T mul = T(0.5) * (V(4, 0, 0, 0) + V(4, e[d][0], e[d][1], e[d][2]));
  const T third = T(1.0 / 3.0);
  const T txx = mul * (T(4) * u_x - T(2) * v_y - T(2) * w_z) * third;
  const T tyy = mul * (T(4) * v_y - T(2) * u_x - T(2) * w_z) * third;
  const T tzz = mul * (T(4) * w_z - T(2) * u_x - T(2) * v_y) * third;
  const T txy = mul * (u_y + v_x);
  const T txz = mul * (u_z + w_x);
  const T tyz = mul * (v_z + w_y);
  const T j0 = Mt(9, 0), j1 = Mt(9, 1);
  const T nx = T(0.5) * (Mt(d * 3 + 0, 0) * j0 + Mt(d * 3 + 0, 1) * j1);
  const T ny = T(0.5) * (Mt(d * 3 + 1, 0) * j0 + Mt(d * 3 + 1, 1) * j1);
  const T nz = T(0.5) * (Mt(d * 3 + 2, 0) * j0 + Mt(d * 3 + 2, 1) * j1);
  fv[0] = nx * txx + ny * txy + nz * txz;
  fv[1] = nx * txy + ny * tyy + nz * tyz;
  fv[2] = nx * txz + ny * tyz + nz * tzz;
  const T um = vref[0] + T(0.5) * (V(0, 0, 0, 0) + V(0, e[d][0], e[d][1], e[d][2]));
  const T vm = vref[1] + T(0.5) * (V(1, 0, 0, 0) + V(1, e[d][0], e[d][1], e[d][2]));
  const T wm = vref[2] + T(0.5) * (V(2, 0, 0, 0) + V(2, e[d][0], e[d][1], e[d][2]));
  const T cp = T(kGamma * kRuD / kMwD / (kGamma - 1));
  const T cond = mul * iprandtl * cp;
  fv[3] = um * fv[0] + vm * fv[1] + wm * fv[2] + cond * (nx * gx[3] + ny * gy[3] + nz * gz[3]);
}

struct StageArgs {
  DevState in, qn, out;
  double a, bcoef, c;
  const double *dt;
  double prandtl;
  int viscous, update;
  unsigned *flags;
};

// Viscous fluxes of all directions (viscous_flux_fv/gv/hv, SchemeSelector.cuh:69-154), then the
// SSP-RK3 combine, EOS and Sutherland viscosity of the new state (update_cv_and_bv_rk, RK.cuh:230-284;
// update_physical_properties<Air>, FieldOperation.cuh:107-140).
// A block owns a TX x TY column of nodes and marches k through [k0, k1).  Shared memory keeps a ring
// of three k planes (k-1, k, k+1) of u, v, w, T, mu and a ring of two (k, k+1) of the metric +
// Jacobian (no face of plane k reads the metric of plane k-1), each with a one-node halo in i and j,
// loaded once (coalesced along i).  Every face flux is computed once: x and y faces of plane k into
// shared memory, the z face k+1/2 in registers (carried to the next plane as k-1/2).
template <typename T, bool DIM3, int TX, int TY>
constexpr size_t visc_smem_bytes() {
  return sizeof(T) * ((DIM3 ? 3 * 5 + 2 * 10 : 15) * (TY + 2) * (TX + 2) + TY * (TX + 1) * 4 + (TY + 1) * TX * 4);
}

template <typename T, bool DIM3, int TX, int TY>
// FP64: two blocks per SM at up to 255 registers; three fit in shared memory, but their 168-register
// cap measured 5 % slower (40.1 against 38.05 ms per AWENO7 + HLLC step at 512 x 256 x 128)
__global__ void __launch_bounds__(TX *TY, sizeof(T) == 8 ? 2 : 4) k_visc_update(DevBlock b, StageArgs a, double *__restrict__ dq,
                                                                      int kseg) {
  constexpr int NP = DIM3 ? 3 : 1;  // planes in the u, v, w, T, mu ring
  constexpr int NM = DIM3 ? 2 : 1;  // planes in the metric ring
  constexpr int SX = TX + 2, SY = TY + 2;
  constexpr int NS = (NP * 5 + NM * 10) * SY * SX;  // staged values
  extern __shared__ __align__(16) unsigned char vsm_raw[];
  auto sv = reinterpret_cast<T(*)[5][SY][SX]>(vsm_raw);
  auto sm = reinterpret_cast<T(*)[10][SY][SX]>(vsm_raw + sizeof(T) * NP * 5 * SY * SX);
  auto fxs = reinterpret_cast<T(*)[TX + 1][4]>(vsm_raw + sizeof(T) * NS);
  auto fys = reinterpret_cast<T(*)[TX][4]>(vsm_raw + sizeof(T) * (NS + TY * (TX + 1) * 4));
  auto mslot = [](int kk) { return DIM3 ? (kk & 1) : 0; };  // kk >= -1
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int tid = ty * TX + tx;
  const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
  const int i = i0 + tx, j = j0 + ty;
  const int k0 = blockIdx.z * kseg;
  const int k1 = min(k0 + kseg, b.mz);
  const bool inside = i < b.mx && j < b.my;
  const long long P = b.plane;
  const T ipr = T(1.0 / a.prandtl);
  // FP32 staging: u, v, w, T are stored as deviations from one reference node of the block, formed
  // in FP64, so that neighbour differences keep their digits (T ~ 300 K varies by mK across a node);
  // the FP64 instantiation stores the values themselves (reference 0).
  double ref[4] = {0.0, 0.0, 0.0, 0.0};
  if constexpr (!std::is_same_v<T, double>) {
    const long long pr0 = b.id(min(i0, b.mx - 1), min(j0, b.my - 1), k0);
    ref[0] = a.in.bv[P + pr0];
    ref[1] = a.in.bv[2 * P + pr0];
    ref[2] = a.in.bv[3 * P + pr0];
    ref[3] = a.in.bv[5 * P + pr0];
  }
  const T tref[3] = {(T)ref[0], (T)ref[1], (T)ref[2]};
  auto load_plane = [&](int kk) {
    const int slot = DIM3 ? (kk + 3) % 3 : 0, ms = mslot(kk);
    for (int n = tid; n < SX * SY; n += TX * TY) {
      const int ii = i0 - 1 + n % SX, jj = j0 - 1 + n / SX;
      if (ii >= b.mx + b.g || jj >= b.my + b.g) continue;
      const long long p = b.id(ii, jj, kk);
      const int x = n % SX, y = n / SX;
      sv[slot][0][y][x] = (T)(a.in.bv[P + p] - ref[0]);
      sv[slot][1][y][x] = (T)(a.in.bv[2 * P + p] - ref[1]);
      sv[slot][2][y][x] = (T)(a.in.bv[3 * P + p] - ref[2]);
      sv[slot][3][y][x] = (T)(a.in.bv[5 * P + p] - ref[3]);
      sv[slot][4][y][x] = (T)a.in.mul[p];
      if constexpr (std::is_same_v<T, float>) {
#pragma unroll
        for (int r = 0; r < 10; ++r) sm[ms][r][y][x] = b.met32[r * P + p];
      } else {
#pragma unroll
        for (int r = 0; r < 9; ++r) sm[ms][r][y][x] = (T)b.met[r * P + p];
        sm[ms][9][y][x] = (T)b.jac[p];
      }
    }
  };
  // face whose first node is tile node (x, y) of plane kk, direction d
  auto face = [&](int d, int x, int y, int kk, T *fv) {
    const int s0 = DIM3 ? (kk + 3) % 3 : 0, m0 = mslot(kk);
    auto V = [&](int q, int di, int dj, int dk) -> T {
      const int sl = DIM3 ? (s0 + dk + 3) % 3 : 0;
      return sv[sl][q][y + dj][x + di];
    };
    auto Mt = [&](int r, int sd) -> T {
      if (sd == 0) return sm[m0][r][y][x];
      if (d == 0) return sm[m0][r][y][x + 1];
      if (d == 1) return sm[m0][r][y + 1][x];
      return sm[mslot(kk + 1)][r][y][x];
    };
    viscous_face<T, DIM3>(d, V, Mt, ipr, tref, fv);
  };
  T fz_prev[4] = {T(0), T(0), T(0), T(0)};
  if (a.viscous) {
    if (DIM3) {
      load_plane(k0 - 1);
      load_plane(k0);
      __syncthreads();
      if (inside) face(2, tx + 1, ty + 1, k0 - 1, fz_prev);
      __syncthreads();  // plane k0 + 1 takes the metric slot of plane k0 - 1
    }
  }
  const double dt = a.update ? *a.dt : 0.0;
  for (int k = k0; k < k1; ++k) {
    T fz_next[4] = {T(0), T(0), T(0), T(0)};
    // the node's update operands are loaded first, so that their latency overlaps the plane load
    // and the face fluxes (only this thread reads or writes node (i, j, k) of these arrays)
    double d[5], cq[5], cin[5], jk = 1.0;
    if (inside) {
      const long long qi = b.iq(i, j, k);
#pragma unroll
      for (int l = 0; l < 5; ++l) d[l] = dq[l * b.n + qi];
      if (a.update) {
        const long long p = b.id(i, j, k);
        jk = b.jac[p];
#pragma unroll
        for (int l = 0; l < 5; ++l) {
          cq[l] = a.qn.cv[l * P + p];
          cin[l] = a.in.cv[l * P + p];
        }
      }
    }
    if (a.viscous) {
      if (DIM3) load_plane(k + 1);
      else load_plane(k);
      __syncthreads();
      if (inside) {
        face(0, tx, ty + 1, k, fxs[ty][tx]);
        if (tx == TX - 1 || i == b.mx - 1) face(0, tx + 1, ty + 1, k, fxs[ty][tx + 1]);
        face(1, tx + 1, ty, k, fys[ty][tx]);
        if (ty == TY - 1 || j == b.my - 1) face(1, tx + 1, ty + 1, k, fys[ty + 1][tx]);
        if (DIM3) face(2, tx + 1, ty + 1, k, fz_next);
      }
      __syncthreads();
    }
    if (inside) {
      const long long qi = b.iq(i, j, k);
      if (a.viscous) {
#pragma unroll
        for (int l = 1; l < 5; ++l) d[l] += (double)(fxs[ty][tx + 1][l - 1] - fxs[ty][tx][l - 1]);
#pragma unroll
        for (int l = 1; l < 5; ++l) d[l] += (double)(fys[ty + 1][tx][l - 1] - fys[ty][tx][l - 1]);
        if (DIM3) {
#pragma unroll
          for (int l = 1; l < 5; ++l) d[l] += (double)(fz_next[l - 1] - fz_prev[l - 1]);
        }
      }
      if (!a.update) {
#pragma unroll
        for (int l = 0; l < 5; ++l) dq[l * b.n + qi] = d[l];
      } else {
        const long long p = b.id(i, j, k);
        const double dtj = dt / jk;
        double cv[5];
#pragma unroll
        for (int l = 0; l < 5; ++l) cv[l] = a.a * cq[l] + a.bcoef * cin[l] + a.c * dtj * d[l];
        if (!DIM3) cv[3] = 0;
        const double rho = cv[0];
        const double di = 1.0 / cv[0];
        const double u = cv[1] * di, v = cv[2] * di, w = cv[3] * di;
        const double V2 = u * u + v * v + w * w;
        const double pr = (kGamma - 1) * (cv[4] - 0.5 * rho * V2);
        const double tt = pr * kMwD * di / kRuD;
#pragma unroll
        for (int l = 0; l < 5; ++l) a.out.cv[l * P + p] = cv[l];
        a.out.bv[p] = rho;
        a.out.bv[P + p] = u;
        a.out.bv[2 * P + p] = v;
        a.out.bv[3 * P + p] = w;
        a.out.bv[4 * P + p] = pr;
        a.out.bv[5 * P + p] = tt;
        a.out.mul[p] = sutherland(tt);
        if (!(rho > 0.0) || !(pr > 0.0) || !(tt > 0.0)) atomicOr(a.flags, (unsigned)OSTC_FLAG_NONPOSITIVE);
        if (isnan(cv[0]) || isnan(cv[1]) || isnan(cv[2]) || isnan(cv[3]) || isnan(cv[4]))
          atomicOr(a.flags, (unsigned)OSTC_FLAG_NAN);
      }
    }
#pragma unroll
    for (int l = 0; l < 4; ++l) fz_prev[l] = fz_next[l];
  }
}

// ------------------------------------------------------------------------------ boundaries

__device__ __forceinline__ void copy_bv(const DevBlock &b, DevState s, long long dst, long long src) {
#pragma unroll
  for (int l = 0; l < 6; ++l) s.bv[l * b.plane + dst] = s.bv[l * b.plane + src];
  if (s.sv)
    for (int l = 0; l < c_mix.ns; ++l) s.sv[l * b.plane + dst] = s.sv[l * b.plane + src];
}

__device__ __forceinline__ void finish_node(const DevBlock &b, DevState s, long long p) {
  if (s.sv) {
    // mixtures: properties of the ghost come from the properties sweep over the padded block
    mix_cv_from_bv_node<0>(b, s, p);
    return;
  }
  cv_from_bv_node(b, s, p);
  s.mul[p] = sutherland(s.bv[5 * b.plane + p]);
}

// apply_farfield for mixtures (BoundCond.cuh:755-1022) at face node pb: the node's gamma, its mixture
// molecular weight from its mass fractions; supersonic inflow takes the far-field state and mass
// fractions, supersonic outflow copies the node; subsonic faces take the Riemann invariants, the
// velocity and composition of the far field (inflow, u_n < 0) or of the node, and a gamma iterated
// with cp of the face temperature until it changes by less than 1e-4.  As in the reference, the
// entropy of the inflow branch is chosen for u_n <= 0 but its velocity and composition for u_n < 0.
__device__ void farfield_mixture(const DevBlock &b, DevState s, const DevFace &f, long long pb, long long dstep,
                                 const double *gam_prev) {
  const long long P = b.plane;
  const int ns = c_mix.ns;
  double nx = b.met[(f.face * 3 + 0) * P + pb], ny = b.met[(f.face * 3 + 1) * P + pb],
         nz = b.met[(f.face * 3 + 2) * P + pb];
  const double gni = f.direction / sqrt(nx * nx + ny * ny + nz * nz);
  nx *= gni;
  ny *= gni;
  nz *= gni;
  const double ub = s.bv[P + pb], vb = s.bv[2 * P + pb], wb = s.bv[3 * P + pb];
  const double uf = nx * ub + ny * vb + nz * wb;
  double svb[kMS];
  for (int l = 0; l < ns; ++l) svb[l] = s.sv[l * P + pb];
  const double gb = gam_prev[pb];
  double mw_inv = 0;
  for (int l = 0; l < ns; ++l) mw_inv += svb[l] / c_mix.mw[l];
  double mw = 1.0 / mw_inv;
  const double pbv = s.bv[4 * P + pb], rb = s.bv[pb];
  const double ab = sqrt(gb * pbv / rb);
  const double mb = uf / ab;
  double vals[6];
  if (mb <= -1) {
    vals[0] = f.density; vals[1] = f.u; vals[2] = f.v; vals[3] = f.w; vals[4] = f.pressure; vals[5] = f.temperature;
    for (int l = 0; l < ns; ++l) svb[l] = f.y[l];
  } else if (mb >= 1) {
    for (int g = 1; g <= b.g; ++g) {
      const long long pg = b.chk(pb + g * dstep);
      for (int l = 0; l < 6; ++l) s.bv[l * P + pg] = s.bv[l * P + pb];
      for (int l = 0; l < ns; ++l) s.sv[l * P + pg] = s.sv[l * P + pb];
      mix_cv_from_bv_node<0>(b, s, pg);
    }
    return;
  } else {
    const double rpos = uf + 2 * ab / (gb - 1);
    const double uinf = f.u * nx + f.v * ny + f.w * nz;
    const double rneg = uinf - 2 * f.acoustic_speed / (f.gamma - 1);
    const double Un = 0.5 * (rpos + rneg);
    if (mb < 0) {
      vals[1] = f.u + (Un - uinf) * nx;
      vals[2] = f.v + (Un - uinf) * ny;
      vals[3] = f.w + (Un - uinf) * nz;
      for (int l = 0; l < ns; ++l) svb[l] = f.y[l];
      mw = f.mw;
    } else {
      vals[1] = ub + (Un - uf) * nx;
      vals[2] = vb + (Un - uf) * ny;
      vals[3] = wb + (Un - uf) * nz;
    }
    double gamma = kGamma, err = 1, rho = 0, pr = 0, t = 0;
    // the reference's loop has no bound; 100 iterations (far more than the few it takes) end it here
    for (int it = 0; err > 1e-4 && it < 100; ++it) {
      const double glast = gamma;
      const double cb = 0.25 * (gamma - 1) * (rpos - rneg);
      const double sb = mb <= 0 ? f.entropy : pbv / pow(rb, gamma);
      rho = pow(cb * cb / (gamma * sb), 1 / (gamma - 1));
      pr = rho * cb * cb / gamma;
      t = pr * mw / (rho * kRuD);
      double cp[kMS];
      mix_h_cp<0>(t, (double *)nullptr, cp);
      double cpt = 0;
      for (int l = 0; l < ns; ++l) cpt += cp[l] * svb[l];
      gamma = cpt / (cpt - kRuD / mw);
      err = fabs(1 - gamma / glast);
    }
    vals[0] = rho;
    vals[4] = pr;
    vals[5] = t;
  }
  for (int g = 0; g <= b.g; ++g) {
    const long long pg = b.chk(pb + g * dstep);
#pragma unroll
    for (int l = 0; l < 6; ++l) s.bv[l * P + pg] = vals[l];
    for (int l = 0; l < ns; ++l) s.sv[l * P + pg] = svb[l];
    mix_cv_from_bv_node<0>(b, s, pg);
  }
}

// One boundary face: apply_symmetry / apply_outflow / apply_periodic / apply_farfield<Air>
// (BoundCond.cuh:137-233, 755-1022, 1443-1486).  Threads cover the two tangential index ranges,
// which include ngg ghost layers on each side (Mesh.cpp:14-32).
__global__ void __launch_bounds__(128) k_bc_face(DevBlock b, DevState s, DevFace f, const double *gam_prev) {
  const int t0 = f.face == 0 ? 1 : 0;
  const int t1 = f.face == 2 ? 1 : 2;
  const int n0 = f.re[t0] - f.rs[t0] + 1, n1 = f.re[t1] - f.rs[t1] + 1;
  const long long nn = (long long)n0 * n1;
  const long long P = b.plane;
  const long long st[3] = {1, b.pitch, (long long)b.pitch * b.sy};
  int dir[3] = {0, 0, 0};
  dir[f.face] = f.direction;
  const long long dstep = dir[0] * st[0] + dir[1] * st[1] + dir[2] * st[2];
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < nn; n += (long long)gridDim.x * blockDim.x) {
    int idx[3];
    idx[f.face] = f.rs[f.face];
    idx[t0] = f.rs[t0] + (int)(n % n0);
    idx[t1] = f.rs[t1] + (int)(n / n0);
    const long long pb = b.id(idx[0], idx[1], idx[2]);
    if (f.type == kSymmetry) {
      const long long pin = b.chk(pb - dstep);
      double kx = b.met[(f.face * 3 + 0) * P + pb], ky = b.met[(f.face * 3 + 1) * P + pb],
             kz = b.met[(f.face * 3 + 2) * P + pb];
      const double km = sqrt(kx * kx + ky * ky + kz * kz);
      kx /= km;
      ky /= km;
      kz /= km;
      const double u1 = s.bv[P + pin], v1 = s.bv[2 * P + pin], w1 = s.bv[3 * P + pin];
      double uk = kx * u1 + ky * v1 + kz * w1;
      s.bv[P + pb] = u1 - kx * uk;
      s.bv[2 * P + pb] = v1 - ky * uk;
      s.bv[3 * P + pb] = w1 - kz * uk;
      s.bv[pb] = s.bv[pin];
      s.bv[4 * P + pb] = s.bv[4 * P + pin];
      s.bv[5 * P + pb] = s.bv[5 * P + pin];
      if (s.sv) {
        for (int l = 0; l < c_mix.ns; ++l) s.sv[l * P + pb] = s.sv[l * P + pin];
      } else {
        s.mul[pb] = sutherland(s.bv[5 * P + pb]);
      }
      for (int g = 1; g <= b.g; ++g) {
        const long long pg = b.chk(pb + g * dstep), pi = b.chk(pb - g * dstep);
        s.bv[pg] = s.bv[pi];
        const double u = s.bv[P + pi], v = s.bv[2 * P + pi], w = s.bv[3 * P + pi];
        uk = kx * u + ky * v + kz * w;
        s.bv[P + pg] = u - 2 * uk * kx;
        s.bv[2 * P + pg] = v - 2 * uk * ky;
        s.bv[3 * P + pg] = w - 2 * uk * kz;
        s.bv[4 * P + pg] = s.bv[4 * P + pi];
        s.bv[5 * P + pg] = s.bv[5 * P + pi];
        if (s.sv)
          for (int l = 0; l < c_mix.ns; ++l) s.sv[l * P + pg] = s.sv[l * P + pi];
        finish_node(b, s, pg);
      }
    } else if (f.type == kOutflow) {
      for (int g = 1; g <= b.g; ++g) {
        const long long pg = b.chk(pb + g * dstep);
        copy_bv(b, s, pg, pb);
        finish_node(b, s, pg);
      }
    } else if (f.type == kInflow) {
      // apply_inflow (BoundCond.cuh:235-613): the face node and every ghost layer take one state -
      // the constant one, or the mixing-layer profile at the face node's y - with the white noise of
      // fluctuation_type 1 added to its velocity
      double rho = f.density, u = f.u, v = f.v, w = f.w, pr = f.pressure, tt = f.temperature;
      const double *ys = f.y;
      double vel = f.velocity;
      bool noisy = f.fluct == 1;
      if (f.inflow_type == 2) {
        const double yc = f.ycoord[n];
        u = 0.5 * (f.u + f.lower[1]) + 0.5 * (f.u - f.lower[1]) * tanh(2 * yc / f.delta_omega);
        if (yc < 0) {
          rho = f.lower[0];
          v = f.lower[2];
          w = f.lower[3];
          pr = f.lower[4];
          tt = f.lower[5];
          ys = f.y_lower;
        }
        vel = sqrt(u * u + v * v + w * w);
        // the noise is confined to |y| < 4 delta_omega (BoundCond.cuh:406)
        noisy = noisy && yc < 4 * f.delta_omega && yc > -4 * f.delta_omega;
      }
      if (noisy) {
        // one generator state per node of the face plane, ghost-padded by ngg (BoundCond.cuh:406-420)
        const int a = f.face == 0 ? idx[1] : idx[0], c2 = f.face == 2 ? idx[1] : idx[2];
        curandState *st = f.rng + ((long long)(c2 + b.g) * f.rng_row + (a + b.g));
        curandState local = *st;
        u += curand_normal_double(&local) * f.fluct_rms * vel;
        if (f.inflow_type == 2) v += curand_normal_double(&local) * f.fluct_rms * vel;
        *st = local;
      }
      for (int g = 0; g <= b.g; ++g) {
        const long long pg = b.chk(pb + g * dstep);
        s.bv[pg] = rho;
        s.bv[P + pg] = u;
        s.bv[2 * P + pg] = v;
        s.bv[3 * P + pg] = w;
        s.bv[4 * P + pg] = pr;
        s.bv[5 * P + pg] = tt;
        if (s.sv)
          for (int l = 0; l < c_mix.ns; ++l) s.sv[l * P + pg] = ys[l];
        finish_node(b, s, pg);
      }
    } else if (f.type == kBackPressure || f.type == kSubsonicInflow) {
      // apply_back_pressure / apply_subsonic_inflow (BoundCond.cuh:1272-1441), air: outward unit
      // normal of the face, normal velocity and speed of sound of the face node (which keeps its
      // values); ghosts from the characteristic relations
      double nx = b.met[(f.face * 3 + 0) * P + pb], ny = b.met[(f.face * 3 + 1) * P + pb],
             nz = b.met[(f.face * 3 + 2) * P + pb];
      const double gni = f.direction / sqrt(nx * nx + ny * ny + nz * nz);
      nx *= gni;
      ny *= gni;
      nz *= gni;
      const double rb = s.bv[pb], ub = s.bv[P + pb], vb = s.bv[2 * P + pb], wb = s.bv[3 * P + pb];
      const double pbv = s.bv[4 * P + pb];
      const double u_face = nx * ub + ny * vb + nz * wb;
      const double ab = sqrt(kGamma * pbv / rb);
      if (f.type == kBackPressure) {
        double rho_b = rb, u_b = ub, v_b = vb, w_b = wb, p_b = pbv;
        const bool sub = fabs(u_face / ab) < 1;
        if (sub) {
          p_b = f.pressure;
          const long long p1 = b.chk(pb - dstep);
          const double d1 = s.bv[p1], u1 = s.bv[P + p1], v1 = s.bv[2 * P + p1], w1 = s.bv[3 * P + p1],
                       pr1 = s.bv[4 * P + p1];
          const double c1 = sqrt(kGamma * pr1 / d1);
          rho_b = d1 + (p_b - pr1) / (c1 * c1);
          u_b = u1 + nx * (pr1 - p_b) / (d1 * c1);
          v_b = v1 + ny * (pr1 - p_b) / (d1 * c1);
          w_b = w1 + nz * (pr1 - p_b) / (d1 * c1);
        }
        for (int g = 1; g <= b.g; ++g) {
          const long long pg = b.chk(pb + g * dstep), pi = b.chk(pb - g * dstep);
          double r, u, v, w, pr;
          if (sub) {
            pr = 2 * p_b - s.bv[4 * P + pi];
            r = 2 * rho_b - s.bv[pi];
            u = 2 * u_b - s.bv[P + pi];
            v = 2 * v_b - s.bv[2 * P + pi];
            w = 2 * w_b - s.bv[3 * P + pi];
          } else {
            r = rho_b;
            u = u_b;
            v = v_b;
            w = w_b;
            pr = p_b;
          }
          s.bv[pg] = r;
          s.bv[P + pg] = u;
          s.bv[2 * P + pg] = v;
          s.bv[3 * P + pg] = w;
          s.bv[4 * P + pg] = pr;
          s.bv[5 * P + pg] = pr / (r * kRuD / kMwD);
          finish_node(b, s, pg);
        }
      } else {
        // negative Riemann invariant and total enthalpy of the face node, then the speed of sound
        // from the quadratic that keeps both with the inflow's total state
        const double riemann_neg = fabs(u_face) - 2 * ab / (kGamma - 1);
        const double hti = pbv / rb * kGamma / (kGamma - 1) + 0.5 * (ub * ub + vb * vb + wb * wb);
        const double qa = 1 + 2.0 / (kGamma - 1);
        const double qb = 2 * riemann_neg;
        const double qc = (kGamma - 1) * (0.5 * riemann_neg * riemann_neg - hti);
        const double delta = qb * qb - 4 * qa * qc;
        double a_new = ab;
        if (delta >= 0) {
          const double a_plus = (-qb + sqrt(delta)) / (2 * qa);
          const double a_minus = (-qb - sqrt(delta)) / (2 * qa);
          a_new = a_plus > a_minus ? a_plus : a_minus;
        }
        const double u_new = riemann_neg + 2 * a_new / (kGamma - 1);
        const double mach = u_new / a_new;
        const double pr = f.pressure * pow(1 + 0.5 * (kGamma - 1) * mach * mach, -kGamma / (kGamma - 1));
        const double tt = f.temperature * pow(pr / f.pressure, (kGamma - 1) / kGamma);
        const double r = pr * kMwD / (tt * kRuD);
        for (int g = 1; g <= b.g; ++g) {
          const long long pg = b.chk(pb + g * dstep);
          s.bv[pg] = r;
          s.bv[P + pg] = u_new * f.u;
          s.bv[2 * P + pg] = u_new * f.v;
          s.bv[3 * P + pg] = u_new * f.w;
          s.bv[4 * P + pg] = pr;
          s.bv[5 * P + pg] = tt;
          finish_node(b, s, pg);
        }
      }
    } else if (f.type == kWall) {
      // apply_wall (BoundCond.cuh:1024-1270), no-slip, isothermal or adiabatic: the wall node takes
      // the first interior node's pressure (and mass fractions) at the wall temperature; ghost g
      // mirrors interior node g with reversed velocity and, isothermal, T_g = 2 T_w - T_in (T_w
      // where that falls to 0.1 T_w or below)
      const long long pin = b.chk(pb - dstep);
      const double tw = f.wall_adiabatic ? s.bv[5 * P + pin] : f.temperature;
      const double pw = s.bv[4 * P + pin];
      double mw = kMwD;
      if (s.sv) {
        double imw = 0;
        for (int l = 0; l < c_mix.ns; ++l) {
          s.sv[l * P + pb] = s.sv[l * P + pin];
          imw += s.sv[l * P + pb] / c_mix.mw[l];
        }
        mw = 1 / imw;
      }
      s.bv[pb] = pw * mw / (tw * kRuD);
      s.bv[P + pb] = 0;
      s.bv[2 * P + pb] = 0;
      s.bv[3 * P + pb] = 0;
      s.bv[4 * P + pb] = pw;
      s.bv[5 * P + pb] = tw;
      finish_node(b, s, pb);
      for (int g = 1; g <= b.g; ++g) {
        const long long pi = b.chk(pb - g * dstep), pg = b.chk(pb + g * dstep);
        const double p_i = s.bv[4 * P + pi], t_i = s.bv[5 * P + pi];
        double t_g = t_i;
        if (!f.wall_adiabatic) {
          t_g = 2 * tw - t_i;
          if (t_g <= 0.1 * tw) t_g = tw;
        }
        if (s.sv) {
          double imw = 0;
          for (int l = 0; l < c_mix.ns; ++l) {
            s.sv[l * P + pg] = s.sv[l * P + pi];
            imw += s.sv[l * P + pg] / c_mix.mw[l];
          }
          mw = 1 / imw;
        }
        s.bv[pg] = p_i * mw / (t_g * kRuD);
        s.bv[P + pg] = -s.bv[P + pi];
        s.bv[2 * P + pg] = -s.bv[2 * P + pi];
        s.bv[3 * P + pg] = -s.bv[3 * P + pi];
        s.bv[4 * P + pg] = p_i;
        s.bv[5 * P + pg] = t_g;
        finish_node(b, s, pg);
      }
    } else if (f.type == kPeriodic) {
      const int ext[3] = {b.mx, b.my, b.mz};
      int other[3] = {idx[0], idx[1], idx[2]};
      other[f.face] = f.direction < 0 ? ext[f.face] - 1 : 0;
      const long long po = b.id(other[0], other[1], other[2]);
      for (int g = 1; g <= b.g; ++g) {
        const long long pg = b.chk(pb + g * dstep), ps = b.chk(po + g * dstep);
        copy_bv(b, s, pg, ps);
        finish_node(b, s, pg);
      }
    } else if (f.type == kFarfield && s.sv) {
      farfield_mixture(b, s, f, pb, dstep, gam_prev);
    } else if (f.type == kFarfield) {
      double nx = b.met[(f.face * 3 + 0) * P + pb], ny = b.met[(f.face * 3 + 1) * P + pb],
             nz = b.met[(f.face * 3 + 2) * P + pb];
      const double gni = f.direction / sqrt(nx * nx + ny * ny + nz * nz);
      nx *= gni;
      ny *= gni;
      nz *= gni;
      const double ub = s.bv[P + pb], vb = s.bv[2 * P + pb], wb = s.bv[3 * P + pb];
      const double uf = nx * ub + ny * vb + nz * wb;
      const double pbv = s.bv[4 * P + pb], rb = s.bv[pb];
      const double ab = sqrt(kGamma * pbv / rb);
      const double mb = uf / ab;
      double vals[6];
      if (mb <= -1) {
        vals[0] = f.density; vals[1] = f.u; vals[2] = f.v; vals[3] = f.w; vals[4] = f.pressure; vals[5] = f.temperature;
      } else if (mb >= 1) {
        for (int g = 1; g <= b.g; ++g) {
          const long long pg = b.chk(pb + g * dstep);
          copy_bv(b, s, pg, pb);
          finish_node(b, s, pg);
        }
        continue;
      } else {
        const double rpos = uf + 2 * ab / (kGamma - 1);
        const double uinf = f.u * nx + f.v * ny + f.w * nz;
        const double rneg = uinf - 2 * f.acoustic_speed / (f.gamma - 1);
        const double Un = 0.5 * (rpos + rneg);
        const double cb = 0.25 * (kGamma - 1) * (rpos - rneg);
        double sb;
        if (mb <= 0) {
          sb = f.entropy;
          vals[1] = f.u + (Un - uinf) * nx;
          vals[2] = f.v + (Un - uinf) * ny;
          vals[3] = f.w + (Un - uinf) * nz;
        } else {
          sb = pbv / pow(rb, kGamma);
          vals[1] = ub + (Un - uf) * nx;
          vals[2] = vb + (Un - uf) * ny;
          vals[3] = wb + (Un - uf) * nz;
        }
        vals[0] = pow(cb * cb / (kGamma * sb), 1 / (kGamma - 1));
        vals[4] = vals[0] * cb * cb / kGamma;
        vals[5] = vals[4] * kMwD / (vals[0] * kRuD);
      }
#pragma unroll
      for (int l = 0; l < 6; ++l) s.bv[l * P + pb] = vals[l];
      finish_node(b, s, pb);
      for (int g = 1; g <= b.g; ++g) {
        const long long pg = b.chk(pb + g * dstep);
#pragma unroll
        for (int l = 0; l < 6; ++l) s.bv[l * P + pg] = vals[l];
        finish_node(b, s, pg);
      }
    }
  }
}

// inner_communication (DataCommunication.cuh:60-105): on the coincident face layer both blocks take
// the average of their values; the ngg layers beyond it take the neighbour's interior values; every
// written node gets its conservative variables (and, for air, its viscosity) again.
__global__ void __launch_bounds__(128) k_inner_face(DevBlock b, DevState s, DevBlock tb, DevState ts, DevInner f) {
  const long long tot = (long long)f.n_point[0] * f.n_point[1] * f.n_point[2];
  const long long P = b.plane, TP = tb.plane;
  const int ns = s.sv ? c_mix.ns : 0;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < tot; n += (long long)gridDim.x * blockDim.x) {
    const int n0 = (int)(n % f.n_point[0]);
    const long long r = n / f.n_point[0];
    const int n1 = (int)(r % f.n_point[1]), n2 = (int)(r / f.n_point[1]);
    const int d_idx[3] = {f.loop_dir[0] * n0, f.loop_dir[1] * n1, f.loop_dir[2] * n2};
    const int idx[3] = {f.rs[0] + d_idx[0], f.rs[1] + d_idx[1], f.rs[2] + d_idx[2]};
    int it[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) it[q] = f.ts[q] + f.target_loop_dir[q] * d_idx[f.src_tar[q]];
    const long long p = b.id(idx[0], idx[1], idx[2]);
    const long long pt = tb.id(it[0], it[1], it[2]);
    if (idx[f.face] == f.face_index) {
#pragma unroll
      for (int l = 0; l < 6; ++l) {
        const double ave = 0.5 * (ts.bv[l * TP + pt] + s.bv[l * P + p]);
        s.bv[l * P + p] = ave;
        ts.bv[l * TP + pt] = ave;
      }
      for (int l = 0; l < ns; ++l) {
        const double ave = 0.5 * (ts.sv[l * TP + pt] + s.sv[l * P + p]);
        s.sv[l * P + p] = ave;
        ts.sv[l * TP + pt] = ave;
      }
    } else {
#pragma unroll
      for (int l = 0; l < 6; ++l) s.bv[l * P + p] = ts.bv[l * TP + pt];
      for (int l = 0; l < ns; ++l) s.sv[l * P + p] = ts.sv[l * TP + pt];
    }
    finish_node(b, s, p);
  }
}

// The reference updates one state in place, so when a stage's boundary faces run, the ghost layers an
// interface fills still hold the previous stage's exchanged values, and faces that reach into them
// (tangential ranges include the ghost layers) read those.  Stages here write a fresh buffer: carry
// the interface ghost layers (not the coincident face, which the update rewrote) from the stage input.
__global__ void __launch_bounds__(128) k_inner_carry(DevBlock b, DevState in, DevState out, DevInner f) {
  const long long tot = (long long)f.n_point[0] * f.n_point[1] * f.n_point[2];
  const long long P = b.plane;
  const int ns = out.sv ? c_mix.ns : 0;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < tot; n += (long long)gridDim.x * blockDim.x) {
    const int n0 = (int)(n % f.n_point[0]);
    const long long r = n / f.n_point[0];
    const int n1 = (int)(r % f.n_point[1]), n2 = (int)(r / f.n_point[1]);
    const int idx[3] = {f.rs[0] + f.loop_dir[0] * n0, f.rs[1] + f.loop_dir[1] * n1, f.rs[2] + f.loop_dir[2] * n2};
    if (idx[f.face] == f.face_index) continue;
    const long long p = b.id(idx[0], idx[1], idx[2]);
#pragma unroll
    for (int l = 0; l < 6; ++l) out.bv[l * P + p] = in.bv[l * P + p];
    for (int l = 0; l < ns; ++l) out.sv[l * P + p] = in.sv[l * P + p];
  }
}

// ------------------------------------------------------------------------------ set-up kernels

// The two streams of a mixing-layer problem, for the initial profile.
struct MlVals {
  double upper[6], lower[6], y_upper[16], y_lower[16], delta_omega;
};

// initialize_mixing_layer_with_info (Initialize.cu:259-326), laminar: every padded node takes the upper
// or the lower stream by the sign of its y, with u blended by tanh(2 y / delta_omega).
__global__ void k_fill_mixing_layer(long long plane, const double *__restrict__ ycoord, double *__restrict__ bv,
                                    double *__restrict__ sv, int ns, MlVals m) {
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < plane; p += (long long)gridDim.x * blockDim.x) {
    const double y = ycoord[p];
    const double *st = y >= 0 ? m.upper : m.lower, *ys = y >= 0 ? m.y_upper : m.y_lower;
    bv[plane + p] = 0.5 * (m.upper[1] + m.lower[1]) + 0.5 * (m.upper[1] - m.lower[1]) * tanh(2 * y / m.delta_omega);
    bv[p] = st[0];
    bv[2 * plane + p] = st[2];
    bv[3 * plane + p] = st[3];
    bv[4 * plane + p] = st[4];
    bv[5 * plane + p] = st[5];
    for (int l = 0; l < ns; ++l) sv[l * plane + p] = ys[l];
  }
}

// initialize_rng (BoundCond.cu:1384-1391): generator state i seeded with seed + i, subsequence i
__global__ void k_rng_init(curandState *st, long long n, unsigned long long seed) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    curand_init(seed + (unsigned long long)i, (unsigned long long)i, 0, &st[i]);
}

// Interior primitive state from the conservative variables already in s.cv (update_cv_and_bv_rk's
// closing part, RK.cuh:250-284): mixtures solve T by the Newton iteration from the node's current T
// (compute_temperature_and_pressure, FieldOperation.cu:3-40); air closes p, T, mu directly.
template <int NS>
__global__ void __launch_bounds__(128) k_state_from_cv(DevBlock b, DevState s, int mixture, unsigned *flags) {
  const long long P = b.plane;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < b.n; n += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(n % b.mx);
    const long long r = n / b.mx;
    const int j = (int)(r % b.my), k = (int)(r / b.my);
    const long long p = b.id(i, j, k);
    const double rho = s.cv[p], di = 1.0 / rho;
    const double u = s.cv[P + p] * di, v = s.cv[2 * P + p] * di, w = s.cv[3 * P + p] * di;
    double pr, t;
    if (mixture) {
      const int ns = OSTC_NS;
      double y[Spec<NS>::A];
      for (int l = 0; l < ns; ++l) {
        y[l] = s.cv[(5 + l) * P + p] * di;
        s.sv[l * P + p] = y[l];
      }
      const double e = s.cv[4 * P + p] * di - 0.5 * (u * u + v * v + w * w);
      t = mix_temperature<NS>(rho, e, s.bv[5 * P + p], y, pr);
    } else {
      pr = (kGamma - 1) * (s.cv[4 * P + p] - 0.5 * rho * (u * u + v * v + w * w));
      t = pr * kMwD * di / kRuD;
      s.mul[p] = sutherland(t);
    }
    s.bv[p] = rho;
    s.bv[P + p] = u;
    s.bv[2 * P + p] = v;
    s.bv[3 * P + p] = w;
    s.bv[4 * P + p] = pr;
    s.bv[5 * P + p] = t;
    if (!(rho > 0) || !(pr > 0) || !(t > 0)) atomicOr(flags, (rho != rho || pr != pr || t != t) ? 2u : 1u);
  }
}

// every padded node of planes dst[0..nv) set to val[l]
__global__ void k_fill_planes(long long plane, double *__restrict__ dst, int nv, FillVals v) {
  const long long tot = plane * nv;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < tot; n += (long long)gridDim.x * blockDim.x)
    dst[n] = v.val[n / plane];
}

// interior [nv][N] (i fastest) <-> padded planes
__global__ void k_scatter(DevBlock b, const double *__restrict__ src, double *__restrict__ dst, int nv) {
  const long long tot = b.n * nv;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < tot; n += (long long)gridDim.x * blockDim.x) {
    const int l = (int)(n / b.n);
    const long long r = n - (long long)l * b.n;
    const int i = (int)(r % b.mx);
    const long long r2 = r / b.mx;
    const int j = (int)(r2 % b.my), k = (int)(r2 / b.my);
    dst[l * b.plane + b.id(i, j, k)] = src[n];
  }
}

__global__ void k_gather(DevBlock b, const double *__restrict__ src, double *__restrict__ dst, int nv) {
  const long long tot = b.n * nv;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < tot; n += (long long)gridDim.x * blockDim.x) {
    const int l = (int)(n / b.n);
    const long long r = n - (long long)l * b.n;
    const int i = (int)(r % b.mx);
    const long long r2 = r / b.mx;
    const int j = (int)(r2 % b.my), k = (int)(r2 / b.my);
    dst[n] = src[l * b.plane + b.id(i, j, k)];
  }
}

// cv <- bv and mu <- Sutherland(T) over the whole padded block (update_physical_properties and
// compute_cv_from_bv over ghosts, Driver.cu:186-191, RK.cuh:37-45)
__global__ void k_init_fields(DevBlock b, DevState s) {
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < b.plane; p += (long long)gridDim.x * blockDim.x) {
    finish_node(b, s, p);
  }
}

// residual snapshot and squared differences (store_last_step, compute_square_of_dbv,
// TimeAdvanceFunc.cu:6-37) reduced with warp shuffles into 4 sums.
__global__ void k_store_last(DevBlock b, DevState s, double *last) {
  const long long P = b.plane;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < b.n; n += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(n % b.mx);
    const long long r = n / b.mx;
    const int j = (int)(r % b.my), k = (int)(r / b.my);
    const long long p = b.id(i, j, k);
    const double u = s.bv[P + p], v = s.bv[2 * P + p], w = s.bv[3 * P + p];
    last[n] = s.bv[p];
    last[b.n + n] = sqrt(u * u + v * v + w * w);
    last[2 * b.n + n] = s.bv[4 * P + p];
    last[3 * b.n + n] = s.bv[5 * P + p];
  }
}

__global__ void __launch_bounds__(256) k_residual(DevBlock b, DevState s, const double *last, double *sums) {
  const long long P = b.plane;
  double acc[4] = {0, 0, 0, 0};
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < b.n; n += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(n % b.mx);
    const long long r = n / b.mx;
    const int j = (int)(r % b.my), k = (int)(r / b.my);
    const long long p = b.id(i, j, k);
    const double u = s.bv[P + p], v = s.bv[2 * P + p], w = s.bv[3 * P + p];
    const double d0 = s.bv[p] - last[n];
    const double d1 = sqrt(u * u + v * v + w * w) - last[b.n + n];
    const double d2 = s.bv[4 * P + p] - last[2 * b.n + n];
    const double d3 = s.bv[5 * P + p] - last[3 * b.n + n];
    acc[0] += d0 * d0;
    acc[1] += d1 * d1;
    acc[2] += d2 * d2;
    acc[3] += d3 * d3;
  }
  __shared__ double red[8][4];
#pragma unroll
  for (int q = 0; q < 4; ++q)
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], off);
  if ((threadIdx.x & 31) == 0)
    for (int q = 0; q < 4; ++q) red[threadIdx.x >> 5][q] = acc[q];
  __syncthreads();
  if (threadIdx.x < 4) {
    double t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w][threadIdx.x];
    atomicAdd(&sums[threadIdx.x], t);
  }
}

__global__ void k_step_end(double *t, const double *dt, long long *step) {
  *t += *dt;
  *step += 1;
}

__global__ void k_dt_decode(const unsigned long long *bits, double *dt) { *dt = __longlong_as_double((long long)*bits); }

// ------------------------------------------------------------------------------ digital-filter inflow

// apply_inflow_df (BoundCond.cuh:614-754): the i = 0 plane and its ngg ghost layers, over the face plane
// padded by ngg, take the upper (y > 0) or lower stream with u from the tanh profile plus the filtered
// fluctuation times DeltaU, v and w the fluctuations, and T / rho moved by the strong Reynolds analogy
// (t' = -u' u / cp, scaled by 0.25; rho' = -t' rho / T), p from the equation of state.
__global__ void k_df_apply(DevBlock b, DevState s, DevFace f, DevDf d, double mw_up, double mw_lo) {
  const long long np = (long long)d.py * d.pz;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < np; t += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(t % d.py) - d.g, k = (int)(t / d.py) - d.g;
    const double y = d.yface[t];
    double u = 0.5 * (f.u + f.lower[1]) + 0.5 * (f.u - f.lower[1]) * tanh(2 * y / f.delta_omega);
    const double uf = d.fluc[df_p(d, j, k, 0)] * d.delta_u;
    const double vf = d.fluc[df_p(d, j, k, 1)] * d.delta_u;
    const double wf = d.fluc[df_p(d, j, k, 2)] * d.delta_u;
    const bool up = y > 0;
    const double mw = up ? mw_up : mw_lo;
    double T = up ? f.temperature : f.lower[5];
    double rho = up ? f.density : f.lower[0];
    const double *ys = up ? f.y : f.y_lower;
    double cp = 0;
    if (s.sv) {
      double cpl[kMS];
      mix_h_cp<0, double>(T, nullptr, cpl);
      for (int l = 0; l < c_mix.ns; ++l) cp += cpl[l] * ys[l];
    } else {
      cp = kGamma * kRuD / kMwAir / (kGamma - 1);
    }
    double tf = -uf * u / cp;
    tf *= 0.25;
    const double rf = -tf * rho / T;
    u += uf;
    rho += rf;
    T += tf;
    const double p = rho * kRuD / mw * T;
    const long long P = b.plane;
    for (int ig = 0; ig <= b.g; ++ig) {
      const long long pg = b.id(-ig, j, k);
      s.bv[pg] = rho;
      s.bv[P + pg] = u;
      s.bv[2 * P + pg] = vf;
      s.bv[3 * P + pg] = wf;
      s.bv[4 * P + pg] = p;
      s.bv[5 * P + pg] = T;
      if (s.sv)
        for (int l = 0; l < c_mix.ns; ++l) s.sv[l * P + pg] = ys[l];
      finish_node(b, s, pg);
    }
  }
}

}  // namespace ostc
