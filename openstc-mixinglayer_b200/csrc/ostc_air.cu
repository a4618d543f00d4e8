// ostc_air.cu -- sm_100a kernels of the calorically-perfect-air RHS + SSP-RK3 path and the C ABI
// (include/ostc.h) that drives them.
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
#include "air_math.cuh"
#include "host.h"
#include "ostc.h"

#include <cuda_runtime.h>
#include <curand_kernel.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <memory>
#include <string>
#include <type_traits>
#include <vector>

namespace ostc {

// Bounds-checked build (-DOSTC_BOUNDS_CHECK, libostc_b200_checked.so; the sanitizer is not
// available): every padded-plane index id() and interior index iq() is checked against the block's
// extents; an index outside them sets bit 1 (padded) or 2 (interior) of this flag and is clamped into
// range, so the access stays inside the arrays.  ostc_bounds_flags reads and clears it.
__device__ unsigned g_ostc_bounds = 0;

struct DevBlock {
  int mx, my, mz, g, gz, pitch, sy, sz;
  long long plane, off0, n;
  const double *met, *jac;
  __host__ __device__ __forceinline__ long long id(int i, int j, int k) const {
#if defined(OSTC_BOUNDS_CHECK) && defined(__CUDA_ARCH__)
    if (i < -g || i >= pitch - g || j < -g || j >= sy - g || k < -gz || k >= sz - gz) {
      atomicOr(&g_ostc_bounds, 1u);
      i = min(max(i, -g), pitch - g - 1);
      j = min(max(j, -g), sy - g - 1);
      k = min(max(k, -gz), sz - gz - 1);
    }
#endif
    return off0 + ((long long)k * sy + j) * pitch + i;
  }
  __host__ __device__ __forceinline__ long long iq(int i, int j, int k) const {
#if defined(OSTC_BOUNDS_CHECK) && defined(__CUDA_ARCH__)
    if (i < 0 || i >= mx || j < 0 || j >= my || k < 0 || k >= mz) {
      atomicOr(&g_ostc_bounds, 2u);
      i = min(max(i, 0), mx - 1);
      j = min(max(j, 0), my - 1);
      k = min(max(k, 0), mz - 1);
    }
#endif
    return ((long long)k * my + j) * mx + i;
  }
};

struct DevState {
  double *cv, *bv, *mul;
  // mixtures (null on the air path): mass fractions, conductivity, rho*D_k, gamma, acoustic speed
  double *sv = nullptr, *cond = nullptr, *rhod = nullptr, *gam = nullptr, *acs = nullptr;
};

struct DevFace {
  int type, face, direction, rs[3], re[3];
  double density, u, v, w, pressure, temperature, acoustic_speed, gamma, entropy, mw;
  int wall_adiabatic;  // walls: 1 adiabatic, 0 isothermal at `temperature`
  double y[16];        // inflow mass fractions (mixtures)
  // inflows: 0 constant / 2 mixing-layer profile (upper stream above, `lower` below, blended in u by
  // tanh(2 y / delta_omega)); fluct 1 adds white noise of relative intensity fluct_rms, drawn from
  // rng[] at the face node's index in a plane of rng_row nodes per row (apply_inflow's indexing)
  int inflow_type, fluct, rng_row;
  double fluct_rms, velocity, delta_omega;
  double lower[6], y_lower[16];
  const double *ycoord;  // mixing-layer inflow: y of every face node, in the kernel's enumeration
  curandState *rng;
};

struct FillVals {
  double val[16];
};

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

// One block interface (InnerFace after register_boundary, Mesh.cpp:38-141).
struct DevInner {
  int rs[3], ts[3], loop_dir[3], target_loop_dir[3], src_tar[3], n_point[3];
  int face, direction, face_index;  // face_index: the coincident node layer along `face`
};

__device__ __forceinline__ void cv_from_bv_node(const DevBlock &b, DevState s, long long p) {
  // compute_cv_from_bv_1_point + compute_total_energy<Air> (FieldOperation.cuh:17-38,78-105)
  const long long P = b.plane;
  const double rho = s.bv[p], u = s.bv[P + p], v = s.bv[2 * P + p], w = s.bv[3 * P + p];
  s.cv[p] = rho;
  s.cv[P + p] = rho * u;
  s.cv[2 * P + p] = rho * v;
  s.cv[3 * P + p] = rho * w;
  const double V2 = u * u + v * v + w * w;
  double te = 0.5 * V2;
  te *= rho;
  te += s.bv[4 * P + p] / (kGamma - 1);
  s.cv[4 * P + p] = te;
}

}  // namespace ostc

#include "ostc_mix.cuh"
#include "ostc_adj.cuh"
#include "ostc_stat.cuh"
#include "ostc_steady.cuh"
#include "pv_mix.cuh"
#include "ostc_df.cuh"

static_assert(ostc::kMS <= 16, "DevFace::y holds the inflow mass fractions of at most 16 species");

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
    const long long p = base + (long long)n * stride;
#pragma unroll
    for (int l = 0; l < 5; ++l) cp_async8(&Raw(sl, l), s.cv + l * P + p);
#pragma unroll
    for (int l = 0; l < 5; ++l) cp_async8(&Raw(sl, 5 + l), s.bv + l * P + p);
#pragma unroll
    for (int c = 0; c < 3; ++c) cp_async8(&Raw(sl, 10 + c), mrow + c * P + p);
    cp_async8(&Raw(sl, 13), b.jac + p);
  };
  auto prefetch_metric = [&](int n, int sl) {
    const long long p = base + (long long)n * stride;
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
    const long long p = base + (long long)n * stride;
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
  long long pc = base + (long long)(s0 - 1) * stride;
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
      const long long pn = pc + stride;
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
      const long long p = base + (long long)d * stride;
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
// of three k planes (k-1, k, k+1) of u, v, w, T, mu and of the metric + Jacobian, each with a one-node
// halo in i and j, loaded once (coalesced along i).  Every face flux is computed once: x and y faces
// of plane k into shared memory, the z face k+1/2 in registers (carried to the next plane as k-1/2).
template <typename T, bool DIM3, int TX, int TY>
constexpr size_t visc_smem_bytes() {
  return sizeof(T) * ((DIM3 ? 3 : 1) * 15 * (TY + 2) * (TX + 2) + TY * (TX + 1) * 4 + (TY + 1) * TX * 4);
}

template <typename T, bool DIM3, int TX, int TY>
// FP64: the plane ring's shared memory admits two blocks per SM, so registers are not capped for three
__global__ void __launch_bounds__(TX *TY, sizeof(T) == 8 ? 2 : 4) k_visc_update(DevBlock b, StageArgs a, double *__restrict__ dq,
                                                                      int kseg) {
  constexpr int NP = DIM3 ? 3 : 1;  // planes in the ring
  constexpr int SX = TX + 2, SY = TY + 2;
  extern __shared__ __align__(16) unsigned char vsm_raw[];
  auto sv = reinterpret_cast<T(*)[5][SY][SX]>(vsm_raw);
  auto sm = reinterpret_cast<T(*)[10][SY][SX]>(vsm_raw + sizeof(T) * NP * 5 * SY * SX);
  auto fxs = reinterpret_cast<T(*)[TX + 1][4]>(vsm_raw + sizeof(T) * NP * 15 * SY * SX);
  auto fys = reinterpret_cast<T(*)[TX][4]>(vsm_raw + sizeof(T) * (NP * 15 * SY * SX + TY * (TX + 1) * 4));
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
    const int slot = DIM3 ? (kk + 3) % 3 : 0;
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
#pragma unroll
      for (int r = 0; r < 9; ++r) sm[slot][r][y][x] = (T)b.met[r * P + p];
      sm[slot][9][y][x] = (T)b.jac[p];
    }
  };
  // face whose first node is tile node (x, y) of plane kk, direction d
  auto face = [&](int d, int x, int y, int kk, T *fv) {
    const int s0 = DIM3 ? (kk + 3) % 3 : 0;
    auto V = [&](int q, int di, int dj, int dk) -> T {
      const int sl = DIM3 ? (s0 + dk + 3) % 3 : 0;
      return sv[sl][q][y + dj][x + di];
    };
    auto Mt = [&](int r, int sd) -> T {
      if (sd == 0) return sm[s0][r][y][x];
      if (d == 0) return sm[s0][r][y][x + 1];
      if (d == 1) return sm[s0][r][y + 1][x];
      return sm[DIM3 ? (s0 + 1) % 3 : 0][r][y][x];
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
      const long long pg = pb + g * dstep;
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
    const long long pg = pb + g * dstep;
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
      const long long pin = pb - dstep;
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
        const long long pg = pb + g * dstep, pi = pb - g * dstep;
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
        const long long pg = pb + g * dstep;
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
        const long long pg = pb + g * dstep;
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
          const long long p1 = pb - dstep;
          const double d1 = s.bv[p1], u1 = s.bv[P + p1], v1 = s.bv[2 * P + p1], w1 = s.bv[3 * P + p1],
                       pr1 = s.bv[4 * P + p1];
          const double c1 = sqrt(kGamma * pr1 / d1);
          rho_b = d1 + (p_b - pr1) / (c1 * c1);
          u_b = u1 + nx * (pr1 - p_b) / (d1 * c1);
          v_b = v1 + ny * (pr1 - p_b) / (d1 * c1);
          w_b = w1 + nz * (pr1 - p_b) / (d1 * c1);
        }
        for (int g = 1; g <= b.g; ++g) {
          const long long pg = pb + g * dstep, pi = pb - g * dstep;
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
          const long long pg = pb + g * dstep;
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
      const long long pin = pb - dstep;
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
        const long long pi = pb - g * dstep, pg = pb + g * dstep;
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
        const long long pg = pb + g * dstep, ps = po + g * dstep;
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
          const long long pg = pb + g * dstep;
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
        const long long pg = pb + g * dstep;
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

}  // namespace ostc

// ================================================================================= C ABI

using namespace ostc;

struct BlockRes {
  DevBlock db{};
  double *met = nullptr, *jac = nullptr;
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
template <typename T>
int enqueue_step(ostc_ctx *ctx) {
  static const double A[3] = {1.0, 0.75, 1.0 / 3.0}, Bc[3] = {0.0, 0.25, 2.0 / 3.0}, C[3] = {1.0, 0.25, 2.0 / 3.0};
  const bool fixed = ctx->der.fixed_time_step;
  for (int rk = 0; rk < 3; ++rk) {
    const int sin = rk, sout = (rk + 1) % 3;
    if (rk == 0 && !fixed) {
      long tok = begin_t(ctx, "cfl_dt");
      k_dt_reset<<<1, 1, 0, ctx->stream>>>(ctx->d_dtbits);
      for (auto &B : ctx->blk)
        k_cfl_dt<<<grid_for(ctx, B.db.n, 256), 256, 0, ctx->stream>>>(B.db, state_of(B, sin), ctx->der.cfl,
                                                                     ctx->der.prandtl, B.db.mz > 1, ctx->d_dtbits);
      k_dt_decode<<<1, 1, 0, ctx->stream>>>(ctx->d_dtbits, ctx->d_dt);
      end_t(ctx, tok);
    }
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
  k_step_end<<<1, 1, 0, ctx->stream>>>(ctx->d_time, ctx->d_dt, ctx->d_step);
  return OSTC_OK;
}

// CFL time step of the current state (slot 0) into d_dt (local_time_step + global_time_step)
void enqueue_mix_dt(ostc_ctx *ctx) {
  long tok = begin_t(ctx, "cfl_dt");
  k_dt_reset<<<1, 1, 0, ctx->stream>>>(ctx->d_dtbits);
  for (auto &B : ctx->blk)
    k_cfl_dt<<<grid_for(ctx, B.db.n, 256), 256, 0, ctx->stream>>>(B.db, state_of(B, 0), ctx->der.cfl,
                                                                 ctx->der.prandtl, B.db.mz > 1, ctx->d_dtbits);
  k_dt_decode<<<1, 1, 0, ctx->stream>>>(ctx->d_dtbits, ctx->d_dt);
  end_t(ctx, tok);
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
  if (!ctx->der.fixed_time_step) enqueue_mix_dt(ctx);
  for (int rk = 0; rk < 3; ++rk) enqueue_mix_stage(ctx, rk);
  k_step_end<<<1, 1, 0, ctx->stream>>>(ctx->d_time, ctx->d_dt, ctx->d_step);
  return OSTC_OK;
}

// ---- adjoint entry points' shared pieces

// what the adjoint covers: the multi-component path, explicit chemistry, one block, periodic and
// outflow faces
int adjoint_check(ostc_ctx *ctx, unsigned mask) {
  if (!ctx->mixture) {
    ctx->err = "the adjoint covers the multi-component path (species = 1)";
    return OSTC_EINVAL;
  }
  if ((mask & OSTC_TERM_INVISCID) && ctx->der.inviscid_type != 3) {
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
int vjp_core(ostc_ctx *ctx, int block, int slot, unsigned mask, double *out, double *out_t = nullptr) {
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
int step_vjp(ostc_ctx *ctx) {
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
  if (int r = adjoint_check(ctx, OSTC_TERM_ALL)) return r;
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
  if (!ctx->der.fixed_time_step) enqueue_mix_dt(ctx);
  if (int r = step_vjp(ctx)) return r;
  if (int r = adjoint_t_to_cv(ctx)) return r;
  CK(cudaMemcpyAsync(lam_in, B.adj_work, bytes,
                     ptr_kind == OSTC_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return OSTC_OK;
}

int ostc_adjoint_steps(ostc_ctx *ctx, int n_steps, int every, const double *lam_final, double *lam_initial,
                       int ptr_kind) {
  if (!ctx || !lam_final || !lam_initial || n_steps < 1 || every < 1) return OSTC_EINVAL;
  if (int r = adjoint_check(ctx, OSTC_TERM_ALL)) return r;
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
  const size_t state_doubles = (size_t)(nv + 6 + ns) * P;
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
    cudaMemcpyAsync(dst + (size_t)(nv + 6) * P, B.sv[0], (size_t)ns * P * sizeof(double), cudaMemcpyDeviceToDevice,
                    ctx->stream);
  };
  auto restore = [&](const double *src) {
    cudaMemcpyAsync(B.cv[0], src, (size_t)nv * P * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream);
    cudaMemcpyAsync(B.bv[0], src + (size_t)nv * P, 6 * P * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream);
    cudaMemcpyAsync(B.sv[0], src + (size_t)(nv + 6) * P, (size_t)ns * P * sizeof(double), cudaMemcpyDeviceToDevice,
                    ctx->stream);
    launch_mix_props(ctx, B, state_of(B, 0));
  };
  // forward sweep: checkpoints and the dt of every step
  std::vector<double> dts(n_steps);
  for (int n = 0; n < n_steps; ++n) {
    if (n % every == 0) save(cps + (size_t)(n / every) * state_doubles);
    if (!ctx->der.fixed_time_step) enqueue_mix_dt(ctx);
    for (int rk = 0; rk < 3; ++rk) enqueue_mix_stage(ctx, rk);
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
        for (int rk = 0; rk < 3; ++rk) enqueue_mix_stage(ctx, rk);
      }
    }
    for (int n = b - 1; n >= a && rc == OSTC_OK; --n) {
      restore(seg + (size_t)(n - a) * state_doubles);
      cudaMemcpyAsync(ctx->d_dt, &dts[n], sizeof(double), cudaMemcpyHostToDevice, ctx->stream);
      rc = step_vjp(ctx);
    }
  }
  // the first checkpoint is the caller's state, whose T is the equation-of-state root of its cv
  if (rc == OSTC_OK) {
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

// ---------------------------------------------------------------- Tecplot flow-field file

// The zone data of one block in the flow-field file's layout, packed on the device
// (FieldIO::print_field, FieldIO.h:560-648): variable-major arrays over the (mx+2g)(my+2g)(mz+2g) output
// nodes, i fastest; x, y, z from xyz (the same layout), then rho u v w p T, the Mach number as
// update_physical_properties stores it (FieldOperation.cuh:107-140: |V| over the mixture speed of sound,
// or over sqrt(gamma R T) for air) and the mass fractions.  2-D blocks hold no k ghosts: their output k
// layers repeat k = 0, the copies eliminate_k_gradient makes in the reference.
__global__ void k_plt_pack(DevBlock b, DevState s, const double *__restrict__ xyz, int g, int ns, int mixture,
                           double *__restrict__ out) {
  const int nx = b.mx + 2 * g, ny = b.my + 2 * g, nz = b.mz + 2 * g;
  const long long npt = (long long)nx * ny * nz, P = b.plane;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < npt; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % nx) - g;
    const long long r = q / nx;
    const int j = (int)(r % ny) - g, k = (int)(r / ny) - g;
    const long long p = b.id(i, j, b.gz ? k : 0);
    out[q] = xyz[q];
    out[npt + q] = xyz[npt + q];
    out[2 * npt + q] = xyz[2 * npt + q];
    for (int l = 0; l < 6; ++l) out[(3 + l) * npt + q] = s.bv[l * P + p];
    const double u = s.bv[P + p], v = s.bv[2 * P + p], w = s.bv[3 * P + p];
    const double vel = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(u, u), __dmul_rn(v, v)), __dmul_rn(w, w)));
    out[9 * npt + q] = mixture ? vel / s.acs[p] : vel / sqrt(kGammaAir * kRu / kMwAir * s.bv[5 * P + p]);
    for (int l = 0; l < ns; ++l) out[(10 + l) * npt + q] = s.sv[l * P + p];
  }
}

// Per-block partial minima and maxima of every packed variable (the file's min/max pairs): block x of
// row y covers variable y; part[(y * gridDim.x + x) * 2 + 0/1].
__global__ void __launch_bounds__(256) k_plt_minmax(const double *__restrict__ a, long long npt, double *__restrict__ part) {
  __shared__ double smin[256], smax[256];
  const double *v = a + (long long)blockIdx.y * npt;
  double mn = v[0], mxv = v[0];
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < npt; q += (long long)gridDim.x * blockDim.x) {
    mn = fmin(mn, v[q]);
    mxv = fmax(mxv, v[q]);
  }
  smin[threadIdx.x] = mn;
  smax[threadIdx.x] = mxv;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) {
      smin[threadIdx.x] = fmin(smin[threadIdx.x], smin[threadIdx.x + h]);
      smax[threadIdx.x] = fmax(smax[threadIdx.x], smax[threadIdx.x + h]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const long long o = ((long long)blockIdx.y * gridDim.x + blockIdx.x) * 2;
    part[o] = smin[0];
    part[o + 1] = smax[0];
  }
}

// The interior primitive state and mass fractions of one zone read from a flow-field file (its
// selected variable columns cols[6 + ns][npt] staged on the device) into [6][N] and [ns][N].
__global__ void k_plt_gather(DevBlock b, int g, int ns, const double *__restrict__ cols, double *__restrict__ bv,
                             double *__restrict__ sv) {
  const int nx = b.mx + 2 * g, ny = b.my + 2 * g;
  const long long npt = (long long)nx * ny * (b.mz + 2 * g);
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < b.n; n += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(n % b.mx);
    const long long r = n / b.mx;
    const int j = (int)(r % b.my), k = (int)(r / b.my);
    const long long q = ((long long)(k + g) * ny + (j + g)) * nx + (i + g);
    for (int l = 0; l < 6; ++l) bv[l * b.n + n] = cols[l * npt + q];
    for (int l = 0; l < ns; ++l) sv[l * b.n + n] = cols[(6 + l) * npt + q];
  }
}

// Variable names of the flow-field file: FieldIO::acquire_variable_names (FieldIO.h:450-488) for a
// laminar air or mixture case without user-defined output (UDIO.cu:9-33).
static std::vector<std::string> plt_names(const ostc_ctx *ctx) {
  std::vector<std::string> v{"x", "y", "z", "density", "u", "v", "w", "pressure", "temperature", "mach"};
  for (int l = 0; l < ctx->der.n_spec; ++l) v.push_back(ctx->chem.names[l]);
  return v;
}

int ostc_write_plt(ostc_ctx *ctx, const char *path, int ngg_out, double solution_time) {
  if (!ctx || !path) return OSTC_EINVAL;
  cudaSetDevice(ctx->device);
  if (int r = check_ready(ctx)) return r;
  if (ngg_out < 0 || ngg_out > ctx->der.ngg) {
    ctx->err = "ostc_write_plt: ngg_out must lie in [0, ngg]";
    return OSTC_EINVAL;
  }
  CK(cudaStreamSynchronize(ctx->stream));
  const std::vector<std::string> names = plt_names(ctx);
  const int nvar = (int)names.size(), ns = ctx->der.n_spec;
  std::vector<char> buf;
  auto put = [&](const void *p, size_t n) { buf.insert(buf.end(), (const char *)p, (const char *)p + n); };
  auto put_i = [&](int v) { put(&v, 4); };
  auto put_f = [&](float v) { put(&v, 4); };
  auto put_d = [&](double v) { put(&v, 8); };
  auto put_s = [&](const std::string &s) {
    for (char c : s) put_i((int)c);
    put_i(0);
  };
  // header (FieldIO::write_header, FieldIO.h:73-200)
  put("#!TDV112", 8);
  put_i(1);
  put_i(0);
  put_s("Solution file");
  put_i(nvar);
  for (const auto &n : names) put_s(n);
  const int g = ngg_out;
  for (size_t b = 0; b < ctx->blk.size(); ++b) {
    const DevBlock &db = ctx->blk[b].db;
    put_f(299.0f);
    put_s("zone " + std::to_string(b));
    put_i(-1);
    put_i(-2);
    put_d(solution_time);
    put_i(-1);
    put_i(0);
    put_i(0);
    put_i(0);
    put_i(0);
    put_i(db.mx + 2 * g);
    put_i(db.my + 2 * g);
    put_i(db.mz + 2 * g);
    put_i(0);
  }
  put_f(357.0f);
  // data sections (write_common_data_section + print_field, FieldIO.h:222-648): per zone the
  // formats, the min/max pairs and the node arrays of x, y, z, bv, mach, Y_k - packed and reduced on
  // the device, then one copy of the packed zone into the file image
  for (size_t b = 0; b < ctx->blk.size(); ++b) {
    BlockRes &B = ctx->blk[b];
    const DevBlock &db = B.db;
    const int nx = db.mx + 2 * g, ny = db.my + 2 * g, nz = db.mz + 2 * g;
    const long long npt = (long long)nx * ny * nz;
    if (!B.plt_xyz || B.plt_g != g) {
      // the zone's coordinates (ghost grid included) uploaded once per output width
      const HostBlock &hb = ctx->mesh.blocks[b];
      std::vector<double> xyz(3 * (size_t)npt);
      for (int k = -g; k < db.mz + g; ++k)
        for (int j = -g; j < db.my + g; ++j)
          for (int i = -g; i < db.mx + g; ++i) {
            const long long q = ((long long)(k + g) * ny + (j + g)) * nx + (i + g);
            const long c = hb.cidx(i, j, k);
            xyz[q] = hb.x[c];
            xyz[npt + q] = hb.y[c];
            xyz[2 * npt + q] = hb.z[c];
          }
      cudaFree(B.plt_xyz);
      B.plt_xyz = nullptr;
      CK(cudaMalloc(&B.plt_xyz, xyz.size() * sizeof(double)));
      CK(cudaMemcpy(B.plt_xyz, xyz.data(), xyz.size() * sizeof(double), cudaMemcpyHostToDevice));
      B.plt_g = g;
    }
    double *dev = nullptr, *part = nullptr;
    const int nb = (int)std::min<long long>(256, (npt + 255) / 256);
    if (cudaMalloc(&dev, (size_t)nvar * npt * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&part, (size_t)nvar * nb * 2 * sizeof(double)) != cudaSuccess) {
      cudaFree(dev);
      ctx->err = "ostc_write_plt: device allocation for the packed zone failed";
      return OSTC_ENOMEM;
    }
    k_plt_pack<<<grid_for(ctx, npt, 256), 256, 0, ctx->stream>>>(db, state_of(B, 0), B.plt_xyz, g, ns,
                                                                  ctx->mixture ? 1 : 0, dev);
    k_plt_minmax<<<dim3(nb, nvar), 256, 0, ctx->stream>>>(dev, npt, part);
    std::vector<double> hp((size_t)nvar * nb * 2);
    const cudaError_t e1 = cudaMemcpyAsync(hp.data(), part, hp.size() * sizeof(double), cudaMemcpyDeviceToHost,
                                           ctx->stream);
    put_f(299.0f);
    for (int l = 0; l < nvar; ++l) put_i(2);
    put_i(0);
    put_i(0);
    put_i(-1);
    const cudaError_t e2 = cudaStreamSynchronize(ctx->stream);
    for (int l = 0; l < nvar; ++l) {
      double mn = hp[(size_t)l * nb * 2], mxv = hp[(size_t)l * nb * 2 + 1];
      for (int x = 1; x < nb; ++x) {
        mn = std::min(mn, hp[((size_t)l * nb + x) * 2]);
        mxv = std::max(mxv, hp[((size_t)l * nb + x) * 2 + 1]);
      }
      put_d(mn);
      put_d(mxv);
    }
    const size_t at = buf.size();
    buf.resize(at + (size_t)nvar * npt * sizeof(double));
    const cudaError_t e3 =
        cudaMemcpy(buf.data() + at, dev, (size_t)nvar * npt * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(dev);
    cudaFree(part);
    if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess) {
      ctx->err = "ostc_write_plt: device packing failed";
      return OSTC_ECUDA;
    }
  }
  FILE *f = std::fopen(path, "wb");
  if (!f) {
    ctx->err = std::string("ostc_write_plt: cannot open ") + path + " for writing";
    return OSTC_EIO;
  }
  const bool ok = std::fwrite(buf.data(), 1, buf.size(), f) == buf.size();
  if (std::fclose(f) != 0 || !ok) {
    ctx->err = std::string("ostc_write_plt: write to ") + path + " failed";
    return OSTC_EIO;
  }
  return OSTC_OK;
}

int ostc_read_plt(ostc_ctx *ctx, const char *path, double *solution_time) {
  if (!ctx || !path) return OSTC_EINVAL;
  cudaSetDevice(ctx->device);
  FILE *f = std::fopen(path, "rb");
  if (!f) {
    ctx->err = std::string("ostc_read_plt: cannot open ") + path;
    return OSTC_EIO;
  }
  std::vector<char> buf;
  char chunk[1 << 16];
  size_t got;
  while ((got = std::fread(chunk, 1, sizeof(chunk), f)) > 0) buf.insert(buf.end(), chunk, chunk + got);
  std::fclose(f);
  size_t pos = 0;
  bool bad = false;
  auto take = [&](void *dst, size_t n) {
    if (pos + n > buf.size()) {
      bad = true;
      std::memset(dst, 0, n);
      return;
    }
    std::memcpy(dst, buf.data() + pos, n);
    pos += n;
  };
  auto get_i = [&]() { int v; take(&v, 4); return v; };
  auto get_f = [&]() { float v; take(&v, 4); return v; };
  auto get_d = [&]() { double v; take(&v, 8); return v; };
  auto get_s = [&]() {
    std::string s;
    for (int c = get_i(); c != 0 && !bad && s.size() < 4096; c = get_i()) s.push_back((char)c);
    return s;
  };
  auto fail = [&](const std::string &why) {
    ctx->err = std::string("ostc_read_plt: ") + path + ": " + why;
    return OSTC_EIO;
  };
  // header (read_flowfield, Initialize.cuh:102-215)
  if (buf.size() < 8 || std::memcmp(buf.data(), "#!TDV", 5) != 0) return fail("not a Tecplot binary file");
  pos = 8;
  get_i();
  get_i();
  get_s();
  const int nvar = get_i();
  if (bad || nvar <= 0 || nvar > 4096) return fail("bad variable count");
  std::vector<std::string> names(nvar);
  for (auto &n : names) n = get_s();
  std::vector<std::array<int, 3>> dims;
  double t0 = 0;
  float marker = get_f();
  while (!bad && std::fabs(marker - 299.0f) < 1e-3f) {
    get_s();
    get_i();
    get_i();
    const double t = get_d();
    if (dims.empty()) t0 = t;
    get_i();
    if (get_i() != 0) return fail("only ordered zones are read");
    if (get_i() != 0) return fail("only node-located data is read");
    get_i();
    get_i();
    const int d0 = get_i(), d1 = get_i(), d2 = get_i();
    dims.push_back({d0, d1, d2});
    if (get_i() != 0) return fail("zone auxiliary data is not read");
    marker = get_f();
  }
  if (bad || std::fabs(marker - 357.0f) > 1e-3f) return fail("header does not end with the end-of-header marker");
  if (dims.size() != ctx->blk.size()) return fail("zone count differs from the case's block count");
  auto find = [&](const std::string &n) {
    for (int l = 0; l < nvar; ++l)
      if (names[l] == n) return l;
    return -1;
  };
  static const char *const kPrim[6] = {"density", "u", "v", "w", "pressure", "temperature"};
  int col[6 + kMS];
  for (int l = 0; l < 6; ++l)
    if ((col[l] = find(kPrim[l])) < 0) return fail(std::string("no variable '") + kPrim[l] + "'");
  const int ns = ctx->der.n_spec;
  for (int l = 0; l < ns; ++l)
    if ((col[6 + l] = find(ctx->chem.names[l])) < 0) return fail("no variable for species " + ctx->chem.names[l]);
  for (size_t b = 0; b < ctx->blk.size(); ++b) {
    const DevBlock &db = ctx->blk[b].db;
    const int nx = dims[b][0], ny = dims[b][1], nz = dims[b][2];
    const int g = (nx - db.mx) / 2;
    if (g < 0 || nx != db.mx + 2 * g || ny != db.my + 2 * g || nz != db.mz + 2 * g)
      return fail("zone " + std::to_string(b) + " extents do not match block " + std::to_string(b));
    if (std::fabs(get_f() - 299.0f) > 1e-3f) return fail("missing zone data marker");
    for (int l = 0; l < nvar; ++l)
      if (get_i() != 2) return fail("only double-precision variables are read");
    if (get_i() != 0 || get_i() != 0) return fail("passive or shared variables are not read");
    get_i();
    for (int l = 0; l < 2 * nvar; ++l) get_d();
    const long long npt = (long long)nx * ny * nz;
    if (bad || pos + (size_t)nvar * npt * 8 > buf.size()) return fail("truncated zone data");
    const char *a = buf.data() + pos;
    pos += (size_t)nvar * npt * 8;
    // the zone's primitive and species columns go to the device as they lie in the file; the interior
    // is gathered there and set as the block's state
    const long long N = db.n;
    double *cols = nullptr, *st = nullptr;
    if (cudaMalloc(&cols, (size_t)(6 + ns) * npt * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&st, (size_t)(6 + ns) * N * sizeof(double)) != cudaSuccess) {
      cudaFree(cols);
      ctx->err = "ostc_read_plt: device allocation for the zone failed";
      return OSTC_ENOMEM;
    }
    bool okc = true;
    for (int l = 0; l < 6 + ns && okc; ++l)
      okc = cudaMemcpyAsync(cols + (size_t)l * npt, a + (size_t)col[l] * npt * 8, npt * sizeof(double),
                            cudaMemcpyHostToDevice, ctx->stream) == cudaSuccess;
    if (okc) k_plt_gather<<<grid_for(ctx, N, 256), 256, 0, ctx->stream>>>(db, g, ns, cols, st, st + 6 * N);
    const int r = okc ? ostc_set_state(ctx, (int)b, st, ns ? st + 6 * N : nullptr, OSTC_DEVICE) : OSTC_ECUDA;
    cudaFree(cols);
    cudaFree(st);
    if (r) return r;
  }
  // the physical time continues from the file's solution time
  CK(cudaMemcpyAsync(ctx->d_time, &t0, sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (solution_time) *solution_time = t0;
  return OSTC_OK;
}

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
