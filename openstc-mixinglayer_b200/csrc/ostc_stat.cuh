// ostc_stat.cuh -- single-point statistics accumulated after time steps: the basic collector of
// SinglePointStat (collect_single_point_basic_statistics, SinglePointStat.cu:641-706, launched after
// every step past start_collect_statistics_iter, RK.cuh:200-203).
//
// Accumulators of one block: four groups back to back, each [n_var][mz+2][my+2][mx+2] (one ghost
// layer on every side, i fastest: the reference's collect arrays and the layout of its stat files):
//   Reynolds 1st: rho, p, then the stat_rey_1st extras (primitive indices 1 u, 2 v, 3 w, 5 T)
//   Favre 1st:    rho u, rho v, rho w, rho T, rho Y_k
//   Reynolds 2nd: rho rho, p p [, rho p with rho_p_correlation]
//   Favre 2nd:    rho u u, rho v v, rho w w, rho u v, rho u w, rho v w, rho T T, rho Y_k Y_k
// One pass reads the 6 primitive planes and the species planes once and read-modify-writes every
// accumulator plane once: an HBM-bound kernel.
#pragma once

namespace ostc {

struct StatSpec {
  int n_rey;       // stat_rey_1st extras (0..4)
  int rey_idx[4];  // their primitive indices
  int rho_p;       // 1: accumulate rho p
  int ns;          // species (mass fractions accumulated Favre-weighted)
};

__host__ __device__ inline int stat_group_vars(const StatSpec &sp, int g) {
  return g == 0 ? 2 + sp.n_rey : g == 1 ? 4 + sp.ns : g == 2 ? 2 + sp.rho_p : 7 + sp.ns;
}

__host__ __device__ inline long long stat_points(const DevBlock &b) {
  return (long long)(b.mx + 2) * (b.my + 2) * (b.mz + 2);
}

// Products and sums are rounded one at a time (no fused multiply-add), in the reference's order:
// rho * u * v is (rho u) v.  Each thread loads every accumulator it updates before it stores any, so
// the loads of one node are all in flight together (the planes share one base pointer, which would
// otherwise order each load after the previous store).  Point counts fit in 32 bits (the host
// checks): the flat index is split with 32-bit division.
__global__ void __launch_bounds__(256) k_stat_collect(DevBlock b, DevState s, double *__restrict__ acc,
                                                      StatSpec sp) {
  const unsigned nx = b.mx + 2, ny = b.my + 2;
  const unsigned np = (unsigned)stat_points(b);
  const long long P = b.plane;
  double *rey1 = acc;
  double *fav1 = rey1 + (long long)(2 + sp.n_rey) * np;
  double *rey2 = fav1 + (long long)(4 + sp.ns) * np;
  double *fav2 = rey2 + (long long)(2 + sp.rho_p) * np;
  for (unsigned n = blockIdx.x * blockDim.x + threadIdx.x; n < np; n += gridDim.x * blockDim.x) {
    const unsigned r = n / nx;
    const int i = (int)(n - r * nx) - 1;
    const int j = (int)(r % ny) - 1;
    const int k = (int)(r / ny) - 1;
    // 2-D blocks hold no k ghosts; the reference's k = -1 and k = 1 layers are copies of k = 0
    // (eliminate_k_gradient, FieldOperation.cu:42-67)
    const long long p = b.id(i, j, b.gz ? k : 0);
    const double rho = s.bv[p], u = s.bv[P + p], v = s.bv[2 * P + p], w = s.bv[3 * P + p];
    const double pr = s.bv[4 * P + p], T = s.bv[5 * P + p];
    double ex[4];
#pragma unroll
    for (int l = 0; l < 4; ++l) ex[l] = l < sp.n_rey ? s.bv[sp.rey_idx[l] * P + p] : 0.0;
    double a1[6], a2[4], a3[3], a4[7];
#pragma unroll
    for (int l = 0; l < 6; ++l) a1[l] = l < 2 + sp.n_rey ? rey1[(long long)l * np + n] : 0.0;
#pragma unroll
    for (int l = 0; l < 4; ++l) a2[l] = fav1[(long long)l * np + n];
#pragma unroll
    for (int l = 0; l < 3; ++l) a3[l] = l < 2 + sp.rho_p ? rey2[(long long)l * np + n] : 0.0;
#pragma unroll
    for (int l = 0; l < 7; ++l) a4[l] = fav2[(long long)l * np + n];
    const double ru = __dmul_rn(rho, u), rv = __dmul_rn(rho, v), rw = __dmul_rn(rho, w), rT = __dmul_rn(rho, T);
    a1[0] = __dadd_rn(a1[0], rho);
    a1[1] = __dadd_rn(a1[1], pr);
#pragma unroll
    for (int l = 0; l < 4; ++l) a1[2 + l] = __dadd_rn(a1[2 + l], ex[l]);
    a2[0] = __dadd_rn(a2[0], ru);
    a2[1] = __dadd_rn(a2[1], rv);
    a2[2] = __dadd_rn(a2[2], rw);
    a2[3] = __dadd_rn(a2[3], rT);
    a3[0] = __dadd_rn(a3[0], __dmul_rn(rho, rho));
    a3[1] = __dadd_rn(a3[1], __dmul_rn(pr, pr));
    a3[2] = __dadd_rn(a3[2], __dmul_rn(rho, pr));
    a4[0] = __dadd_rn(a4[0], __dmul_rn(ru, u));
    a4[1] = __dadd_rn(a4[1], __dmul_rn(rv, v));
    a4[2] = __dadd_rn(a4[2], __dmul_rn(rw, w));
    a4[3] = __dadd_rn(a4[3], __dmul_rn(ru, v));
    a4[4] = __dadd_rn(a4[4], __dmul_rn(ru, w));
    a4[5] = __dadd_rn(a4[5], __dmul_rn(rv, w));
    a4[6] = __dadd_rn(a4[6], __dmul_rn(rT, T));
#pragma unroll
    for (int l = 0; l < 6; ++l)
      if (l < 2 + sp.n_rey) rey1[(long long)l * np + n] = a1[l];
#pragma unroll
    for (int l = 0; l < 4; ++l) fav1[(long long)l * np + n] = a2[l];
#pragma unroll
    for (int l = 0; l < 3; ++l)
      if (l < 2 + sp.rho_p) rey2[(long long)l * np + n] = a3[l];
#pragma unroll
    for (int l = 0; l < 7; ++l) fav2[(long long)l * np + n] = a4[l];
    // species in groups of 8: mass fractions and both accumulators loaded, then stored
    for (int l0 = 0; l0 < sp.ns; l0 += 8) {
      double y[8], f1[8], f2[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int l = l0 + q;
        y[q] = l < sp.ns ? s.sv[l * P + p] : 0.0;
        f1[q] = l < sp.ns ? fav1[(long long)(4 + l) * np + n] : 0.0;
        f2[q] = l < sp.ns ? fav2[(long long)(7 + l) * np + n] : 0.0;
      }
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int l = l0 + q;
        if (l < sp.ns) {
          const double ry = __dmul_rn(rho, y[q]);
          fav1[(long long)(4 + l) * np + n] = __dadd_rn(f1[q], ry);
          fav2[(long long)(7 + l) * np + n] = __dadd_rn(f2[q], __dmul_rn(ry, y[q]));
        }
      }
    }
  }
}

}  // namespace ostc
