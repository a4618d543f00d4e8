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
  // the additional collectors (stat_lib/, SinglePointStat.cu:707-722), interior nodes only:
  // tke: the viscous stresses and their work (TkeBudget); svc: rho u Y, rho v Y, rho w Y
  // (SpeciesVelocityCorrelation); sdr: rho D |grad Y|^2, rho D grad Y, rho D
  // (SpeciesDissipationRate) of the nss species ss_idx (stat_species)
  int tke, svc, sdr, nss;
  int ss_idx[16];
};

// Groups 0-3: the basic collector (one ghost layer); 4 TKE budget, 5 species velocity correlation,
// 6 species dissipation rate (no ghost layer); a group that is off has no variables.
constexpr int kStatGroups = 7;

__host__ __device__ inline int stat_group_vars(const StatSpec &sp, int g) {
  switch (g) {
    case 0: return 2 + sp.n_rey;
    case 1: return 4 + sp.ns;
    case 2: return 2 + sp.rho_p;
    case 3: return 7 + sp.ns;
    case 4: return sp.tke ? 7 : 0;
    case 5: return sp.svc ? 3 * sp.nss : 0;
    default: return sp.sdr ? 5 * sp.nss : 0;
  }
}

__host__ __device__ inline long long stat_points(const DevBlock &b) {
  return (long long)(b.mx + 2) * (b.my + 2) * (b.mz + 2);
}

__host__ __device__ inline long long stat_group_points(const DevBlock &b, int g) {
  return g < 4 ? stat_points(b) : (long long)b.mx * b.my * b.mz;
}

// offset (doubles) of group g in a block's accumulator buffer
__host__ __device__ inline long long stat_group_offset(const StatSpec &sp, const DevBlock &b, int g) {
  long long o = 0;
  for (int q = 0; q < g; ++q) o += stat_group_vars(sp, q) * stat_group_points(b, q);
  return o;
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

// collect_single_point_additional_statistics (SinglePointStat.cu:707-722) over the interior nodes:
// collect_tke_budget (TkeBudget.cu:123-170), collect_species_velocity_correlation and
// collect_species_dissipation_rate (SpeciesStat.cu:5-85).  Velocity and mass-fraction gradients by
// central differences in computational space times the metric; 2-D blocks hold no k ghosts and their
// zeta differences (copies of k = 0 in the reference) are zero, so those terms are left out.
// ext: the block's accumulators of group 4 onwards.
__global__ void __launch_bounds__(128) k_stat_extra(DevBlock b, DevState s, double *__restrict__ ext, StatSpec sp) {
  const long long P = b.plane, n_all = b.n;
  double *tke = ext;
  double *svc = tke + (long long)stat_group_vars(sp, 4) * n_all;
  double *sdr = svc + (long long)stat_group_vars(sp, 5) * n_all;
  const bool is3d = b.gz > 0;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < n_all; n += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(n % b.mx);
    const long long r = n / b.mx;
    const int j = (int)(r % b.my), k = (int)(r / b.my);
    const long long p = b.id(i, j, k);
    const long long pi0 = b.id(i - 1, j, k), pi1 = b.id(i + 1, j, k), pj0 = b.id(i, j - 1, k), pj1 = b.id(i, j + 1, k);
    const long long pk0 = is3d ? b.id(i, j, k - 1) : p, pk1 = is3d ? b.id(i, j, k + 1) : p;
    double m[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) m[q] = b.met[q * P + p];
    // d/dx, d/dy, d/dz of plane f at this node
    auto grad = [&](const double *f, double g[3]) {
      const double dxi = f[pi1] - f[pi0], deta = f[pj1] - f[pj0];
      const double dzeta = is3d ? f[pk1] - f[pk0] : 0.0;
#pragma unroll
      for (int c = 0; c < 3; ++c)
        g[c] = is3d ? 0.5 * (m[c] * dxi + m[3 + c] * deta + m[6 + c] * dzeta) : 0.5 * (m[c] * dxi + m[3 + c] * deta);
    };
    if (sp.tke) {
      double gu[3], gv[3], gw[3];
      grad(s.bv + P, gu);
      grad(s.bv + 2 * P, gv);
      grad(s.bv + 3 * P, gw);
      const double mu = s.mul[p];
      const double t11 = mu * (4.0 * gu[0] - 2 * gv[1] - 2 * gw[2]) / 3.0;
      const double t12 = mu * (gu[1] + gv[0]);
      const double t13 = mu * (gu[2] + gw[0]);
      const double t22 = mu * (4.0 * gv[1] - 2 * gu[0] - 2 * gw[2]) / 3.0;
      const double t23 = mu * (gv[2] + gw[1]);
      const double t33 = mu * (4.0 * gw[2] - 2 * gu[0] - 2 * gv[1]) / 3.0;
      tke[n] += t11;
      tke[n_all + n] += t12;
      tke[2 * n_all + n] += t13;
      tke[3 * n_all + n] += t22;
      tke[4 * n_all + n] += t23;
      tke[5 * n_all + n] += t33;
      tke[6 * n_all + n] += t11 * gu[0] + t12 * gu[1] + t13 * gu[2] + t12 * gv[0] + t22 * gv[1] + t23 * gv[2] +
                            t13 * gw[0] + t23 * gw[1] + t33 * gw[2];
    }
    if (sp.svc) {
      const double rho = s.bv[p], u = s.bv[P + p], v = s.bv[2 * P + p], w = s.bv[3 * P + p];
      for (int q = 0; q < sp.nss; ++q) {
        const double z = s.sv[sp.ss_idx[q] * P + p];
        svc[(3 * q) * n_all + n] += rho * u * z;
        svc[(3 * q + 1) * n_all + n] += rho * v * z;
        svc[(3 * q + 2) * n_all + n] += rho * w * z;
      }
    }
    if (sp.sdr) {
      for (int q = 0; q < sp.nss; ++q) {
        const int is = sp.ss_idx[q];
        double gz[3];
        grad(s.sv + is * P, gz);
        const double rd = s.rhod[is * P + p];
        sdr[(5 * q) * n_all + n] += rd * (gz[0] * gz[0] + gz[1] * gz[1] + gz[2] * gz[2]);
        sdr[(5 * q + 1) * n_all + n] += rd * gz[0];
        sdr[(5 * q + 2) * n_all + n] += rd * gz[1];
        sdr[(5 * q + 3) * n_all + n] += rd * gz[2];
        sdr[(5 * q + 4) * n_all + n] += rd;
      }
    }
  }
}

}  // namespace ostc
