// ostc_adj.cuh -- vector-Jacobian product of the multi-component right-hand side (ostc_rhs_vjp):
// cv_bar = (d dq / d cv)^T dq_bar at the current state, for the flux-split WENO7 sweeps (71 / 72),
// the mixture viscous sweeps, the finite-rate chemistry source, the mixture transport properties, the
// equation of state and the periodic / outflow ghost fills.  The reference has no adjoint; this is
// the discrete adjoint of the forward kernels in ostc_mix.cuh, term by term:
//   1. face sweeps (hand-written reverse): dq_bar -> adjoints of the node quantities they read
//      (cv, p, acoustic speed; u, v, w, T, Y, mu, lambda, rho*D), accumulated per padded node;
//   2. chemistry and transport properties (node-local, forward-mode Dual evaluations of the same
//      templated device code, one seeded input per pass): -> adjoints of rho, p, T, Y;
//   3. equation of state reverse (rho, u, v, w, p, T, Y as functions of cv, T through the
//      implicit energy relation) -> cv adjoint per padded node;
//   4. ghost fills in reverse order: a ghost's cv adjoint is added to the node it was copied from.
// Accumulation into shared memory and into the node planes uses atomicAdd, so results are
// reproducible to rounding, not bitwise.
#pragma once

#include "ostc_mix.cuh"

namespace ostc {

// Node adjoint planes (padded layout of the state): cv[nv], p, c (acoustic speed), rho, vel[3], T,
// Y[ns], mu, lam (conductivity), rhod[ns].
struct DevAdj {
  double *cv, *p, *c, *rho, *vel, *T, *Y, *mu, *lam, *rhod;
};

// One side of the flux-split WENO7-Z (fvs_weno7_core) with its gradient.  v[0..6] in the orientation
// of the + side (the - side passes its stencil mirrored, v[j] = vm[6 - j]); returns the side's face
// value and adds af * d(value)/d(v[j]) to g[j].  The third smoothness indicator reuses the second
// stencil's second difference, as the forward function does.
__device__ __forceinline__ double weno7_side_bwd(const double *v, double eps, double af, double *g) {
  const double c[4] = {1.0 / 35, 12.0 / 35, 18.0 / 35, 4.0 / 35};
  const double one6th = 1.0 / 6, one12th = 1.0 / 12;
  double s1[4], s2[4], s3[4], b[4], q[4], d[4], a[4];
  s1[0] = one6th * (-2 * v[0] + 9 * v[1] - 18 * v[2] + 11 * v[3]);
  s2[0] = -v[0] + 4 * v[1] - 5 * v[2] + 2 * v[3];
  s3[0] = -v[0] + 3 * v[1] - 3 * v[2] + v[3];
  s1[1] = one6th * (v[1] - 6 * v[2] + 3 * v[3] + 2 * v[4]);
  s2[1] = v[2] - 2 * v[3] + v[4];
  s3[1] = -v[1] + 3 * v[2] - 3 * v[3] + v[4];
  s1[2] = one6th * (-2 * v[2] - 3 * v[3] + 6 * v[4] - v[5]);
  s2[2] = s2[1];
  s3[2] = -v[2] + 3 * v[3] - 3 * v[4] + v[5];
  s1[3] = one6th * (-11 * v[3] + 18 * v[4] - 9 * v[5] + 2 * v[6]);
  s2[3] = 2 * v[3] - 5 * v[4] + 4 * v[5] - v[6];
  s3[3] = -v[3] + 3 * v[4] - 3 * v[5] + v[6];
#pragma unroll
  for (int k = 0; k < 4; ++k) b[k] = fvs_beta7(s1[k], s2[k], s3[k]);
  q[0] = one12th * (-3 * v[0] + 13 * v[1] - 23 * v[2] + 25 * v[3]);
  q[1] = one12th * (v[1] - 5 * v[2] + 13 * v[3] + 3 * v[4]);
  q[2] = one12th * (-v[2] + 7 * v[3] + 7 * v[4] - v[5]);
  q[3] = one12th * (3 * v[3] + 13 * v[4] - 5 * v[5] + v[6]);
  const double tau = (b[0] - b[3]) * (b[0] - b[3]);
  double S = 0, num = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    d[k] = eps + b[k];
    a[k] = c[k] + c[k] * tau / (d[k] * d[k]);
    S += a[k];
    num += a[k] * q[k];
  }
  const double f = num / S;
  // reverse
  double aq[4], ab[4], atau = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    aq[k] = af * a[k] / S;
    const double aa = af * (q[k] - f) / S;
    const double id2 = 1.0 / (d[k] * d[k]);
    atau += aa * c[k] * id2;
    ab[k] = -2.0 * aa * c[k] * tau * id2 / d[k];
  }
  ab[0] += 2.0 * atau * (b[0] - b[3]);
  ab[3] -= 2.0 * atau * (b[0] - b[3]);
  double a1[4], a2[4], a3[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    a1[k] = ab[k] * (2 * s1[k] + s3[k] / 12);
    a2[k] = ab[k] * (26.0 / 12.0) * s2[k];
    a3[k] = ab[k] * (2 * (1043.0 / 960) * s3[k] + s1[k] / 12);
  }
  a2[1] += a2[2];  // the reused second difference
  // stencil 0: v0..v3
  g[0] += one6th * -2 * a1[0] - a2[0] - a3[0] + one12th * -3 * aq[0];
  g[1] += one6th * 9 * a1[0] + 4 * a2[0] + 3 * a3[0] + one12th * 13 * aq[0];
  g[2] += one6th * -18 * a1[0] - 5 * a2[0] - 3 * a3[0] + one12th * -23 * aq[0];
  g[3] += one6th * 11 * a1[0] + 2 * a2[0] + a3[0] + one12th * 25 * aq[0];
  // stencil 1: v1..v4
  g[1] += one6th * a1[1] - a3[1] + one12th * aq[1];
  g[2] += one6th * -6 * a1[1] + a2[1] + 3 * a3[1] + one12th * -5 * aq[1];
  g[3] += one6th * 3 * a1[1] - 2 * a2[1] - 3 * a3[1] + one12th * 13 * aq[1];
  g[4] += one6th * 2 * a1[1] + a2[1] + a3[1] + one12th * 3 * aq[1];
  // stencil 2: v2..v5
  g[2] += one6th * -2 * a1[2] - a3[2] - one12th * aq[2];
  g[3] += one6th * -3 * a1[2] + 3 * a3[2] + one12th * 7 * aq[2];
  g[4] += one6th * 6 * a1[2] - 3 * a3[2] + one12th * 7 * aq[2];
  g[5] += one6th * -1 * a1[2] + a3[2] - one12th * aq[2];
  // stencil 3: v3..v6
  g[3] += one6th * -11 * a1[3] + 2 * a2[3] - a3[3] + one12th * 3 * aq[3];
  g[4] += one6th * 18 * a1[3] - 5 * a2[3] + 3 * a3[3] + one12th * 13 * aq[3];
  g[5] += one6th * -9 * a1[3] + 4 * a2[3] - 3 * a3[3] + one12th * -5 * aq[3];
  g[6] += one6th * 2 * a1[3] - a2[3] + a3[3] + one12th * aq[3];
  return f;
}

// fvs_weno7 (both sides) reverse: gp[j] += af d/d vp[j], gm[j] += af d/d vm[j]
__device__ __forceinline__ void weno7_bwd(const double *vp, const double *vm, double eps, double af, double *gp,
                                          double *gm) {
  weno7_side_bwd(vp, eps, af, gp);
  double r[7], gr[7];
#pragma unroll
  for (int j = 0; j < 7; ++j) {
    r[j] = vm[6 - j];
    gr[j] = 0.0;
  }
  weno7_side_bwd(r, eps, af, gr);
#pragma unroll
  for (int j = 0; j < 7; ++j) gm[6 - j] += gr[j];
}

// Reverse of the node's split fluxes F+- = J/2 (Uk Q + p grad k (+ p Uk in energy) +- l0 Q),
// Uk = (Q1 kx + Q2 ky + Q3 kz) / Q0, l0 = |Uk| + c |grad k| (compute_flux, WENO.cu:697-720):
// adds to aQ[nv], ap, ac.
__device__ __forceinline__ void fvs_node_bwd(const double *Q, double pk, double c, double k0m, double k1m, double k2m,
                                             double jac, const double *aFp, const double *aFm, int nv, double *aQ,
                                             double &ap, double &ac) {
  const double Uk = (Q[1] * k0m + Q[2] * k1m + Q[3] * k2m) / Q[0];
  const double kn = sqrt(k0m * k0m + k1m * k1m + k2m * k2m);
  const double l0 = fabs(Uk) + c * kn;
  const double hj = 0.5 * jac;
  double aUk = 0, al0 = 0;
  const double km[3] = {k0m, k1m, k2m};
  for (int q = 0; q < nv; ++q) {
    const double S = aFp[q] + aFm[q], D = aFp[q] - aFm[q];
    aQ[q] += hj * (Uk * S + l0 * D);
    aUk += hj * Q[q] * S;
    al0 += hj * Q[q] * D;
    if (q >= 1 && q <= 3) ap += hj * km[q - 1] * S;
    if (q == 4) {
      ap += hj * Uk * S;
      aUk += hj * pk * S;
    }
  }
  aUk += al0 * (Uk > 0 ? 1.0 : (Uk < 0 ? -1.0 : 0.0));
  ac += al0 * kn;
  const double iq0 = 1.0 / Q[0];
  aQ[1] += aUk * k0m * iq0;
  aQ[2] += aUk * k1m * iq0;
  aQ[3] += aUk * k2m * iq0;
  aQ[0] -= aUk * Uk * iq0;
}

// d cp_i / dT of the NASA-7 polynomials (0 below t_low, where cp is frozen), per species
template <int NS>
__device__ __forceinline__ void mix_dcp_dt(double t, double *dcp) {
#pragma unroll
  for (int i = 0; i < OSTC_NS; ++i) {
    if (t < c_mix.t_low[i]) {
      dcp[i] = 0.0;
    } else {
      const double *a = t < c_mix.t_mid[i] ? c_mix.low[i] : c_mix.high[i];
      dcp[i] = (a[1] + t * (2 * a[2] + t * (3 * a[3] + t * 4 * a[4]))) * c_mix.ru_mw[i];
    }
  }
}

// Left-eigenvector row l (0..4) of the Roe-averaged mixture eigensystem (WENO.cu:822-898) as the
// forward sweep forms it: L[0..4] on the five flow components and cs, the factor of the species part.
__device__ __forceinline__ void fvs_lrow(int l, double alpha, double Ukb, double cm, double c2i, double gm1, double um,
                                         double vm, double wm, double kx, double ky, double kz, double *L, double &cs) {
  cs = 0.5;
  if (l == 0) {
    L[0] = (alpha + Ukb * cm) * c2i * 0.5;
    L[1] = -(gm1 * um + kx * cm) * c2i * 0.5;
    L[2] = -(gm1 * vm + ky * cm) * c2i * 0.5;
    L[3] = -(gm1 * wm + kz * cm) * c2i * 0.5;
    L[4] = gm1 * c2i * 0.5;
  } else if (l == 1) {
    cs = -kx;
    L[0] = kx * (1 - alpha * c2i) - (kz * vm - ky * wm) / cm;
    L[1] = kx * gm1 * um * c2i;
    L[2] = (kx * gm1 * vm + kz * cm) * c2i;
    L[3] = (kx * gm1 * wm - ky * cm) * c2i;
    L[4] = -kx * gm1 * c2i;
  } else if (l == 2) {
    cs = -ky;
    L[0] = ky * (1 - alpha * c2i) - (kx * wm - kz * um) / cm;
    L[1] = (ky * gm1 * um - kz * cm) * c2i;
    L[2] = ky * gm1 * vm * c2i;
    L[3] = (ky * gm1 * wm + kx * cm) * c2i;
    L[4] = -ky * gm1 * c2i;
  } else if (l == 3) {
    cs = -kz;
    L[0] = kz * (1 - alpha * c2i) - (ky * um - kx * vm) / cm;
    L[1] = (kz * gm1 * um + ky * cm) * c2i;
    L[2] = (kz * gm1 * vm - kx * cm) * c2i;
    L[3] = kz * gm1 * wm * c2i;
    L[4] = -kz * gm1 * c2i;
  } else {
    L[0] = (alpha - Ukb * cm) * c2i * 0.5;
    L[1] = -(gm1 * um - kx * cm) * c2i * 0.5;
    L[2] = -(gm1 * vm - ky * cm) * c2i * 0.5;
    L[3] = -(gm1 * wm - kz * cm) * c2i * 0.5;
    L[4] = gm1 * c2i * 0.5;
  }
}

// Adjoint of the Roe-state symbols that the rows of fvs_lrow read, given AL = adjoint of L[0..4]
struct RoeBar {
  double alpha, Ukb, cm, c2i, gm1, um, vm, wm;
};
__device__ __forceinline__ void fvs_lrow_bwd(int l, const double *AL, double alpha, double Ukb, double cm, double c2i,
                                             double gm1, double um, double vm, double wm, double kx, double ky,
                                             double kz, RoeBar &r) {
  const double V[3] = {um, vm, wm}, k[3] = {kx, ky, kz};
  double aV[3] = {0, 0, 0};
  if (l == 0 || l == 4) {
    const double sg = l == 0 ? 1.0 : -1.0;
    r.alpha += AL[0] * c2i * 0.5;
    r.Ukb += sg * AL[0] * cm * c2i * 0.5;
    r.cm += sg * AL[0] * Ukb * c2i * 0.5;
    r.c2i += AL[0] * (alpha + sg * Ukb * cm) * 0.5;
    for (int q = 0; q < 3; ++q) {
      const double a = AL[q + 1];
      r.gm1 -= a * V[q] * c2i * 0.5;
      aV[q] -= a * gm1 * c2i * 0.5;
      r.cm -= sg * a * k[q] * c2i * 0.5;
      r.c2i -= a * (gm1 * V[q] + sg * k[q] * cm) * 0.5;
    }
    r.gm1 += AL[4] * c2i * 0.5;
    r.c2i += AL[4] * gm1 * 0.5;
  } else {
    const int d = l - 1;
    const double kd = k[d];
    // E[d][q]: coefficient of cm in L[q + 1] (antisymmetric, from the rows above)
    const double E[3][3] = {{0.0, kz, -ky}, {-kz, 0.0, kx}, {ky, -kx, 0.0}};
    r.alpha -= AL[0] * kd * c2i;
    r.c2i -= AL[0] * kd * alpha;
    // L0's cross term -X/cm, X = (kz vm - ky wm, kx wm - kz um, ky um - kx vm)[d]
    const double X = d == 0 ? kz * vm - ky * wm : (d == 1 ? kx * wm - kz * um : ky * um - kx * vm);
    r.cm += AL[0] * X / (cm * cm);
    const double aX = -AL[0] / cm;
    if (d == 0) {
      aV[1] += kz * aX;
      aV[2] -= ky * aX;
    } else if (d == 1) {
      aV[2] += kx * aX;
      aV[0] -= kz * aX;
    } else {
      aV[0] += ky * aX;
      aV[1] -= kx * aX;
    }
    for (int q = 0; q < 3; ++q) {
      const double a = AL[q + 1];
      r.gm1 += a * kd * V[q] * c2i;
      aV[q] += a * kd * gm1 * c2i;
      r.cm += a * E[d][q] * c2i;
      r.c2i += a * (kd * gm1 * V[q] + E[d][q] * cm);
    }
    r.gm1 -= AL[4] * kd * c2i;
    r.c2i -= AL[4] * kd * gm1;
  }
  r.um += aV[0];
  r.vm += aV[1];
  r.wm += aV[2];
}

template <int DIR>
__host__ __device__ constexpr size_t adj_fvs_smem_bytes(int nv) {
  // F+, F- (recomputed), their adjoints, and the Roe-average adjoints (cv and p) per staged node
  return (size_t)FvsTile<DIR>::NST * FvsTile<DIR>::TXL * (5 * nv + 1) * sizeof(double);
}

// Reverse of k_fvs: the tile recomputes the staged split fluxes, every face thread turns its face
// adjoint (from dq_bar of the nodes this tile owns) into adjoints of the staged split fluxes (shared
// atomics) and of the Roe-averaged face state, and after a barrier every staged node maps its split-
// flux adjoints back to cv, p and c and adds them to the node planes.
template <int DIR, int NS>
__global__ void __launch_bounds__(FvsTile<DIR>::TD * FvsTile<DIR>::TXL) k_adj_fvs(DevBlock b, DevState s,
                                                                                   const double *__restrict__ dqb,
                                                                                   int nv, int scheme, DevAdj A) {
  constexpr int TXL = FvsTile<DIR>::TXL, TD = FvsTile<DIR>::TD, NST = FvsTile<DIR>::NST;
  extern __shared__ __align__(16) unsigned char adj_smem[];
  if (NS > 0) nv = 5 + NS;
  const int ns = OSTC_NS;
  double *Fp = reinterpret_cast<double *>(adj_smem);
  double *Fm = Fp + NST * TXL * nv;
  double *aFp = Fm + NST * TXL * nv;
  double *aFm = aFp + NST * TXL * nv;
  double *aR = aFm + NST * TXL * nv;  // [NST][TXL][nv + 1]
  const int lane = DIR == 0 ? 0 : (int)threadIdx.x;
  const int t = DIR == 0 ? (int)threadIdx.x : (int)threadIdx.y;
  const int tid = DIR == 0 ? t : t * TXL + lane;
  const long long P = b.plane;
  const int nd = DIR == 0 ? b.mx : DIR == 1 ? b.my : b.mz;
  const int start = (DIR == 0 ? blockIdx.x : blockIdx.y) * (TD - 1);
  int i0, j0, k0;
  if (DIR == 0) {
    i0 = 0; j0 = blockIdx.y; k0 = blockIdx.z;
  } else if (DIR == 1) {
    i0 = blockIdx.x * TXL + lane; j0 = 0; k0 = blockIdx.z;
  } else {
    i0 = blockIdx.x * TXL + lane; j0 = blockIdx.z; k0 = 0;
  }
  const bool lane_ok = i0 < b.mx;
  auto pid = [&](int n) -> long long {
    return DIR == 0 ? b.id(n, j0, k0) : DIR == 1 ? b.id(i0, n, k0) : b.id(i0, j0, n);
  };
  auto qid = [&](int n) -> long long {
    return DIR == 0 ? b.iq(n, j0, k0) : DIR == 1 ? b.iq(i0, n, k0) : b.iq(i0, j0, n);
  };
  for (int e = tid; e < NST * TXL * (3 * nv + 1); e += TD * TXL) aFp[e] = 0.0;
  if (lane_ok) {
    for (int st = t; st < NST; st += TD) {
      const int n = start - 4 + st;
      if (n > nd + 3) continue;
      const long long p = pid(n);
      double Q[Spec<NS>::A + 5];
      for (int l = 0; l < nv; ++l) Q[l] = s.cv[l * P + p];
      const double pk = s.bv[4 * P + p], c = s.acs[p];
      const double k0m = b.met[(DIR * 3 + 0) * P + p], k1m = b.met[(DIR * 3 + 1) * P + p],
                   k2m = b.met[(DIR * 3 + 2) * P + p];
      const double jac = b.jac[p];
      const double Uk = (Q[1] * k0m + Q[2] * k1m + Q[3] * k2m) / Q[0];
      const double l0 = fabs(Uk) + c * sqrt(k0m * k0m + k1m * k1m + k2m * k2m);
      double *fp = Fp + ((long long)st * TXL + lane) * nv, *fm = Fm + ((long long)st * TXL + lane) * nv;
      for (int l = 0; l < nv; ++l) {
        const double pt = l >= 1 && l <= 3 ? pk * (l == 1 ? k0m : l == 2 ? k1m : k2m) : 0.0;
        const double conv = l == 4 ? Uk * (Q[4] + pk) : Uk * Q[l] + pt;
        fp[l] = 0.5 * jac * (conv + l0 * Q[l]);
        fm[l] = 0.5 * jac * (conv - l0 * Q[l]);
      }
    }
  }
  __syncthreads();
  const int n = start - 1 + t;  // left node of this thread's face
  const bool face_ok = lane_ok && n < nd;
  auto FP = [&](int m, int l) -> double { return Fp[((long long)(t + m) * TXL + lane) * nv + l]; };
  auto FM = [&](int m, int l) -> double { return Fm[((long long)(t + m) * TXL + lane) * nv + l]; };
  auto AFP = [&](int m, int l) -> double * { return aFp + ((long long)(t + m) * TXL + lane) * nv + l; };
  auto AFM = [&](int m, int l) -> double * { return aFm + ((long long)(t + m) * TXL + lane) * nv + l; };
  double afc[Spec<NS>::A + 5];
  bool any = false;
  for (int l = 0; l < nv; ++l) {
    double a = 0.0;
    if (face_ok && t >= 1) a -= dqb[l * b.n + qid(n)];
    if (face_ok && t <= TD - 2 && n + 1 < nd) a += dqb[l * b.n + qid(n + 1)];
    afc[l] = a;
    any = any || a != 0.0;
  }
  if (face_ok && any && scheme == 71) {
    const long long pl = pid(n), pr = pid(n + 1);
    const double j1 = b.jac[pl], j2 = b.jac[pr];
    double a[3];
    for (int q = 0; q < 3; ++q) a[q] = b.met[(DIR * 3 + q) * P + pl] * j1 + b.met[(DIR * 3 + q) * P + pr] * j2;
    const double eps_ref = 1e-20 * c_mix.weno_eps_scale * 0.25 * (a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
    const double e1 = eps_ref * c_mix.v_ref * c_mix.v_ref;
    const double e2 = e1 * c_mix.v_ref * c_mix.v_ref;
    for (int l = 0; l < nv; ++l) {
      const double e = (l >= 1 && l <= 3) ? e1 : (l == 4 ? e2 : eps_ref);
      double vp[7], vm[7], gp[7], gm[7];
      for (int m = 0; m < 7; ++m) {
        vp[m] = FP(m, l);
        vm[m] = FM(m + 1, l);
        gp[m] = gm[m] = 0.0;
      }
      weno7_bwd(vp, vm, e, afc[l], gp, gm);
      for (int m = 0; m < 7; ++m) {
        atomicAdd(AFP(m, l), gp[m]);
        atomicAdd(AFM(m + 1, l), gm[m]);
      }
    }
  } else if (face_ok && any) {
    // forward: Roe-averaged mixture state at the face (as k_fvs)
    const long long pl = pid(n), pr = pid(n + 1);
    double cvl[Spec<NS>::A + 5], cvr[Spec<NS>::A + 5];
    for (int l = 0; l < nv; ++l) {
      cvl[l] = s.cv[l * P + pl];
      cvr[l] = s.cv[l * P + pr];
    }
    const double p_l = s.bv[4 * P + pl], p_r = s.bv[4 * P + pr];
    const double rli = 1.0 / cvl[0], rri = 1.0 / cvr[0];
    const double sl = sqrt(cvl[0]), sr = sqrt(cvr[0]);
    const double den = sl + sr, rlc = sl / den, rrc = sr / den;
    const double um = rlc * cvl[1] * rli + rrc * cvr[1] * rri;
    const double vm = rlc * cvl[2] * rli + rrc * cvr[2] * rri;
    const double wm = rlc * cvl[3] * rli + rrc * cvr[3] * rri;
    const double ekm = 0.5 * (um * um + vm * vm + wm * wm);
    const double hm = rlc * ((cvl[4] + p_l) * rli) + rrc * ((cvr[4] + p_r) * rri);
    double svm[Spec<NS>::A], hi[Spec<NS>::A], cpi[Spec<NS>::A], al[Spec<NS>::A];
    double mw_inv = 0;
    for (int l = 0; l < ns; ++l) {
      svm[l] = rlc * cvl[l + 5] * rli + rrc * cvr[l + 5] * rri;
      mw_inv += svm[l] / c_mix.mw[l];
    }
    const double prm = rlc * (p_l * rli) + rrc * (p_r * rri);
    const double tm = prm / (kRuD * mw_inv);
    mix_h_cp<NS, double>(tm, hi, cpi);
    double cp = 0, cvt = 0;
    for (int l = 0; l < ns; ++l) {
      cp += svm[l] * cpi[l];
      cvt += svm[l] * (cpi[l] - c_mix.ru_mw[l]);
    }
    const double gamma = cp / cvt;
    const double cm = sqrt(gamma * kRuD * mw_inv * tm);
    const double gm1 = gamma - 1;
    const double jl = b.jac[pl], jr = b.jac[pr];
    const double kxJ = b.met[(DIR * 3 + 0) * P + pl] * jl + b.met[(DIR * 3 + 0) * P + pr] * jr;
    const double kyJ = b.met[(DIR * 3 + 1) * P + pl] * jl + b.met[(DIR * 3 + 1) * P + pr] * jr;
    const double kzJ = b.met[(DIR * 3 + 2) * P + pl] * jl + b.met[(DIR * 3 + 2) * P + pr] * jr;
    double kx = kxJ / (jl + jr), ky = kyJ / (jl + jr), kz = kzJ / (jl + jr);
    const double gradK = sqrt(kx * kx + ky * ky + kz * kz);
    kx /= gradK;
    ky /= gradK;
    kz /= gradK;
    const double Ukb = kx * um + ky * vm + kz * wm;
    const double alpha = gm1 * ekm;
    const double c2i = 1.0 / (cm * cm);
    const double eps = 1e-40 * c_mix.weno_eps_scale * 0.25 * (kxJ * kxJ + kyJ * kyJ + kzJ * kzJ);
    for (int l = 0; l < ns; ++l) al[l] = (gamma * kRuD / c_mix.mw[l] * tm - (gamma - 1) * hi[l]) * c2i;
    // characteristic projections and face values
    auto project = [&](int l, double *vp, double *vmn) {
      if (l < 5) {
        double L[5], cs;
        fvs_lrow(l, alpha, Ukb, cm, c2i, gm1, um, vm, wm, kx, ky, kz, L, cs);
        for (int m = 0; m < 7; ++m) {
          double a = 0, bq = 0;
          for (int q = 0; q < 5; ++q) {
            a += L[q] * FP(m, q);
            bq += L[q] * FM(m + 1, q);
          }
          for (int q = 0; q < ns; ++q) {
            a += cs * al[q] * FP(m, 5 + q);
            bq += cs * al[q] * FM(m + 1, 5 + q);
          }
          vp[m] = a;
          vmn[m] = bq;
        }
      } else {
        for (int m = 0; m < 7; ++m) {
          vp[m] = -svm[l - 5] * FP(m, 0) + FP(m, l);
          vmn[m] = -svm[l - 5] * FM(m + 1, 0) + FM(m + 1, l);
        }
      }
    };
    double fch[Spec<NS>::A + 5];
    for (int l = 0; l < nv; ++l) {
      double vp[7], vmn[7];
      project(l, vp, vmn);
      fch[l] = fvs_weno7(vp, vmn, eps);
    }
    // reverse of fc = R fch (WENO.cu:1069-1117)
    const double ca = fch[0] + kx * fch[1] + ky * fch[2] + kz * fch[3] + fch[4];
    const double cg = cm * cm / gm1;
    const double hc = hm - cg;
    double add = 0, aca = afc[0];
    for (int l = 0; l < ns; ++l) {
      add += al[l] * fch[l + 5];
      aca += svm[l] * afc[5 + l];
    }
    double afch[Spec<NS>::A + 5], a_svm[Spec<NS>::A], a_al[Spec<NS>::A];
    for (int l = 0; l < ns; ++l) {
      afch[5 + l] = afc[5 + l] - afc[4] * al[l] * cg;
      a_svm[l] = ca * afc[5 + l];
      a_al[l] = -afc[4] * fch[5 + l] * cg;
    }
    double a_cg = -afc[4] * add;
    afch[0] = aca + afc[1] * (um - kx * cm) + afc[2] * (vm - ky * cm) + afc[3] * (wm - kz * cm) + afc[4] * (hm - Ukb * cm);
    afch[1] = aca * kx + afc[1] * kx * um + afc[2] * (kx * vm + kz * cm) + afc[3] * (kx * wm - ky * cm) +
              afc[4] * (kx * hc + (kz * vm - ky * wm) * cm);
    afch[2] = aca * ky + afc[1] * (ky * um - kz * cm) + afc[2] * ky * vm + afc[3] * (ky * wm + kx * cm) +
              afc[4] * (ky * hc + (kx * wm - kz * um) * cm);
    afch[3] = aca * kz + afc[1] * (kz * um + ky * cm) + afc[2] * (kz * vm - kx * cm) + afc[3] * kz * wm +
              afc[4] * (kz * hc + (ky * um - kx * vm) * cm);
    afch[4] = aca + afc[1] * (um + kx * cm) + afc[2] * (vm + ky * cm) + afc[3] * (wm + kz * cm) + afc[4] * (hm + Ukb * cm);
    RoeBar r{};
    r.um = afc[1] * ca + afc[4] * cm * (-kz * fch[2] + ky * fch[3]);
    r.vm = afc[2] * ca + afc[4] * cm * (kz * fch[1] - kx * fch[3]);
    r.wm = afc[3] * ca + afc[4] * cm * (-ky * fch[1] + kx * fch[2]);
    r.cm = afc[1] * (-kx * fch[0] - kz * fch[2] + ky * fch[3] + kx * fch[4]) +
           afc[2] * (-ky * fch[0] + kz * fch[1] - kx * fch[3] + ky * fch[4]) +
           afc[3] * (-kz * fch[0] - ky * fch[1] + kx * fch[2] + kz * fch[4]) +
           afc[4] * (-Ukb * fch[0] + (kz * vm - ky * wm) * fch[1] + (kx * wm - kz * um) * fch[2] +
                     (ky * um - kx * vm) * fch[3] + Ukb * fch[4]);
    double a_hm = afc[4] * (fch[0] + fch[4]);
    const double a_hc = afc[4] * (kx * fch[1] + ky * fch[2] + kz * fch[3]);
    r.Ukb = afc[4] * cm * (fch[4] - fch[0]);
    a_hm += a_hc;
    a_cg -= a_hc;
    r.cm += a_cg * 2 * cm / gm1;
    r.gm1 -= a_cg * cg / gm1;
    // WENO and projection reverse per characteristic field; split-flux adjoints into shared memory
    for (int l = 0; l < nv; ++l) {
      double vp[7], vmn[7], gp[7], gm[7];
      project(l, vp, vmn);
      for (int m = 0; m < 7; ++m) gp[m] = gm[m] = 0.0;
      weno7_bwd(vp, vmn, eps, afch[l], gp, gm);
      if (l < 5) {
        double L[5], cs, AL[5];
        fvs_lrow(l, alpha, Ukb, cm, c2i, gm1, um, vm, wm, kx, ky, kz, L, cs);
        for (int q = 0; q < 5; ++q) {
          double s_ = 0;
          for (int m = 0; m < 7; ++m) {
            s_ += FP(m, q) * gp[m] + FM(m + 1, q) * gm[m];
            atomicAdd(AFP(m, q), L[q] * gp[m]);
            atomicAdd(AFM(m + 1, q), L[q] * gm[m]);
          }
          AL[q] = s_;
        }
        for (int q = 0; q < ns; ++q) {
          double s_ = 0;
          for (int m = 0; m < 7; ++m) {
            s_ += FP(m, 5 + q) * gp[m] + FM(m + 1, 5 + q) * gm[m];
            atomicAdd(AFP(m, 5 + q), cs * al[q] * gp[m]);
            atomicAdd(AFM(m + 1, 5 + q), cs * al[q] * gm[m]);
          }
          a_al[q] += cs * s_;
        }
        fvs_lrow_bwd(l, AL, alpha, Ukb, cm, c2i, gm1, um, vm, wm, kx, ky, kz, r);
      } else {
        double s_ = 0;
        for (int m = 0; m < 7; ++m) {
          s_ += FP(m, 0) * gp[m] + FM(m + 1, 0) * gm[m];
          atomicAdd(AFP(m, 0), -svm[l - 5] * gp[m]);
          atomicAdd(AFM(m + 1, 0), -svm[l - 5] * gm[m]);
          atomicAdd(AFP(m, l), gp[m]);
          atomicAdd(AFM(m + 1, l), gm[m]);
        }
        a_svm[l - 5] -= s_;
      }
    }
    // Roe symbols -> Roe averages
    r.gm1 += r.alpha * ekm;
    r.um += r.alpha * gm1 * um + r.Ukb * kx;
    r.vm += r.alpha * gm1 * vm + r.Ukb * ky;
    r.wm += r.alpha * gm1 * wm + r.Ukb * kz;
    double a_gamma = 0, a_tm = 0, a_mwinv = 0;
    double a_al_sum = 0;
    for (int l = 0; l < ns; ++l) {
      a_gamma += a_al[l] * kRuD / c_mix.mw[l] * tm * c2i;
      r.gm1 -= a_al[l] * hi[l] * c2i;
      a_tm += a_al[l] * gamma * kRuD / c_mix.mw[l] * c2i;
      a_al_sum += a_al[l] * al[l];
    }
    r.c2i += a_al_sum / c2i;
    r.cm -= 2.0 * r.c2i * c2i / cm;
    a_gamma += r.gm1;
    a_gamma += r.cm * cm / (2 * gamma);
    a_mwinv += r.cm * cm / (2 * mw_inv);
    a_tm += r.cm * cm / (2 * tm);
    const double a_cp = a_gamma / cvt, a_cvt = -a_gamma * gamma / cvt;
    double dcp[Spec<NS>::A];
    mix_dcp_dt<NS>(tm, dcp);
    for (int l = 0; l < ns; ++l) {
      a_svm[l] += a_cp * cpi[l] + a_cvt * (cpi[l] - c_mix.ru_mw[l]);
      const double a_cpi = (a_cp + a_cvt) * svm[l];
      const double a_hi = -a_al[l] * gm1 * c2i;
      a_tm += a_hi * cpi[l] + a_cpi * dcp[l];
    }
    const double a_prm = a_tm / (kRuD * mw_inv);
    a_mwinv -= a_tm * tm / mw_inv;
    for (int l = 0; l < ns; ++l) a_svm[l] += a_mwinv / c_mix.mw[l];
    // averages X = rlc X_l + rrc X_r of u, v, w, H, Y, p/rho; per side X = num / rho
    double a_rlc = 0, a_rrc = 0;
    double gl[Spec<NS>::A + 6], gr[Spec<NS>::A + 6];  // adjoints of cv[0..nv-1] and p, per side
    for (int l = 0; l <= nv; ++l) gl[l] = gr[l] = 0.0;
    auto avg = [&](double aX, double Xl, double Xr, int numl) {
      // numl: index of the numerator in cv (or nv for p); X = num / rho
      a_rlc += aX * Xl;
      a_rrc += aX * Xr;
      gl[numl] += aX * rlc * rli;
      gr[numl] += aX * rrc * rri;
      gl[0] -= aX * rlc * Xl * rli;
      gr[0] -= aX * rrc * Xr * rri;
    };
    avg(r.um, cvl[1] * rli, cvr[1] * rri, 1);
    avg(r.vm, cvl[2] * rli, cvr[2] * rri, 2);
    avg(r.wm, cvl[3] * rli, cvr[3] * rri, 3);
    avg(a_hm, (cvl[4] + p_l) * rli, (cvr[4] + p_r) * rri, 4);
    gl[nv] += a_hm * rlc * rli;  // H = (rho E + p) / rho
    gr[nv] += a_hm * rrc * rri;
    for (int l = 0; l < ns; ++l) avg(a_svm[l], cvl[5 + l] * rli, cvr[5 + l] * rri, 5 + l);
    avg(a_prm, p_l * rli, p_r * rri, nv);
    const double a_sl = (a_rlc - a_rrc) * sr / (den * den), a_sr = (a_rrc - a_rlc) * sl / (den * den);
    gl[0] += a_sl / (2 * sl);
    gr[0] += a_sr / (2 * sr);
    double *rl = aR + ((long long)(t + 3) * TXL + lane) * (nv + 1);
    double *rr = aR + ((long long)(t + 4) * TXL + lane) * (nv + 1);
    for (int l = 0; l <= nv; ++l) {
      atomicAdd(rl + l, gl[l]);
      atomicAdd(rr + l, gr[l]);
    }
  }
  __syncthreads();
  // staged nodes: split-flux and Roe adjoints -> node planes
  if (lane_ok) {
    for (int st = t; st < NST; st += TD) {
      const int nn = start - 4 + st;
      if (nn > nd + 3) continue;
      const long long p = pid(nn);
      double Q[Spec<NS>::A + 5], aQ[Spec<NS>::A + 5];
      const double *ra = aR + ((long long)st * TXL + lane) * (nv + 1);
      for (int l = 0; l < nv; ++l) {
        Q[l] = s.cv[l * P + p];
        aQ[l] = ra[l];
      }
      double ap = ra[nv], ac = 0.0;
      fvs_node_bwd(Q, s.bv[4 * P + p], s.acs[p], b.met[(DIR * 3 + 0) * P + p], b.met[(DIR * 3 + 1) * P + p],
                   b.met[(DIR * 3 + 2) * P + p], b.jac[p], aFp + ((long long)st * TXL + lane) * nv,
                   aFm + ((long long)st * TXL + lane) * nv, nv, aQ, ap, ac);
      for (int l = 0; l < nv; ++l)
        if (aQ[l] != 0.0) atomicAdd(A.cv + l * P + p, aQ[l]);
      if (ap != 0.0) atomicAdd(A.p + p, ap);
      if (ac != 0.0) atomicAdd(A.c + p, ac);
    }
  }
}

// Reverse of mix_visc_face (FP64) for the face between p0 and p0 + e[d] with face adjoint afv[nv]:
// adds to the adjoints of u, v, w, T, Y, mu, lambda and rho*D of the nodes its gradients read.
template <bool DIM3, int NS>
__device__ __forceinline__ void mix_visc_face_bwd(const DevBlock &b, const DevState &s, long long p0, int d,
                                                  const double *afv, const DevAdj &A) {
  const long long P = b.plane;
  const long long st[3] = {1, b.pitch, (long long)b.pitch * b.sy};
  const long long p1 = b.chk(p0 + st[d]);
  double m[9];
  for (int r = 0; r < 9; ++r) m[r] = 0.5 * (b.met[r * P + p0] + b.met[r * P + p1]);
  auto grad = [&](const double *B, double *out) {
    double g[3];
    for (int c = 0; c < 3; ++c) {
      if (c == d) {
        g[c] = B[p1] - B[p0];
      } else if (c == 2 && !DIM3) {
        g[c] = 0.0;
      } else {
        const long long a = st[c];
        g[c] = 0.25 * (B[p0 + a] - B[p0 - a] + B[p1 + a] - B[p1 - a]);
      }
    }
    out[0] = g[0] * m[0] + g[1] * m[3] + g[2] * m[6];
    out[1] = g[0] * m[1] + g[1] * m[4] + g[2] * m[7];
    out[2] = g[0] * m[2] + g[1] * m[5] + g[2] * m[8];
  };
  // reverse of grad: adjoint aout[3] of the metric-transformed gradient -> node adjoints of plane AB
  auto grad_bwd = [&](const double *aout, double *AB) {
    for (int c = 0; c < 3; ++c) {
      const double ag = aout[0] * m[c * 3 + 0] + aout[1] * m[c * 3 + 1] + aout[2] * m[c * 3 + 2];
      if (ag == 0.0) continue;
      if (c == d) {
        atomicAdd(AB + p1, ag);
        atomicAdd(AB + p0, -ag);
      } else if (c == 2 && !DIM3) {
      } else {
        const long long a = st[c];
        const double q = 0.25 * ag;
        atomicAdd(AB + p0 + a, q);
        atomicAdd(AB + p0 - a, -q);
        atomicAdd(AB + p1 + a, q);
        atomicAdd(AB + p1 - a, -q);
      }
    }
  };
  double gu[3], gv[3], gw[3], gt[3];
  grad(s.bv + P, gu);
  grad(s.bv + 2 * P, gv);
  grad(s.bv + 3 * P, gw);
  grad(s.bv + 5 * P, gt);
  const double mul = 0.5 * (s.mul[p0] + s.mul[p1]);
  const double txx = mul * (4 * gu[0] - 2 * gv[1] - 2 * gw[2]) / 3.0;
  const double tyy = mul * (4 * gv[1] - 2 * gu[0] - 2 * gw[2]) / 3.0;
  const double tzz = mul * (4 * gw[2] - 2 * gu[0] - 2 * gv[1]) / 3.0;
  const double txy = mul * (gu[1] + gv[0]);
  const double txz = mul * (gu[2] + gw[0]);
  const double tyz = mul * (gv[2] + gw[1]);
  const double j0 = b.jac[p0], j1 = b.jac[p1];
  const double nx = 0.5 * (b.met[(d * 3 + 0) * P + p0] * j0 + b.met[(d * 3 + 0) * P + p1] * j1);
  const double ny = 0.5 * (b.met[(d * 3 + 1) * P + p0] * j0 + b.met[(d * 3 + 1) * P + p1] * j1);
  const double nz = 0.5 * (b.met[(d * 3 + 2) * P + p0] * j0 + b.met[(d * 3 + 2) * P + p1] * j1);
  const double fv1 = nx * txx + ny * txy + nz * txz;
  const double fv2 = nx * txy + ny * tyy + nz * tyz;
  const double fv3 = nx * txz + ny * tyz + nz * tzz;
  const double um = 0.5 * (s.bv[P + p0] + s.bv[P + p1]);
  const double vm = 0.5 * (s.bv[2 * P + p0] + s.bv[2 * P + p1]);
  const double wm = 0.5 * (s.bv[3 * P + p0] + s.bv[3 * P + p1]);
  const double cond = 0.5 * (s.cond[p0] + s.cond[p1]);
  const int ns = OSTC_NS;
  double dif[Spec<NS>::A], yk[Spec<NS>::A], ddf[Spec<NS>::A];
  double sgw = 0, srdy = 0, corr = 0, mwt = 0;
  for (int l = 0; l < ns; ++l) {
    const double *Y = s.sv + (long long)l * P;
    yk[l] = 0.5 * (Y[p0] + Y[p1]);
    dif[l] = 0.5 * (s.rhod[l * P + p0] + s.rhod[l * P + p1]);
    double gy[3];
    grad(Y, gy);
    const double gdy = nx * gy[0] + ny * gy[1] + nz * gy[2];
    ddf[l] = gdy;
    corr += dif[l] * gdy;
    sgw += gdy / c_mix.mw[l];
    mwt += yk[l] / c_mix.mw[l];
    srdy += dif[l] * yk[l];
  }
  mwt = 1.0 / mwt;
  corr -= mwt * srdy * sgw;
  const double tf = 0.5 * (s.bv[5 * P + p0] + s.bv[5 * P + p1]);
  double h[Spec<NS>::A], cp[Spec<NS>::A];
  mix_h_cp<NS, double>(tf, h, cp);
  // ---- reverse
  const double a4 = afv[4];
  double a_tf = 0, a_corr = 0, a_sgw = 0, a_mwt = 0, a_srdy = 0;
  double a_yk[Spec<NS>::A], a_dif[Spec<NS>::A], a_gdy[Spec<NS>::A];
  for (int l = 0; l < ns; ++l) {
    const double flux = dif[l] * (ddf[l] - mwt * yk[l] * sgw) - yk[l] * corr;
    const double af = afv[5 + l] + a4 * h[l];
    a_tf += a4 * flux * cp[l];
    a_dif[l] = af * (ddf[l] - mwt * yk[l] * sgw);
    a_gdy[l] = af * dif[l];
    a_mwt -= af * dif[l] * yk[l] * sgw;
    a_yk[l] = -af * (dif[l] * mwt * sgw + corr);
    a_sgw -= af * dif[l] * mwt * yk[l];
    a_corr -= af * yk[l];
  }
  // corr = sum dif gdy - mwt srdy sgw
  for (int l = 0; l < ns; ++l) {
    a_dif[l] += a_corr * ddf[l];
    a_gdy[l] += a_corr * dif[l];
  }
  a_mwt -= a_corr * srdy * sgw;
  a_srdy -= a_corr * mwt * sgw;
  a_sgw -= a_corr * mwt * srdy;
  for (int l = 0; l < ns; ++l) {
    a_dif[l] += a_srdy * yk[l];
    a_yk[l] += a_srdy * dif[l] - a_mwt * mwt * mwt / c_mix.mw[l];
    a_gdy[l] += a_sgw / c_mix.mw[l];
    const double agy[3] = {a_gdy[l] * nx, a_gdy[l] * ny, a_gdy[l] * nz};
    grad_bwd(agy, A.Y + (long long)l * P);
    atomicAdd(A.Y + (long long)l * P + p0, 0.5 * a_yk[l]);
    atomicAdd(A.Y + (long long)l * P + p1, 0.5 * a_yk[l]);
    atomicAdd(A.rhod + (long long)l * P + p0, 0.5 * a_dif[l]);
    atomicAdd(A.rhod + (long long)l * P + p1, 0.5 * a_dif[l]);
  }
  atomicAdd(A.T + p0, 0.5 * a_tf);
  atomicAdd(A.T + p1, 0.5 * a_tf);
  // energy: fv4 = um fv1 + vm fv2 + wm fv3 + cond (n . gT) + sum h flux
  const double A1 = afv[1] + a4 * um, A2 = afv[2] + a4 * vm, A3 = afv[3] + a4 * wm;
  const double a_um = a4 * fv1, a_vm = a4 * fv2, a_wm = a4 * fv3;
  const double a_cond = a4 * (nx * gt[0] + ny * gt[1] + nz * gt[2]);
  const double agt[3] = {a4 * cond * nx, a4 * cond * ny, a4 * cond * nz};
  grad_bwd(agt, A.T);
  atomicAdd(A.lam + p0, 0.5 * a_cond);
  atomicAdd(A.lam + p1, 0.5 * a_cond);
  atomicAdd(A.vel + p0, 0.5 * a_um);
  atomicAdd(A.vel + p1, 0.5 * a_um);
  atomicAdd(A.vel + P + p0, 0.5 * a_vm);
  atomicAdd(A.vel + P + p1, 0.5 * a_vm);
  atomicAdd(A.vel + 2 * P + p0, 0.5 * a_wm);
  atomicAdd(A.vel + 2 * P + p1, 0.5 * a_wm);
  // stress
  const double a_txx = A1 * nx, a_tyy = A2 * ny, a_tzz = A3 * nz;
  const double a_txy = A1 * ny + A2 * nx, a_txz = A1 * nz + A3 * nx, a_tyz = A2 * nz + A3 * ny;
  const double a_mul = a_txx * (4 * gu[0] - 2 * gv[1] - 2 * gw[2]) / 3.0 +
                       a_tyy * (4 * gv[1] - 2 * gu[0] - 2 * gw[2]) / 3.0 +
                       a_tzz * (4 * gw[2] - 2 * gu[0] - 2 * gv[1]) / 3.0 + a_txy * (gu[1] + gv[0]) +
                       a_txz * (gu[2] + gw[0]) + a_tyz * (gv[2] + gw[1]);
  atomicAdd(A.mu + p0, 0.5 * a_mul);
  atomicAdd(A.mu + p1, 0.5 * a_mul);
  double agu[3], agv[3], agw[3];
  agu[0] = mul * (4 * a_txx - 2 * a_tyy - 2 * a_tzz) / 3.0;
  agv[1] = mul * (-2 * a_txx + 4 * a_tyy - 2 * a_tzz) / 3.0;
  agw[2] = mul * (-2 * a_txx - 2 * a_tyy + 4 * a_tzz) / 3.0;
  agu[1] = mul * a_txy;
  agv[0] = mul * a_txy;
  agu[2] = mul * a_txz;
  agw[0] = mul * a_txz;
  agv[2] = mul * a_tyz;
  agw[1] = mul * a_tyz;
  grad_bwd(agu, A.vel);
  grad_bwd(agv, A.vel + P);
  grad_bwd(agw, A.vel + 2 * P);
}

// Reverse of k_mix_visc: one thread per face; the face adjoint is dq_bar(n) - dq_bar(n + 1) over the
// nodes this tile owns (the forward adds fv(n + 1/2) to node n and subtracts it from node n + 1).
template <int DIR, bool DIM3, int NS>
__global__ void __launch_bounds__(FvsTile<DIR>::TD * FvsTile<DIR>::TXL, 3) k_adj_visc(DevBlock b, DevState s,
                                                                                    const double *__restrict__ dqb,
                                                                                    int nv, DevAdj A) {
  if (NS > 0) nv = 5 + NS;
  constexpr int TXL = FvsTile<DIR>::TXL, TD = FvsTile<DIR>::TD;
  const int lane = DIR == 0 ? 0 : (int)threadIdx.x;
  const int t = DIR == 0 ? (int)threadIdx.x : (int)threadIdx.y;
  const int nd = DIR == 0 ? b.mx : DIR == 1 ? b.my : b.mz;
  const int start = (DIR == 0 ? blockIdx.x : blockIdx.y) * (TD - 1);
  int i0, j0, k0;
  if (DIR == 0) {
    i0 = 0; j0 = blockIdx.y; k0 = blockIdx.z;
  } else if (DIR == 1) {
    i0 = blockIdx.x * TXL + lane; j0 = 0; k0 = blockIdx.z;
  } else {
    i0 = blockIdx.x * TXL + lane; j0 = blockIdx.z; k0 = 0;
  }
  const int n = start - 1 + t;
  if (!(i0 < b.mx && n < nd)) return;
  auto qid = [&](int m) -> long long {
    return DIR == 0 ? b.iq(m, j0, k0) : DIR == 1 ? b.iq(i0, m, k0) : b.iq(i0, j0, m);
  };
  double afv[Spec<NS>::A + 5];
  bool any = false;
  for (int l = 0; l < nv; ++l) {
    double a = 0.0;
    if (t >= 1) a += dqb[l * b.n + qid(n)];
    if (t <= TD - 2 && n + 1 < nd) a -= dqb[l * b.n + qid(n + 1)];
    afv[l] = a;
    any = any || a != 0.0;
  }
  if (!any) return;
  const long long p0 = DIR == 0 ? b.id(n, j0, k0) : DIR == 1 ? b.id(i0, n, k0) : b.id(i0, j0, n);
  mix_visc_face_bwd<DIM3, NS>(b, s, p0, DIR, afv, A);
}

// Reverse of the chemical source dq[5+l] += J omega_l(rho, T, Y) (compute_source<FR>,
// SourceTerm.cuh:11-35; finite_rate_chemistry, FiniteRateChem.cu:7-195), interior nodes.
// omega_l = 1e3 W_l sum_r (nu_b - nu_f)_rl (q1_r - q2_r), q1 = kf prod c^nu_f, q2 = kb prod c^nu_b,
// c_l = rho Y_l / W_l 1e-3: per reaction the adjoint of q1 - q2 goes to kf, kb and the
// concentrations; kf, kb are differentiated in T (and in the third-body sum) by Dual evaluations of
// the same rate-constant code.
template <int NS>
__global__ void __launch_bounds__(128, 4) k_adj_source(DevBlock b, DevState s, const double *__restrict__ dqb, DevAdj A) {
  const long long P = b.plane;
  const int ns = OSTC_NS, nr = c_mix.nr;
  constexpr int SA = Spec<NS>::A;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < b.n; n += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(n % b.mx);
    const long long r0 = n / b.mx;
    const int j = (int)(r0 % b.my), k = (int)(r0 / b.my);
    const long long p = b.id(i, j, k);
    double aw[SA];
    bool any = false;
    for (int l = 0; l < ns; ++l) {
      aw[l] = b.jac[p] * dqb[(5 + l) * b.n + n] * c_mix.mw[l] * 1e+3;
      any = any || aw[l] != 0.0;
    }
    if (!any) continue;
    const double rho = s.bv[p], t = s.bv[5 * P + p];
    double y[SA], c[SA], ac[SA];
    for (int l = 0; l < ns; ++l) {
      y[l] = s.sv[l * P + p];
      c[l] = rho * y[l] * c_mix.imw[l] * 1e-3;
      ac[l] = 0.0;
    }
    const double lt = log(t), ti = 1.0 / t;
    const Dual tT(t, 1.0), ltT = log(tT), tiT = 1.0 / tT;
    Dual gT[SA], gC[SA];
    if (c_mix.use_gibbs) {
      mix_gibbs_rt<NS, Dual>(tT, gT);
      for (int l = 0; l < ns; ++l) gC[l] = Dual(gT[l].v, 0.0);
    }
    double aT = 0;
    for (int r = 0; r < nr; ++r) {
      double aq = 0;
      for (int l = 0; l < ns; ++l) aq += aw[l] * (c_mix.stoi_b[r][l] - c_mix.stoi_f[r][l]);
      if (aq == 0.0) continue;
      const int ty = c_mix.label[r];
      double cc = 0;
      if (ty >= 4)
        for (int l = 0; l < ns; ++l) cc += c[l] * c_mix.third_body[r][l];
      Dual kf, kb;
      reaction_rates<NS, Dual>(r, tT, ltT, tiT, Dual(cc), gT, kf, kb);
      double dkf_dcc = 0, dkb_dcc = 0;
      if (ty >= 4) {
        Dual kfc, kbc;
        reaction_rates<NS, Dual>(r, Dual(t), Dual(lt), Dual(ti), Dual(cc, 1.0), gC, kfc, kbc);
        dkf_dcc = kfc.d;
        dkb_dcc = kbc.d;
      }
      // concentration products as the forward forms them, and their partial derivatives
      auto fpow = [](double x, int nu) { return nu == 1 ? x : (nu == 2 ? x * x : pow(x, (double)nu)); };
      auto dpow = [](double x, int nu) { return nu == 1 ? 1.0 : (nu == 2 ? 2 * x : nu * pow(x, (double)(nu - 1))); };
      double p1 = 1.0, p2 = 1.0;
      for (int l = 0; l < ns; ++l) {
        if (c_mix.stoi_f[r][l]) p1 *= fpow(c[l], c_mix.stoi_f[r][l]);
        if (c_mix.stoi_b[r][l]) p2 *= fpow(c[l], c_mix.stoi_b[r][l]);
      }
      const double akf = aq * p1, akb = ty != 0 ? -aq * p2 : 0.0;
      aT += akf * kf.d + akb * kb.d;
      if (ty >= 4) {
        const double acc = akf * dkf_dcc + akb * dkb_dcc;
        for (int l = 0; l < ns; ++l) ac[l] += acc * c_mix.third_body[r][l];
      }
      for (int l = 0; l < ns; ++l) {
        const int nf = c_mix.stoi_f[r][l], nb = ty != 0 ? c_mix.stoi_b[r][l] : 0;
        if (nf) {
          double d = dpow(c[l], nf);
          for (int m = 0; m < ns; ++m)
            if (m != l && c_mix.stoi_f[r][m]) d *= fpow(c[m], c_mix.stoi_f[r][m]);
          ac[l] += aq * kf.v * d;
        }
        if (nb) {
          double d = dpow(c[l], nb);
          for (int m = 0; m < ns; ++m)
            if (m != l && c_mix.stoi_b[r][m]) d *= fpow(c[m], c_mix.stoi_b[r][m]);
          ac[l] -= aq * kb.v * d;
        }
      }
    }
    double arho = 0;
    for (int l = 0; l < ns; ++l) {
      arho += ac[l] * y[l] * c_mix.imw[l] * 1e-3;
      A.Y[(long long)l * P + p] += ac[l] * rho * c_mix.imw[l] * 1e-3;
    }
    A.rho[p] += arho;
    A.T[p] += aT;
  }
}

// Reverse of the transport and acoustic properties (update_physical_properties<mixture>,
// FieldOperation.cuh:107-134, compute_transport_property, Transport.cu:43-136) at every padded node:
// adjoints of c, mu, lambda and rho*D_k -> adjoints of rho, p, T and Y.  Hand-written reverse of
// mix_properties (one forward sweep keeping its intermediates, then the reverse sweep).
template <int NS>
__global__ void __launch_bounds__(128, 4) k_adj_props(DevBlock b, DevState s, DevAdj A) {
  const long long P = b.plane;
  const int ns = OSTC_NS;
  constexpr int SA = Spec<NS>::A;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < P; p += (long long)gridDim.x * blockDim.x) {
    const double rho = s.bv[p];
    if (!(rho > 0)) continue;
    const double ac = A.c[p], amu = A.mu[p], alam = A.lam[p];
    double ard[SA];
    bool any = ac != 0.0 || amu != 0.0 || alam != 0.0;
    for (int l = 0; l < ns; ++l) {
      ard[l] = A.rhod[(long long)l * P + p];
      any = any || ard[l] != 0.0;
    }
    if (!any) continue;
    const double pr = s.bv[4 * P + p], t = s.bv[5 * P + p];
    double y[SA], cp[SA], dcp[SA];
    for (int l = 0; l < ns; ++l) y[l] = s.sv[l * P + p];
    mix_h_cp<NS, double>(t, nullptr, cp);
    mix_dcp_dt<NS>(t, dcp);
    // ---- forward (as mix_properties)
    double smw = 0, cpt = 0, cvt = 0;
    for (int l = 0; l < ns; ++l) {
      smw += y[l] * c_mix.imw[l];
      cpt += y[l] * cp[l];
      cvt += y[l] * (cp[l] - c_mix.ru_mw[l]);
    }
    const double mw = 1 / smw;
    const double gamma = cpt / cvt;
    const double acoustic = sqrt(gamma * kRuD * t / mw);
    double X[SA], vis[SA], dlvis[SA];  // dlvis = d ln(vis) / dT
    const double st = sqrt(t);
    for (int l = 0; l < ns; ++l) {
      X[l] = y[l] * mw * c_mix.imw[l];
      const double lj = c_mix.lj_potent_inv[l], tdl = t * lj;
      const double a1 = pow(tdl, -0.145), a2 = pow(tdl + 0.5, -2.0);
      const double ci = 1.147 * a1 + a2;
      vis[l] = c_mix.vis_coeff[l] * st / ci;
      const double dci = lj * (1.147 * -0.145 * a1 / tdl - 2.0 * a2 / (tdl + 0.5));
      dlvis[l] = 0.5 / t - dci / ci;
    }
    double vt[SA], ct[SA];
    for (int m = 0; m < ns; ++m) {
      double v_ = 0;
      for (int n = 0; n < ns; ++n) {
        double pf = 1.0;
        if (m != n) {
          const double nm = 1 + sqrt(vis[m] / vis[n]) * c_mix.wj_div_wi_1_4[m][n];
          pf = nm * nm * c_mix.sqrt_wiwj_8[m][n];
        }
        v_ += pf * X[n];
      }
      vt[m] = v_;
      ct[m] = 1.065 * v_ - 0.065 * X[m];
    }
    const double t32p = t * st / pr;
    const double eps = 1e-12;
    double num[SA], den[SA];
    for (int l = 0; l < ns; ++l) num[l] = den[l] = 0;
    for (int l = 0; l < ns; ++l)
      for (int n = l + 1; n < ns; ++n) {
        const double tr = t * c_mix.kb_over_eps[l][n];
        const double om = 1.0 / pow(tr, 0.145) + 1.0 / ((tr + 0.5) * (tr + 0.5));
        const double dln = c_mix.binary_diff[l][n] * t32p / om;
        num[l] += (X[n] + eps) * c_mix.mw[n];
        den[l] += (X[n] + eps) / dln;
        num[n] += (X[l] + eps) * c_mix.mw[l];
        den[n] += (X[l] + eps) / dln;
      }
    // ---- reverse
    double aX[SA], avis[SA], aY[SA], acp[SA], aden[SA], avt[SA];
    for (int l = 0; l < ns; ++l) aX[l] = avis[l] = aY[l] = acp[l] = 0.0;
    double arho = 0, aT = 0, ap = 0, amw = 0, at32p = 0;
    // rho D_l = rho num_l / (den_l mw)
    for (int l = 0; l < ns; ++l) {
      const double rd = rho * num[l] / (den[l] * mw);
      arho += ard[l] * rd / rho;
      const double anum = ard[l] * rd / num[l];
      aden[l] = -ard[l] * rd / den[l];
      amw -= ard[l] * rd / mw;
      for (int n = 0; n < ns; ++n)
        if (n != l) aX[n] += anum * c_mix.mw[n];
    }
    for (int l = 0; l < ns; ++l)
      for (int n = l + 1; n < ns; ++n) {
        const double kbe = c_mix.kb_over_eps[l][n], tr = t * kbe;
        const double a1 = pow(tr, 0.145), a2 = 1.0 / ((tr + 0.5) * (tr + 0.5));
        const double om = 1.0 / a1 + a2;
        const double bd = c_mix.binary_diff[l][n];
        const double dln = bd * t32p / om;
        const double idl = 1.0 / dln;
        aX[n] += aden[l] * idl;
        aX[l] += aden[n] * idl;
        const double adln = -(aden[l] * (X[n] + eps) + aden[n] * (X[l] + eps)) * idl * idl;
        at32p += adln * bd / om;
        const double aom = -adln * dln / om;
        // om = tr^-0.145 + (tr + 0.5)^-2
        aT += aom * kbe * (-0.145 / (a1 * tr) - 2.0 * a2 / (tr + 0.5));
      }
    // t32p = T^1.5 / p
    aT += at32p * 1.5 * t32p / t;
    ap -= at32p * t32p / pr;
    // lambda = sum lam_m X_m / ct_m, lam_m = vis_m (cp_m + 1.25 Ru / W_m); mu = sum vis_m X_m / vt_m
    for (int m = 0; m < ns; ++m) {
      const double lfac = cp[m] + 1.25 * c_mix.ru_mw[m];
      const double lamm = vis[m] * lfac;
      const double alm = alam * X[m] / ct[m];
      aX[m] += alam * lamm / ct[m];
      const double act = -alam * lamm * X[m] / (ct[m] * ct[m]);
      avt[m] = 1.065 * act;
      aX[m] -= 0.065 * act;
      avis[m] += alm * lfac;
      acp[m] += alm * vis[m];
      avis[m] += amu * X[m] / vt[m];
      aX[m] += amu * vis[m] / vt[m];
      avt[m] -= amu * vis[m] * X[m] / (vt[m] * vt[m]);
    }
    // vt_m = sum_n pf_mn X_n, pf_mn = (1 + sqrt(vis_m / vis_n) w_mn)^2 s_mn
    for (int m = 0; m < ns; ++m)
      for (int n = 0; n < ns; ++n) {
        if (m == n) {
          aX[n] += avt[m];
          continue;
        }
        const double r = sqrt(vis[m] / vis[n]), w = c_mix.wj_div_wi_1_4[m][n], sw = c_mix.sqrt_wiwj_8[m][n];
        const double nm = 1 + r * w;
        aX[n] += avt[m] * nm * nm * sw;
        const double ar = avt[m] * X[n] * 2 * nm * sw * w;
        avis[m] += ar * r / (2 * vis[m]);
        avis[n] -= ar * r / (2 * vis[n]);
      }
    for (int l = 0; l < ns; ++l) aT += avis[l] * vis[l] * dlvis[l];
    // c = sqrt(gamma Ru T / mw)
    const double agamma = ac * acoustic / (2 * gamma);
    aT += ac * acoustic / (2 * t);
    amw -= ac * acoustic / (2 * mw);
    // X_l = Y_l mw / W_l
    for (int l = 0; l < ns; ++l) {
      aY[l] += aX[l] * mw * c_mix.imw[l];
      amw += aX[l] * y[l] * c_mix.imw[l];
    }
    // gamma = cpt / cvt; mw = 1 / sum Y / W; cp_l(T)
    const double acpt = agamma / cvt, acvt = -agamma * gamma / cvt;
    for (int l = 0; l < ns; ++l) {
      aY[l] += acpt * cp[l] + acvt * (cp[l] - c_mix.ru_mw[l]) - amw * mw * mw * c_mix.imw[l];
      acp[l] += (acpt + acvt) * y[l];
      aT += acp[l] * dcp[l];
    }
    A.rho[p] += arho;
    A.p[p] += ap;
    A.T[p] += aT;
    for (int l = 0; l < ns; ++l) A.Y[(long long)l * P + p] += aY[l];
  }
}

// Ghost nodes hold copies of their source node's primitive state (bv, sv) and recompute their cv from
// it (compute_cv_from_bv_1_point<mixture>, FieldOperation.cuh:78-105): rho E = rho (sum h(T) Y +
// |V|^2 / 2) - p.  This moves a ghost's cv adjoint onto its primitive adjoints (rho, u, v, w, p, T, Y).
template <int NS>
__global__ void __launch_bounds__(128, 4) k_adj_ghost_cv(DevBlock b, DevState s, DevAdj A, int nv) {
  if (NS > 0) nv = 5 + NS;
  const long long P = b.plane;
  const int ns = OSTC_NS;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < P; p += (long long)gridDim.x * blockDim.x) {
    if (!(s.bv[p] > 0)) continue;
    const int i = (int)(p % b.pitch) - b.g;
    const long long r = p / b.pitch;
    const int j = (int)(r % b.sy) - b.g, k = (int)(r / b.sy) - b.gz;
    if (i >= 0 && i < b.mx && j >= 0 && j < b.my && k >= 0 && k < b.mz) continue;
    const double rho = s.bv[p], u = s.bv[P + p], v = s.bv[2 * P + p], w = s.bv[3 * P + p], t = s.bv[5 * P + p];
    double a[Spec<NS>::A + 5];
    bool any = false;
    for (int l = 0; l < nv; ++l) {
      a[l] = A.cv[l * P + p];
      any = any || a[l] != 0.0;
      A.cv[l * P + p] = 0.0;
    }
    if (!any) continue;
    double h[Spec<NS>::A], cp[Spec<NS>::A];
    mix_h_cp<NS, double>(t, h, cp);
    double hy = 0, cpy = 0;
    for (int l = 0; l < ns; ++l) {
      const double y = s.sv[l * P + p];
      hy += h[l] * y;
      cpy += cp[l] * y;
    }
    const double ek = 0.5 * (u * u + v * v + w * w);
    double arho = a[0] + a[1] * u + a[2] * v + a[3] * w + a[4] * (hy + ek);
    for (int l = 0; l < ns; ++l) {
      arho += a[5 + l] * s.sv[l * P + p];
      A.Y[(long long)l * P + p] += a[4] * rho * h[l] + a[5 + l] * rho;
    }
    A.rho[p] += arho;
    A.vel[p] += (a[1] + a[4] * u) * rho;
    A.vel[P + p] += (a[2] + a[4] * v) * rho;
    A.vel[2 * P + p] += (a[3] + a[4] * w) * rho;
    A.T[p] += a[4] * rho * cpy;
    A.p[p] -= a[4];
  }
}

// Interior nodes: primitive adjoints -> cv (and T) adjoints.  rho = cv0, u = cv1 / rho (v, w
// alike), Y_l = cv_{5+l} / rho, p = rho Ru T sum Y / W.  With exact_t the node's T is the root of
// e = cv4 / rho - |V|^2 / 2 = sum Y h(T) - Ru T sum Y / W (compute_temperature_and_pressure,
// FieldOperation.cu:3-40) and its adjoint goes to cv by the implicit-function derivative; otherwise
// T is a state variable of its own and its adjoint is left in A.T.
template <int NS>
__global__ void __launch_bounds__(128, 4) k_adj_eos(DevBlock b, DevState s, DevAdj A, int exact_t) {
  const long long P = b.plane;
  const int ns = OSTC_NS;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < b.n; n += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(n % b.mx);
    const long long r = n / b.mx;
    const int j = (int)(r % b.my), k = (int)(r / b.my);
    const long long p = b.id(i, j, k);
    const double rho = s.cv[p];
    const double t = s.bv[5 * P + p];
    const double irho = 1.0 / rho;
    const double u = s.cv[P + p] * irho, v = s.cv[2 * P + p] * irho, w = s.cv[3 * P + p] * irho;
    double y[Spec<NS>::A], ay[Spec<NS>::A];
    double gsum = 0;  // sum Y / W
    for (int l = 0; l < ns; ++l) {
      y[l] = s.cv[(5 + l) * P + p] * irho;
      ay[l] = A.Y[(long long)l * P + p];
      gsum += y[l] * c_mix.imw[l];
    }
    double arho = A.rho[p], aT = A.T[p];
    const double ap = A.p[p];
    double au = A.vel[p], av = A.vel[P + p], aw = A.vel[2 * P + p];
    // p = rho Ru T gsum
    arho += ap * kRuD * t * gsum;
    aT += ap * rho * kRuD * gsum;
    for (int l = 0; l < ns; ++l) ay[l] += ap * rho * kRuD * t * c_mix.imw[l];
    if (exact_t) {
      double h[Spec<NS>::A], cp[Spec<NS>::A];
      mix_h_cp<NS, double>(t, h, cp);
      double cvm = 0;
      for (int l = 0; l < ns; ++l) cvm += y[l] * (cp[l] - kRuD * c_mix.imw[l]);
      const double ae = aT / cvm;
      for (int l = 0; l < ns; ++l) ay[l] -= aT * (h[l] - kRuD * t * c_mix.imw[l]) / cvm;
      // e = cv4 / rho - (u^2 + v^2 + w^2) / 2
      A.cv[4 * P + p] += ae * irho;
      arho -= ae * s.cv[4 * P + p] * irho * irho;
      au -= ae * u;
      av -= ae * v;
      aw -= ae * w;
      aT = 0.0;
    }
    A.T[p] = aT;
    A.cv[P + p] += au * irho;
    A.cv[2 * P + p] += av * irho;
    A.cv[3 * P + p] += aw * irho;
    arho -= (au * u + av * v + aw * w) * irho;
    for (int l = 0; l < ns; ++l) {
      A.cv[(5 + l) * P + p] += ay[l] * irho;
      arho -= ay[l] * y[l] * irho;
    }
    A.cv[p] += arho;
  }
}

// Ghost fills in reverse (apply_outflow / apply_periodic, BoundCond.cuh:205-233, 1443-1486): each
// ghost node's primitive adjoints (rho, u, v, w, p, T, Y) move to the node it was copied from.  Faces
// run in the reverse of the forward order, so a ghost filled from another face's ghost passes its
// adjoint on in turn.
__global__ void __launch_bounds__(128) k_adj_bc_face(DevBlock b, DevAdj A, int ns, DevFace f) {
  const int t0 = f.face == 0 ? 1 : 0;
  const int t1 = f.face == 2 ? 1 : 2;
  const int n0 = f.re[t0] - f.rs[t0] + 1, n1 = f.re[t1] - f.rs[t1] + 1;
  const long long nn = (long long)n0 * n1;
  const long long P = b.plane;
  const long long st[3] = {1, b.pitch, (long long)b.pitch * b.sy};
  int dir[3] = {0, 0, 0};
  dir[f.face] = f.direction;
  const long long dstep = dir[0] * st[0] + dir[1] * st[1] + dir[2] * st[2];
  double *planes[6] = {A.rho, A.vel, A.vel + P, A.vel + 2 * P, A.p, A.T};
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < nn; n += (long long)gridDim.x * blockDim.x) {
    int idx[3];
    idx[f.face] = f.rs[f.face];
    idx[t0] = f.rs[t0] + (int)(n % n0);
    idx[t1] = f.rs[t1] + (int)(n / n0);
    const long long pb = b.id(idx[0], idx[1], idx[2]);
    long long po = pb;
    if (f.type == kPeriodic) {
      const int ext[3] = {b.mx, b.my, b.mz};
      int other[3] = {idx[0], idx[1], idx[2]};
      other[f.face] = f.direction < 0 ? ext[f.face] - 1 : 0;
      po = b.id(other[0], other[1], other[2]);
    }
    for (int g = b.g; g >= 1; --g) {
      const long long pg = b.chk(pb + g * dstep);
      const long long ps = b.chk(f.type == kPeriodic ? po + g * dstep : pb);
      for (int q = 0; q < 6; ++q) {
        planes[q][ps] += planes[q][pg];
        planes[q][pg] = 0.0;
      }
      for (int l = 0; l < ns; ++l) {
        A.Y[l * P + ps] += A.Y[l * P + pg];
        A.Y[l * P + pg] = 0.0;
      }
    }
  }
}

// Reverse of the stage's temperature Newton iteration (update_cv_and_bv_rk + compute_temperature_and_
// pressure, RK.cuh:230-284, FieldOperation.cu:3-40): T_out = N(T_start; e, Y) of the stage output's
// cv, started from the stage input's T, iterated to the reference's relative tolerance 1e-3.  The
// iterate (not the exact root) is differentiated, by Dual evaluations seeded on e, each Y and the
// start T: lam_cv += (dT_out / d cv_out)^T lam_t, lam_t_start += dT_out / dT_start * lam_t.
template <int NS>
__global__ void __launch_bounds__(128, 4) k_adj_newton(DevBlock b, DevState in, DevState out, const double *lam_t,
                                                    double *lam_cv, double *lam_t_start) {
  const long long P = b.plane;
  const int ns = OSTC_NS;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < b.n; n += (long long)gridDim.x * blockDim.x) {
    const double lt = lam_t[n];
    if (lt == 0.0) continue;
    const int i = (int)(n % b.mx);
    const long long r = n / b.mx;
    const int j = (int)(r % b.my), k = (int)(r / b.my);
    const long long p = b.id(i, j, k);
    const double rho = out.cv[p], irho = 1.0 / rho;
    const double u = out.cv[P + p] * irho, v = out.cv[2 * P + p] * irho, w = out.cv[3 * P + p] * irho;
    const double e = out.cv[4 * P + p] / rho - 0.5 * (u * u + v * v + w * w);
    const double t0 = in.bv[5 * P + p];
    double yv[Spec<NS>::A];
    for (int l = 0; l < ns; ++l) yv[l] = out.cv[(5 + l) * P + p] * irho;
    double de = 0, dts = 0, dy[Spec<NS>::A];
    for (int in_ = 0; in_ < ns + 2; ++in_) {
      Dual y[Spec<NS>::A], pr;
      for (int l = 0; l < ns; ++l) y[l] = Dual(yv[l], in_ == 2 + l ? 1.0 : 0.0);
      const Dual t = mix_temperature<NS, Dual>(Dual(rho), Dual(e, in_ == 0 ? 1.0 : 0.0), Dual(t0, in_ == 1 ? 1.0 : 0.0),
                                               y, pr);
      if (in_ == 0) de = t.d;
      else if (in_ == 1) dts = t.d;
      else dy[in_ - 2] = t.d;
    }
    lam_t_start[n] += dts * lt;
    // e = cv4 / rho - |V|^2 / 2, Y = cv_{5+l} / rho
    const double ae = de * lt;
    double arho = -ae * out.cv[4 * P + p] * irho * irho + ae * (u * u + v * v + w * w) * irho;
    lam_cv[4 * b.n + n] += ae * irho;
    lam_cv[b.n + n] -= ae * u * irho;
    lam_cv[2 * b.n + n] -= ae * v * irho;
    lam_cv[3 * b.n + n] -= ae * w * irho;
    for (int l = 0; l < ns; ++l) {
      const double ay = dy[l] * lt;
      lam_cv[(5 + l) * b.n + n] += ay * irho;
      arho -= ay * yv[l] * irho;
    }
    lam_cv[n] += arho;
  }
}

// interior part of nv adjoint planes, in the layout of dq
__global__ void k_adj_gather(DevBlock b, const double *__restrict__ Acv, int nv, double *__restrict__ out) {
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < b.n; n += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(n % b.mx);
    const long long r = n / b.mx;
    const int j = (int)(r % b.my), k = (int)(r / b.my);
    const long long p = b.id(i, j, k);
    for (int l = 0; l < nv; ++l) out[l * b.n + n] = Acv[l * b.plane + p];
  }
}

// Seed of a stage's right-hand-side adjoint: dqb = c dt / J * lam (the stage adds c dt / J * dq to
// cv, update_cv_and_bv_rk, RK.cuh:230-284).  2-D blocks zero component 3 of lam in place first: the
// stage output's rho*w is set to 0, so its adjoint never reaches the stage's inputs.
__global__ void k_adj_stage_seed(DevBlock b, double *lam, double c, const double *dtp, double *dqb, int nv) {
  const double dt = *dtp;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < b.n; n += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(n % b.mx);
    const long long r = n / b.mx;
    const int j = (int)(r % b.my), k = (int)(r / b.my);
    const double f = c * dt / b.jac[b.id(i, j, k)];
    if (b.mz == 1) lam[3 * b.n + n] = 0.0;
    for (int l = 0; l < nv; ++l) dqb[l * b.n + n] = f * lam[l * b.n + n];
  }
}

// y = a x + c y over n values
__global__ void k_axpby(long long n, double a, const double *__restrict__ x, double c, double *__restrict__ y) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    y[i] = a * x[i] + c * y[i];
}

// lam_cv += (dT / dcv)^T lam_t for T the equation-of-state root of the node's cv (implicit-function
// derivative of sum Y h(T) - Ru T sum Y / W = cv4 / rho - |V|^2 / 2), interior nodes
template <int NS>
__global__ void __launch_bounds__(128) k_adj_t_to_cv(DevBlock b, DevState s, const double *lam_t, double *lam_cv) {
  const long long P = b.plane;
  const int ns = OSTC_NS;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < b.n; n += (long long)gridDim.x * blockDim.x) {
    const double lt = lam_t[n];
    if (lt == 0.0) continue;
    const int i = (int)(n % b.mx);
    const long long r = n / b.mx;
    const int j = (int)(r % b.my), k = (int)(r / b.my);
    const long long p = b.id(i, j, k);
    const double rho = s.cv[p], irho = 1.0 / rho, t = s.bv[5 * P + p];
    const double u = s.cv[P + p] * irho, v = s.cv[2 * P + p] * irho, w = s.cv[3 * P + p] * irho;
    double y[Spec<NS>::A], h[Spec<NS>::A], cp[Spec<NS>::A];
    mix_h_cp<NS, double>(t, h, cp);
    double cvm = 0;
    for (int l = 0; l < ns; ++l) {
      y[l] = s.cv[(5 + l) * P + p] * irho;
      cvm += y[l] * (cp[l] - kRuD * c_mix.imw[l]);
    }
    const double ae = lt / cvm;
    double arho = -ae * s.cv[4 * P + p] * irho * irho + ae * (u * u + v * v + w * w) * irho;
    lam_cv[4 * b.n + n] += ae * irho;
    lam_cv[b.n + n] -= ae * u * irho;
    lam_cv[2 * b.n + n] -= ae * v * irho;
    lam_cv[3 * b.n + n] -= ae * w * irho;
    for (int l = 0; l < ns; ++l) {
      const double ay = -lt * (h[l] - kRuD * t * c_mix.imw[l]) / cvm;
      lam_cv[(5 + l) * b.n + n] += ay * irho;
      arho -= ay * y[l] * irho;
    }
    lam_cv[n] += arho;
  }
}

}  // namespace ostc
