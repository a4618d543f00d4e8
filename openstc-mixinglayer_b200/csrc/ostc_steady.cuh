// ostc_steady.cuh -- the reference's steady driver (steady_simulation, SteadySim.cuh:15-140) on the
// device: per-node local time steps, the point-implicit chemical source (EPI / diagonal approximation,
// FiniteRateChem.cu:197-254, 414-426) and the DPLUR implicit operator (DPLUR.cuh:14-327, DPLUR.cu:5-40).
// Included by ostc_b200.cu after the air and mixture kernels; the host side is ostc_steady_step there.
//
// Layout: every per-node array of this driver is interior-indexed like dq (node n = (k*my + j)*mx + i):
// dt_local[n], the inviscid spectral radii srad[d*N + n] (d = 0..2), the chemical source Jacobian
// cj[e*N + n] (e = m*ns + q for the full matrix, e = l for its diagonal), and the DPLUR iterates
// dq0 / dqk [l*N + n].  One thread per node; the arrays are SoA so that every access is coalesced.
#pragma once

namespace ostc {

// local_time_step<mix, Laminar> (TimeAdvanceFunc.cuh:28-83): the CFL step of every node and its three
// inviscid spectral radii (the third zero in 2-D), the expressions of k_cfl_dt.
__global__ void __launch_bounds__(256) k_local_dt(DevBlock b, DevState s, double cfl, double prandtl, int dim3,
                                                  double *__restrict__ dtl, double *__restrict__ srad) {
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
    dtl[n] = cfl / (sinv + sv);
    srad[n] = s0;
    srad[b.n + n] = s1;
    srad[2 * b.n + n] = s2;
  }
}

// compute_source<FR> of the steady driver (FiniteRateChem.cu:7-58): dq starts from the chemical
// source (flow part zero), and with chemSrcMethod 1 the source Jacobian (compute_chem_src_jacobian,
// :197-217) or with 2 its diagonal approximation -omega_d,k / (rho Y_k) (:219-231) is stored in cj.
template <int NS>
__global__ void __launch_bounds__(128, 4) k_mix_source_jac(DevBlock b, DevState s, double *__restrict__ dq,
                                                         int method, double *__restrict__ cj) {
  const long long P = b.plane;
  const int ns = OSTC_NS;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < b.n; n += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(n % b.mx);
    const long long r = n / b.mx;
    const int j = (int)(r % b.my), k = (int)(r / b.my);
    const long long p = b.id(i, j, k);
    for (int l = 0; l < 5; ++l) dq[l * b.n + n] = 0.0;
    double y[Spec<NS>::A], om[Spec<NS>::A], od[Spec<NS>::A];
    for (int l = 0; l < ns; ++l) y[l] = s.sv[l * P + p];
    const double rho = s.bv[p];
    if (method == 1) {
      double jc[Spec<NS>::A * Spec<NS>::A];
      for (int l = 0; l < ns * ns; ++l) jc[l] = 0.0;
      mix_chemistry<NS>(rho, s.bv[5 * P + p], y, om, jc);
      for (int l = 0; l < ns * ns; ++l) cj[l * b.n + n] = jc[l];
    } else {
      mix_chemistry<NS>(rho, s.bv[5 * P + p], y, om, (double *)nullptr, od);
      for (int l = 0; l < ns; ++l) cj[l * b.n + n] = y[l] > 1e-25 ? -od[l] / (y[l] * rho) : 0.0;
    }
    const double jac = b.jac[p];
    for (int l = 0; l < ns; ++l) dq[(5 + l) * b.n + n] = jac * om[l];
  }
}

// (diag I - dt J) x = rhs for the species of node n (EPI, EPI_for_dq0, EPI_for_dqk:
// FiniteRateChem.cu:233-300), rhs solved in place by the column-pivoted LU of solve_chem_system.
template <int NS>
__device__ __forceinline__ void epi_solve(const double *__restrict__ cj, long long N, long long n, double diag,
                                          double dt, double *rhs) {
  const int ns = OSTC_NS;
  double lhs[Spec<NS>::A * Spec<NS>::A];
  for (int m = 0; m < ns; ++m)
    for (int q = 0; q < ns; ++q) {
      const double jm = cj[(m * ns + q) * N + n];
      lhs[m * ns + q] = m == q ? diag - dt * jm : -dt * jm;
    }
  mix_lu_solve<NS>(lhs, rhs);
}

// implicit_treatment with implicit_method 0 (ImplicitTreatmentHPP.cuh:12-27): the species part of dq
// replaced by EPI (method 1, lhs I - dt_local J) or divided by 1 - dt_local J_kk (DA, method 2).
template <int NS>
__global__ void __launch_bounds__(128, 4) k_point_implicit(DevBlock b, double *__restrict__ dq,
                                                         const double *__restrict__ dtl,
                                                         const double *__restrict__ cj, int method) {
  const int ns = OSTC_NS;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < b.n; n += (long long)gridDim.x * blockDim.x) {
    const double dt = dtl[n];
    if (method == 1) {
      double rhs[Spec<NS>::A];
      for (int l = 0; l < ns; ++l) rhs[l] = dq[(5 + l) * b.n + n];
      epi_solve<NS>(cj, b.n, n, 1.0, dt, rhs);
      for (int l = 0; l < ns; ++l) dq[(5 + l) * b.n + n] = rhs[l];
    } else {
      for (int l = 0; l < ns; ++l) dq[(5 + l) * b.n + n] /= 1 - dt * cj[l * b.n + n];
    }
  }
}

// Arguments of the DPLUR kernels.  chem: 0 no finite-rate chemistry (every variable on the scalar
// diagonal), else the chemSrcMethod of the species rows (0 explicit, 1 EPI, 2 DA) plus one.
struct DplurArgs {
  const double *dtl, *srad, *cj;
  double *dq, *dq0, *dqk;
  int nv, chem;
  double diag_factor;  // 0 for the steady driver, 1.5 / dt for dual time stepping
};

// compute_DQ_0 (DPLUR.cuh:14-92): dq <- dt dq / diag, diag = 1 + diag_factor dt + dt (sum of the
// inviscid spectral radii).  The reference adds 2 dt times a viscous spectral radius that it never computes (its array
// keeps the zeros of its allocation, Field.cu:553-565): that term is zero and left out.
template <int NS>
__global__ void __launch_bounds__(128) k_dplur_dq0(DevBlock b, DplurArgs a) {
  const int ns = OSTC_NS;
  const int nv = NS > 0 ? 5 + NS : a.nv;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < b.n; n += (long long)gridDim.x * blockDim.x) {
    const double dt = a.dtl[n];
    for (int l = 0; l < nv; ++l) a.dq[l * b.n + n] *= dt;
    const double diag = 1 + a.diag_factor * dt + dt * (a.srad[n] + a.srad[b.n + n] + a.srad[2 * b.n + n]);
    const int nflow = a.chem ? 5 : nv;
    for (int l = 0; l < nflow; ++l) a.dq[l * b.n + n] /= diag;
    if (!a.chem) continue;
    if (a.chem == 2) {
      double rhs[Spec<NS>::A];
      for (int l = 0; l < ns; ++l) rhs[l] = a.dq[(5 + l) * b.n + n];
      epi_solve<NS>(a.cj, b.n, n, diag, dt, rhs);
      for (int l = 0; l < ns; ++l) a.dq[(5 + l) * b.n + n] = rhs[l];
    } else if (a.chem == 3) {
      for (int l = 0; l < ns; ++l) a.dq[(5 + l) * b.n + n] /= diag - dt * a.cj[l * b.n + n];
    } else {
      for (int l = 0; l < ns; ++l) a.dq[(5 + l) * b.n + n] /= diag;
    }
  }
}

// compute_jacobian_times_dq (DPLUR.cuh:96-154): the convective flux Jacobian of direction dir, shifted by
// lam, at interior node (i, j, k) times that node's dq.
template <int NS>
__device__ __forceinline__ void jac_times_dq(const DevBlock &b, const DevState &s, const double *__restrict__ dq,
                                             int nv, int i, int j, int k, int dir, double lam, double *out) {
  const long long P = b.plane;
  const long long p = b.id(i, j, k), q = b.iq(i, j, k);
  const double xi_x = b.met[(dir * 3) * P + p], xi_y = b.met[(dir * 3 + 1) * P + p], xi_z = b.met[(dir * 3 + 2) * P + p];
  const double u = s.bv[P + p], v = s.bv[2 * P + p], w = s.bv[3 * P + p];
  const double U = xi_x * u + xi_y * v + xi_z * w;
  const double lmd1 = U + lam;
  const double e = 0.5 * (u * u + v * v + w * w);
  double gamma = kGamma, b3 = 0, b4 = 0, h = 0;
  double d[5 + Spec<NS>::A];
  for (int l = 0; l < nv; ++l) d[l] = dq[l * b.n + q];
  if (!s.sv) {
    h = gamma / (gamma - 1) * s.bv[4 * P + p] / s.bv[p] + e;
  } else {
    const int ns = OSTC_NS;
    double hs[Spec<NS>::A];
    const double t = s.bv[5 * P + p];
    mix_h_cp<NS>(t, hs, (double *)nullptr);
    gamma = s.gam[p];
    for (int l = 0; l < ns; ++l) {
      b3 += kRuD * t / c_mix.mw[l] * d[5 + l];
      b4 += hs[l] * d[5 + l];
      h += s.sv[l * P + p] * hs[l];
    }
    b3 *= gamma;
    b4 *= gamma - 1;
    h += e;
  }
  const double b1 = xi_x * d[1] + xi_y * d[2] + xi_z * d[3] - U * d[0];
  const double b2 = (gamma - 1) * (e * d[0] - u * d[1] - v * d[2] - w * d[3] + d[4]);
  out[0] = b1 + lmd1 * d[0];
  out[1] = u * b1 + xi_x * b2 + lmd1 * d[1] + xi_x * (b3 - b4);
  out[2] = v * b1 + xi_y * b2 + lmd1 * d[2] + xi_y * (b3 - b4);
  out[3] = w * b1 + xi_z * b2 + lmd1 * d[3] + xi_z * (b3 - b4);
  out[4] = h * b1 + U * b2 + lmd1 * d[4] + U * (b3 - b4);
  for (int l = 5; l < nv; ++l) out[l] = lmd1 * d[l] + s.sv[(l - 5) * P + p] * b1;
}

// DPLUR_inner_iteration (DPLUR.cuh:156-268): dqk = dq0 + dt (sum of the neighbours' half Jacobian
// products, lower neighbours added, upper ones subtracted) / diag, the species rows through the
// chemistry treatment.  Neighbours outside the block contribute nothing (the reference reads only
// interior neighbours: its dq ghost layer is never filled on a single block).
template <int NS>
__global__ void __launch_bounds__(128) k_dplur_inner(DevBlock b, DevState s, DplurArgs a) {
  const int ns = OSTC_NS;
  const int nv = NS > 0 ? 5 + NS : a.nv;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < b.n; n += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(n % b.mx);
    const long long r = n / b.mx;
    const int j = (int)(r % b.my), k = (int)(r / b.my);
    double conv[5 + Spec<NS>::A], tot[5 + Spec<NS>::A];
    for (int l = 0; l < nv; ++l) tot[l] = 0.0;
    const int at[3] = {i, j, k}, ext[3] = {b.mx, b.my, b.mz};
    for (int d = 0; d < 3; ++d) {
      if (at[d] > 0) {
        const int ii = i - (d == 0), jj = j - (d == 1), kk = k - (d == 2);
        const long long qn = b.iq(ii, jj, kk);
        jac_times_dq<NS>(b, s, a.dq, nv, ii, jj, kk, d, a.srad[d * b.n + qn], conv);
        for (int l = 0; l < nv; ++l) tot[l] += 0.5 * conv[l];
      }
    }
    for (int d = 0; d < 3; ++d) {
      if (at[d] != ext[d] - 1) {
        const int ii = i + (d == 0), jj = j + (d == 1), kk = k + (d == 2);
        const long long qn = b.iq(ii, jj, kk);
        jac_times_dq<NS>(b, s, a.dq, nv, ii, jj, kk, d, -a.srad[d * b.n + qn], conv);
        for (int l = 0; l < nv; ++l) tot[l] -= 0.5 * conv[l];
      }
    }
    const double dt = a.dtl[n];
    const double diag = 1 + a.diag_factor * dt + dt * (a.srad[n] + a.srad[b.n + n] + a.srad[2 * b.n + n]);
    const int nflow = a.chem ? 5 : nv;
    for (int l = 0; l < nflow; ++l) a.dqk[l * b.n + n] = a.dq0[l * b.n + n] + dt * tot[l] / diag;
    if (!a.chem) continue;
    if (a.chem == 2) {
      double rhs[Spec<NS>::A];
      for (int l = 0; l < ns; ++l) rhs[l] = tot[5 + l] * dt;
      epi_solve<NS>(a.cj, b.n, n, diag, dt, rhs);
      for (int l = 0; l < ns; ++l) a.dqk[(5 + l) * b.n + n] = a.dq0[(5 + l) * b.n + n] + rhs[l];
    } else if (a.chem == 3) {
      for (int l = 0; l < ns; ++l)
        a.dqk[(5 + l) * b.n + n] = a.dq0[(5 + l) * b.n + n] + dt * tot[5 + l] / (diag - dt * a.cj[l * b.n + n]);
    } else {
      for (int l = 0; l < ns; ++l) a.dqk[(5 + l) * b.n + n] = a.dq0[(5 + l) * b.n + n] + dt * tot[5 + l] / diag;
    }
  }
}

// set_dq_to_0 on a wall face (DPLUR.cu:22-40), over the face's interior nodes.  The reference pads the
// face's tangential range by ngg (Mesh.cpp:14-32) while its DPLUR dq carries one ghost layer, so its
// padded part writes outside that layer; here only the nodes of the block are zeroed.
__global__ void k_wall_dq_zero(DevBlock b, DevFace f, double *__restrict__ dq, int nv) {
  const int fi = f.face;
  const int at = f.direction < 0 ? 0 : (fi == 0 ? b.mx - 1 : fi == 1 ? b.my - 1 : b.mz - 1);
  const int e0 = fi == 0 ? b.my : b.mx, e1 = fi == 2 ? b.my : b.mz;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < (long long)e0 * e1;
       t += (long long)gridDim.x * blockDim.x) {
    const int a0 = (int)(t % e0), a1 = (int)(t / e0);
    const int i = fi == 0 ? at : a0, j = fi == 1 ? at : (fi == 0 ? a0 : a1), k = fi == 2 ? at : a1;
    const long long q = b.iq(i, j, k);
    for (int l = 0; l < nv; ++l) dq[l * b.n + q] = 0.0;
  }
}

// convert_dq_back_to_dqDt (DPLUR.cu:5-17)
__global__ void k_dplur_back(DevBlock b, double *__restrict__ dq, const double *__restrict__ dtl, int nv) {
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < b.n; n += (long long)gridDim.x * blockDim.x) {
    const double dt = dtl[n];
    for (int l = 0; l < nv; ++l) dq[l * b.n + n] /= dt;
  }
}

// compute_qn_star (DualTimeStepping.cu:3-14): q* = jac / (2 dt) (4 cv^n - cv^(n-1)) of every interior
// node, from the current state and the previous physical step's conservative state qn1 (padded planes).
__global__ void k_qn_star(DevBlock b, DevState s, const double *__restrict__ qn1, double *__restrict__ qstar,
                          int nv, double dt) {
  const long long P = b.plane;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < b.n; n += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(n % b.mx);
    const long long r = n / b.mx;
    const int j = (int)(r % b.my), k = (int)(r / b.my);
    const long long p = b.id(i, j, k);
    const double factor = 0.5 * b.jac[p] / dt;
    for (int l = 0; l < nv; ++l) qstar[l * b.n + n] = factor * (4 * s.cv[l * P + p] - qn1[l * P + p]);
  }
}

// compute_modified_rhs (DualTimeStepping.cu:16-30): dq += q* - 1.5 jac / dt cv.
__global__ void k_modified_rhs(DevBlock b, DevState s, const double *__restrict__ qstar, double *__restrict__ dq,
                               int nv, double dt) {
  const long long P = b.plane;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < b.n; n += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(n % b.mx);
    const long long r = n / b.mx;
    const int j = (int)(r % b.my), k = (int)(r / b.my);
    const long long p = b.id(i, j, k);
    const double factor = 1.5 * b.jac[p] / dt;
    for (int l = 0; l < nv; ++l) dq[l * b.n + n] += qstar[l * b.n + n] - factor * s.cv[l * P + p];
  }
}

// update_cv_and_bv<Air> (FieldOperation.cuh:189-232) in place, with the Sutherland viscosity of the
// new state (update_physical_properties<Air>, FieldOperation.cuh:107-140, for the interior nodes).
__global__ void __launch_bounds__(256) k_steady_update_air(DevBlock b, DevState s, const double *__restrict__ dq,
                                                           const double *__restrict__ dtl, unsigned *flags) {
  const long long P = b.plane;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < b.n; n += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(n % b.mx);
    const long long r = n / b.mx;
    const int j = (int)(r % b.my), k = (int)(r / b.my);
    const long long p = b.id(i, j, k);
    const double dtj = dtl[n] / b.jac[p];
    double cv[5];
#pragma unroll
    for (int l = 0; l < 5; ++l) cv[l] = s.cv[l * P + p] + dtj * dq[l * b.n + n];
    if (b.mz == 1) cv[3] = 0;
#pragma unroll
    for (int l = 0; l < 5; ++l) s.cv[l * P + p] = cv[l];
    const double rho = cv[0];
    const double di = 1.0 / rho;
    const double u = cv[1] * di, v = cv[2] * di, w = cv[3] * di;
    const double V2 = u * u + v * v + w * w;
    const double pr = (kGamma - 1) * (cv[4] - 0.5 * rho * V2);
    const double tt = pr * kMwD * di / kRuD;
    s.bv[p] = rho;
    s.bv[P + p] = u;
    s.bv[2 * P + p] = v;
    s.bv[3 * P + p] = w;
    s.bv[4 * P + p] = pr;
    s.bv[5 * P + p] = tt;
    s.mul[p] = sutherland(tt);
    if (!(rho > 0.0) || !(pr > 0.0) || !(tt > 0.0)) atomicOr(flags, (unsigned)OSTC_FLAG_NONPOSITIVE);
    if (isnan(cv[0]) || isnan(cv[1]) || isnan(cv[2]) || isnan(cv[3]) || isnan(cv[4]))
      atomicOr(flags, (unsigned)OSTC_FLAG_NAN);
  }
}

}  // namespace ostc
