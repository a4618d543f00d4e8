// mix_math.cuh -- device arithmetic of the multi-component (species = 1) path: NASA-7 thermodynamics,
// mixture transport, the temperature Newton iteration, finite-rate chemistry and the flux-split
// characteristic WENO7-Z face flux.  The species and reaction tables sit in constant memory: every
// thread of a warp reads the same coefficient at the same time, which the constant cache broadcasts.
#pragma once

#include "air_math.cuh"

namespace ostc {

constexpr int kMS = 16;  // species capacity of the device tables
constexpr int kMR = 64;  // reaction capacity
constexpr int kMV = 5 + kMS;
constexpr double kPatmD = 101325.0;

// Species count as a compile-time constant: NS > 0 instantiates for exactly NS species (arrays in
// registers, loops unrolled); NS = 0 is the generic build that reads the count from the tables.
template <int NS> struct Spec {
  static constexpr int A = NS > 0 ? NS : kMS;  // array extent
};
#define OSTC_NS (NS > 0 ? NS : c_mix.ns)

template <typename T> __device__ __forceinline__ T tpow(T x, T y);
template <> __device__ __forceinline__ double tpow<double>(double x, double y) { return pow(x, y); }
template <> __device__ __forceinline__ float tpow<float>(float x, float y) { return powf(x, y); }
}  // namespace ostc
#include "dual.cuh"
namespace ostc {

struct MixTables {
  int ns, nr;
  int use_gibbs;  // some reaction takes kb from the equilibrium constant (backward_reaction_rate's n_gibbs)
  double weno_eps_scale, v_ref;
  double mw[kMS], imw[kMS], ru_mw[kMS], t_low[kMS], t_mid[kMS];
  double low[kMS][7], high[kMS][7];
  double lj_potent_inv[kMS], vis_coeff[kMS];
  double wj_div_wi_1_4[kMS][kMS], sqrt_wiwj_8[kMS][kMS], binary_diff[kMS][kMS], kb_over_eps[kMS][kMS];
  // ln of lj_potent_inv and of kb_over_eps: the reduced temperatures' powers T*^a = exp(a (ln T + ln c))
  // then take one log per node instead of one pow per species / species pair
  double ln_lj[kMS], ln_kbe[kMS][kMS];
  int label[kMR], rev_type[kMR], order[kMR];
  signed char stoi_f[kMR][kMS], stoi_b[kMR][kMS];
  double A[kMR], b[kMR], Ea[kMR], A2[kMR], b2[kMR], Ea2[kMR], third_body[kMR][kMS];
  double troe_alpha[kMR], troe_t3[kMR], troe_t1[kMR], troe_t2[kMR];
};

// the tables of the bound context (one translation unit includes this header)
__constant__ MixTables c_mix;

// compute_enthalpy_and_cp (Thermo.cu:136-192): h_k and cp_k in J/kg, linear h extrapolation below
// t_low.  Either output may be null (compute_enthalpy / compute_cp).
template <int NS, typename T = double>
__device__ __forceinline__ void mix_h_cp(T t, T *h, T *cp) {
  const T t2 = t * t, t3 = t2 * t, t4 = t3 * t, t5 = t4 * t;
#pragma unroll
  for (int i = 0; i < OSTC_NS; ++i) {
    T hh, cc;
    if (t < (T)c_mix.t_low[i]) {
      const T tt = (T)c_mix.t_low[i], tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt, tt5 = tt4 * tt;
      const double *a = c_mix.low[i];
      hh = (T)a[0] * tt + T(0.5) * (T)a[1] * tt2 + (T)a[2] * tt3 / T(3) + T(0.25) * (T)a[3] * tt4 +
           T(0.2) * (T)a[4] * tt5 + (T)a[5];
      cc = (T)a[0] + (T)a[1] * tt + (T)a[2] * tt2 + (T)a[3] * tt3 + (T)a[4] * tt4;
      hh += cc * (t - tt);
    } else {
      const double *a = t < (T)c_mix.t_mid[i] ? c_mix.low[i] : c_mix.high[i];
      hh = (T)a[0] * t + T(0.5) * (T)a[1] * t2 + (T)a[2] * t3 / T(3) + T(0.25) * (T)a[3] * t4 +
           T(0.2) * (T)a[4] * t5 + (T)a[5];
      cc = (T)a[0] + (T)a[1] * t + (T)a[2] * t2 + (T)a[3] * t3 + (T)a[4] * t4;
    }
    if (h) h[i] = hh * (T)c_mix.ru_mw[i];
    if (cp) cp[i] = cc * (T)c_mix.ru_mw[i];
  }
}

// compute_gibbs_div_rt (Thermo.cu:194-210)
template <int NS, typename T = double>
__device__ __forceinline__ void mix_gibbs_rt(T t, T *g) {
  const T t2 = t * t, t3 = t2 * t, t4 = t3 * t, ti = 1 / t, lt = log(t);
#pragma unroll
  for (int i = 0; i < OSTC_NS; ++i) {
    if (t < c_mix.t_low[i]) {
      const double tt = c_mix.t_low[i], tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt, tti = 1 / tt, ltt = log(tt);
      const double *a = c_mix.low[i];
      g[i] = a[0] * (1.0 - ltt) - 0.5 * a[1] * tt - a[2] * tt2 / 6.0 - a[3] * tt3 / 12.0 - a[4] * tt4 * 0.05 +
             a[5] * tti - a[6];
    } else {
      const double *a = t < c_mix.t_mid[i] ? c_mix.low[i] : c_mix.high[i];
      g[i] = a[0] * (1.0 - lt) - 0.5 * a[1] * t - a[2] * t2 / 6.0 - a[3] * t3 / 12.0 - a[4] * t4 * 0.05 + a[5] * ti -
             a[6];
    }
  }
}

// Node properties of update_physical_properties<mixture> (FieldOperation.cuh:116-134) with
// compute_transport_property (Transport.cu:43-136): cp, gamma, acoustic speed, Wilke viscosity,
// Eucken-type conductivity and mixture-averaged rho*D_k (outputs written through the pointers).
template <int NS, typename T = double>
__device__ __forceinline__ void mix_properties(T rho, T p, T t, const T *y, T &gamma, T &acoustic, T &mu, T &cond,
                                               T *rhod) {
  const int ns = OSTC_NS;
  T cp[Spec<NS>::A];
  mix_h_cp<NS, T>(t, nullptr, cp);
  T mw = 0, cpt = 0, cvt = 0;
  for (int l = 0; l < ns; ++l) {
    mw += y[l] * (T)c_mix.imw[l];
    cpt += y[l] * cp[l];
    cvt += y[l] * (cp[l] - (T)c_mix.ru_mw[l]);
  }
  mw = 1 / mw;
  gamma = cpt / cvt;
  acoustic = tsqrt(gamma * T(kRuD) * t / mw);
  // (T*)^-0.145 = exp(-0.145 (ln T + ln c)) and (T* + 0.5)^-2 = 1 / (T* + 0.5)^2: the same values as
  // pow to within a few ulp, at one log per node
  T X[Spec<NS>::A], vis[Spec<NS>::A], svis[Spec<NS>::A], isvis[Spec<NS>::A];
  const T st = tsqrt(t), lt = log(t);
  for (int l = 0; l < ns; ++l) {
    X[l] = y[l] * mw * (T)c_mix.imw[l];
    const T tdl = t * (T)c_mix.lj_potent_inv[l];
    const T ci = T(1.147) * exp(T(-0.145) * (lt + (T)c_mix.ln_lj[l])) + T(1) / ((tdl + T(0.5)) * (tdl + T(0.5)));
    vis[l] = (T)c_mix.vis_coeff[l] * st / ci;
    svis[l] = tsqrt(vis[l]);
    isvis[l] = T(1) / svis[l];
  }
  T visc = 0, cd = 0;
  for (int m = 0; m < ns; ++m) {
    T vt = 0;
    for (int n = 0; n < ns; ++n) {
      T pf = 1;
      if (m != n) {
        const T num = T(1) + svis[m] * isvis[n] * (T)c_mix.wj_div_wi_1_4[m][n];
        pf = num * num * (T)c_mix.sqrt_wiwj_8[m][n];
      }
      vt += pf * X[n];
    }
    const T ct = T(1.065) * vt - T(0.065) * X[m];
    visc += vis[m] * X[m] / vt;
    const T lam = vis[m] * (cp[m] + T(1.25) * (T)c_mix.ru_mw[m]);
    cd += lam * X[m] / ct;
  }
  mu = visc;
  cond = cd;
  // mixture-averaged diffusion with the binary coefficients D_ln = coeff T^1.5 / (p Omega_D(T*)).
  // D_ln is symmetric in (l, n) (both of its tables are), so each pair is evaluated once and added to
  // both species' sums; every sum still runs over n in increasing order.
  const T t32p = t * st / p;
  const T eps = T(1e-12);
  T num[Spec<NS>::A], den[Spec<NS>::A];
  for (int l = 0; l < ns; ++l) num[l] = den[l] = 0;
  for (int l = 0; l < ns; ++l) {
    for (int n = l + 1; n < ns; ++n) {
      const T tr = t * (T)c_mix.kb_over_eps[l][n];
      const T om = exp(T(-0.145) * (lt + (T)c_mix.ln_kbe[l][n])) + T(1) / ((tr + T(0.5)) * (tr + T(0.5)));
      const T dln = (T)c_mix.binary_diff[l][n] * t32p / om;
      num[l] += (X[n] + eps) * (T)c_mix.mw[n];
      den[l] += (X[n] + eps) / dln;
      num[n] += (X[l] + eps) * (T)c_mix.mw[l];
      den[n] += (X[l] + eps) / dln;
    }
  }
  for (int l = 0; l < ns; ++l) rhod[l] = rho * num[l] / (den[l] * mw);
}

// compute_temperature_and_pressure (FieldOperation.cu:3-40): Newton on e(T) starting from t, relative
// tolerance 1e-3, at most 1000 iterations.  Returns T; p = rho R T through pout.
template <int NS, typename T = double>
__device__ __forceinline__ T mix_temperature(T rho, T e, T t, const T *y, T &pout) {
  const int ns = OSTC_NS;
  T mw = 0;
  for (int l = 0; l < ns; ++l) mw += y[l] * c_mix.imw[l];
  mw = 1 / mw;
  const T gc = kRuD / mw;
  T err = 1.0;
  int iter = 0;
  T h[Spec<NS>::A], cp[Spec<NS>::A];
  while (err > 1e-3 && iter++ < 1000) {
    mix_h_cp<NS, T>(t, h, cp);
    T cpt = 0.0, hm = 0.0;
    for (int l = 0; l < ns; ++l) {
      cpt += cp[l] * y[l];
      hm += h[l] * y[l];
    }
    const T t1 = t - (hm - gc * t - e) / (cpt - gc);
    err = fabs(1 - t1 / t);
    t = t1;
  }
  pout = rho * t * gc;
  return t;
}

// A T^b exp(-Ea/T) (arrhenius, FiniteRateChem.cu:104-106) as A exp(b ln T - Ea/T): one exp per
// rate with ln T and 1/T formed once per node (the argument's rounding, ~1e-16 of |Ea/T| <= ~60,
// is the only difference from pow * exp)
__device__ __forceinline__ double arrhenius(double lt, double ti, double A, double b, double Ea) {
  return A * exp(fma(b, lt, -Ea * ti));
}

// x^n for the small integer reaction orders of the equilibrium constant, pow beyond |n| = 2
template <typename T>
__device__ __forceinline__ T ipow(T x, int n) {
  switch (n) {
    case 0: return T(1.0);
    case 1: return x;
    case -1: return 1.0 / x;
    case 2: return x * x;
    case -2: return 1.0 / (x * x);
    default: return pow(x, (double)n);
  }
}

// Forward and backward rate constants of reaction r (forward_reaction_rate, backward_reaction_rate,
// FiniteRateChem.cu:60-150) at T (with ln T, 1/T), third-body concentration sum cc and, where the
// equilibrium constant is used, g = g_k / (Ru T) of every species.  Irreversible: kb = 0; the
// equilibrium constant for every other type but 2 when any reaction needs it (it also overwrites
// REV coefficients); else the REV Arrhenius coefficients (times the third-body sum for type 4).
template <int NS, typename T>
__device__ __forceinline__ void reaction_rates(int r, T t, T lt, T ti, T cc, const T *g, T &kf_out, T &kb_out) {
  const int ns = OSTC_NS;
  const int ty = c_mix.label[r];
  T kf = arrhenius(lt, ti, c_mix.A[r], c_mix.b[r], c_mix.Ea[r]);
  if (ty == 3) {
    kf += arrhenius(lt, ti, c_mix.A2[r], c_mix.b2[r], c_mix.Ea2[r]);
  } else if (ty == 4) {
    kf *= cc;
  } else if (ty > 4) {
    const T klow = arrhenius(lt, ti, c_mix.A2[r], c_mix.b2[r], c_mix.Ea2[r]);
    const T pr = klow * cc / kf;
    T F = 1.0;
    if (ty > 5) {
      T fc = (1 - c_mix.troe_alpha[r]) * exp(-t / c_mix.troe_t3[r]) +
                  c_mix.troe_alpha[r] * exp(-t / c_mix.troe_t1[r]);
      if (ty == 7) fc += exp(-c_mix.troe_t2[r] / t);
      const T lfc = log10(fc);
      const T cq = -0.4 - 0.67 * lfc, nq = 0.75 - 1.27 * lfc;
      const T lpr = log10(pr);
      const T tmp = (lpr + cq) / (nq - 0.14 * (lpr + cq));
      F = pow(10.0, lfc / (1.0 + tmp * tmp));
    }
    kf = kf * pr / (1.0 + pr) * F;
  }
  T kb = 0;
  if (ty == 0) {
    kb = 0;
  } else if (ty != 2 && c_mix.use_gibbs) {
    T dg = 0;
    for (int l = 0; l < ns; ++l) dg += g[l] * (c_mix.stoi_b[r][l] - c_mix.stoi_f[r][l]);
    const T temp_t = kPatmD / kRuD * 1e-3 / t;
    const T kc = ipow(temp_t, c_mix.order[r]) * exp(-dg);
    kb = kf / kc;
  } else if (c_mix.rev_type[r] == 1) {
    kb = arrhenius(lt, ti, c_mix.A2[r], c_mix.b2[r], c_mix.Ea2[r]);
    if (ty == 4) kb *= cc;
  }
  kf_out = kf;
  kb_out = kb;
}

// finite_rate_chemistry (FiniteRateChem.cu:7-58, rates :60-195): omega_k in kg/(m^3 s) at one node.
// With jac non-null also the chemical source Jacobian of compute_chem_src_jacobian
// (FiniteRateChem.cu:197-217), [ns][ns] row-major, in 1/s; with omega_d non-null the destruction
// rates omega_d,k of chemical_source (:179-195), kg/(m^3 s).
template <int NS, typename T = double>
__device__ __forceinline__ void mix_chemistry(T rho, T t, const T *y, T *omega, T *jac = nullptr,
                                              T *omega_d = nullptr) {
  const int ns = OSTC_NS, nr = c_mix.nr;
  const T lt = log(t), ti = 1.0 / t;
  T c[Spec<NS>::A];
  for (int l = 0; l < ns; ++l) c[l] = rho * y[l] * c_mix.imw[l] * 1e-3;
  T g[Spec<NS>::A];
  if (c_mix.use_gibbs) mix_gibbs_rt<NS, T>(t, g);
  for (int l = 0; l < ns; ++l) omega[l] = 0;
  T cre[Spec<NS>::A], des[Spec<NS>::A];
  for (int l = 0; l < ns; ++l) cre[l] = des[l] = 0;
  for (int r = 0; r < nr; ++r) {
    const int ty = c_mix.label[r];
    T cc = 0;
    if (ty >= 4)
      for (int l = 0; l < ns; ++l) cc += c[l] * c_mix.third_body[r][l];
    T kf, kb;
    reaction_rates<NS, T>(r, t, lt, ti, cc, g, kf, kb);
    // concentration products: integer powers as products (pow(c, 1) = c, pow(c, 2) = c*c to within
    // the rounding of pow itself), pow only for higher orders
    T q1 = 1.0, q2 = ty != 0 ? 1.0 : 0.0;
#pragma unroll
    for (int l = 0; l < ns; ++l) {
      const int nf = c_mix.stoi_f[r][l];
      if (nf == 1) q1 *= c[l];
      else if (nf == 2) q1 *= c[l] * c[l];
      else if (nf) q1 *= pow(c[l], (double)nf);
    }
    if (ty != 0) {
#pragma unroll
      for (int l = 0; l < ns; ++l) {
        const int nb = c_mix.stoi_b[r][l];
        if (nb == 1) q2 *= c[l];
        else if (nb == 2) q2 *= c[l] * c[l];
        else if (nb) q2 *= pow(c[l], (double)nb);
      }
    }
    q1 *= kf;
    if (ty != 0) q2 *= kb;
    if (jac) {
      // sum over reactions in order, per (m, n): (nu_b,m - nu_f,m)(nu_f,n q1 - nu_b,n q2)
#pragma unroll
      for (int m = 0; m < ns; ++m) {
        const int dm = c_mix.stoi_b[r][m] - c_mix.stoi_f[r][m];
        if (dm == 0) continue;
#pragma unroll
        for (int n = 0; n < ns; ++n)
          jac[m * ns + n] += dm * (c_mix.stoi_f[r][n] * q1 - c_mix.stoi_b[r][n] * q2);
      }
    }
    for (int l = 0; l < ns; ++l) {
      cre[l] += q2 * c_mix.stoi_f[r][l] + q1 * c_mix.stoi_b[r][l];
      des[l] += q1 * c_mix.stoi_f[r][l] + q2 * c_mix.stoi_b[r][l];
    }
  }
  for (int l = 0; l < ns; ++l) omega[l] = cre[l] * (c_mix.mw[l] * 1e+3) - des[l] * (c_mix.mw[l] * 1e+3);
  if (omega_d)
    for (int l = 0; l < ns; ++l) omega_d[l] = des[l] * (c_mix.mw[l] * 1e+3);
  if (jac) {
#pragma unroll
    for (int n = 0; n < ns; ++n) {
      const bool live = y[n] > 1e-25;
      const T inv = live ? 1.0 / (rho * y[n]) : 0.0;
#pragma unroll
      for (int m = 0; m < ns; ++m) jac[m * ns + n] = c_mix.mw[m] * (live ? jac[m * ns + n] * inv : 0.0) * 1e+3;
    }
  }
}

// solve_chem_system (FiniteRateChem.cu:302-357): column-pivoted LU of the ns x ns matrix lhs in place,
// then forward / back substitution of b (length ns) in place.
template <int NS>
__device__ __forceinline__ void mix_lu_solve(double *lhs, double *b) {
  const int dim = OSTC_NS;
  int ipiv[Spec<NS>::A];
  for (int n = 0; n < dim; ++n) {
    int ik = n;
    for (int m = n; m < dim; ++m) {
      for (int t = 0; t < n; ++t) lhs[m * dim + n] -= lhs[m * dim + t] * lhs[t * dim + n];
      if (fabs(lhs[m * dim + n]) > fabs(lhs[ik * dim + n])) ik = m;
    }
    ipiv[n] = ik;
    if (ik != n)
      for (int t = 0; t < dim; ++t) {
        const double mid = lhs[ik * dim + t];
        lhs[ik * dim + t] = lhs[n * dim + t];
        lhs[n * dim + t] = mid;
      }
    for (int p = n + 1; p < dim; ++p)
      for (int t = 0; t < n; ++t) lhs[n * dim + p] -= lhs[n * dim + t] * lhs[t * dim + p];
    for (int m = n + 1; m < dim; ++m) lhs[m * dim + n] /= lhs[n * dim + n];
  }
  for (int m = 0; m < dim; ++m) {
    const int t = ipiv[m];
    if (t != m) {
      const double mid = b[t];
      b[t] = b[m];
      b[m] = mid;
    }
  }
  for (int m = 1; m < dim; ++m)
    for (int t = 0; t < m; ++t) b[m] -= lhs[m * dim + t] * b[t];
  b[dim - 1] /= lhs[dim * dim - 1];
  for (int m = dim - 2; m >= 0; --m) {
    for (int t = m + 1; t < dim; ++t) b[m] -= lhs[m * dim + t] * b[t];
    b[m] /= lhs[m * dim + m];
  }
}

// ---------------------------------------------------------------- flux-split WENO7 (71 / 72)

template <typename T>
__device__ __forceinline__ T fvs_beta7(T s1, T s2, T s3) {
  return s1 * s1 + T(13.0 / 12.0) * s2 * s2 + T(1043.0 / 960) * s3 * s3 + T(1.0 / 12) * s1 * s3;
}

// (eps + beta)^2 of the Z weights; in FP32 floored at 1e-30 so that a smooth stencil (beta = 0,
// where the scaled eps underflows) gives the linear weights instead of 0/0
template <typename T>
__device__ __forceinline__ T fvs_den(T eps, T beta) {
  const T d = (eps + beta) * (eps + beta);
  if constexpr (sizeof(T) == 4) return fmaxf(d, 1e-30f);
  return d;
}

// Unnormalised Z weights a_k = c_k (1 + tau / D_k), D_k = (eps + beta_k)^2.  FP64 forms the four
// quotients from two divisions, 1 / D0 = D1 / (D0 D1) and alike (D_k >= eps^2 keeps the pair products
// in range for any practical eps; if one underflows the four divisions are taken); FP32 divides each
// (its scaled D_k may be as small as 1e-30).
template <typename T>
__device__ __forceinline__ void fvs_weights(T c0, T c1, T c2, T c3, T tau, T d0, T d1, T d2, T d3, T &a0, T &a1, T &a2,
                                            T &a3) {
  const T p01 = d0 * d1, p23 = d2 * d3;
  if (sizeof(T) == 8 && p01 > T(0) && p23 > T(0)) {  // pair products representable (always, for eps > 1e-77)
    const T r01 = tau / p01, r23 = tau / p23;
    a0 = c0 + c0 * (d1 * r01);
    a1 = c1 + c1 * (d0 * r01);
    a2 = c2 + c2 * (d3 * r23);
    a3 = c3 + c3 * (d2 * r23);
  } else {
    a0 = c0 + c0 * tau / d0;
    a1 = c1 + c1 * tau / d1;
    a2 = c2 + c2 * tau / d2;
    a3 = c3 + c3 * tau / d3;
  }
}

// WENO7 of the flux-split path (WENO.cu:1619-1693): returns f+ + f-.
template <typename T>
__device__ __forceinline__ T fvs_weno7_core(const T *vp, const T *vm, T eps) {
  const T one6th = T(1.0 / 6), one12th = T(1.0 / 12);
  const T c0 = T(1.0 / 35), c1 = T(12.0 / 35), c2 = T(18.0 / 35), c3 = T(4.0 / 35);
  T s1 = one6th * (-2 * vp[0] + 9 * vp[1] - 18 * vp[2] + 11 * vp[3]);
  T s2 = -vp[0] + 4 * vp[1] - 5 * vp[2] + 2 * vp[3];
  T s3 = -vp[0] + 3 * vp[1] - 3 * vp[2] + vp[3];
  T b0 = fvs_beta7(s1, s2, s3);
  s1 = one6th * (vp[1] - 6 * vp[2] + 3 * vp[3] + 2 * vp[4]);
  s2 = vp[2] - 2 * vp[3] + vp[4];
  s3 = -vp[1] + 3 * vp[2] - 3 * vp[3] + vp[4];
  T b1 = fvs_beta7(s1, s2, s3);
  s1 = one6th * (-2 * vp[2] - 3 * vp[3] + 6 * vp[4] - vp[5]);
  s3 = -vp[2] + 3 * vp[3] - 3 * vp[4] + vp[5];
  T b2 = fvs_beta7(s1, s2, s3);
  s1 = one6th * (-11 * vp[3] + 18 * vp[4] - 9 * vp[5] + 2 * vp[6]);
  s2 = 2 * vp[3] - 5 * vp[4] + 4 * vp[5] - vp[6];
  s3 = -vp[3] + 3 * vp[4] - 3 * vp[5] + vp[6];
  T b3 = fvs_beta7(s1, s2, s3);
  T tau = (b0 - b3) * (b0 - b3);
  T a0, a1, a2, a3;
  fvs_weights(c0, c1, c2, c3, tau, fvs_den(eps, b0), fvs_den(eps, b1), fvs_den(eps, b2), fvs_den(eps, b3), a0, a1, a2,
              a3);
  T v0 = one12th * (-3 * vp[0] + 13 * vp[1] - 23 * vp[2] + 25 * vp[3]);
  T v1 = one12th * (vp[1] - 5 * vp[2] + 13 * vp[3] + 3 * vp[4]);
  T v2 = one12th * (-vp[2] + 7 * vp[3] + 7 * vp[4] - vp[5]);
  T v3 = one12th * (3 * vp[3] + 13 * vp[4] - 5 * vp[5] + vp[6]);
  const T fp = (a0 * v0 + a1 * v1 + a2 * v2 + a3 * v3) / (a0 + a1 + a2 + a3);
  s1 = one6th * (-2 * vm[6] + 9 * vm[5] - 18 * vm[4] + 11 * vm[3]);
  s2 = -vm[6] + 4 * vm[5] - 5 * vm[4] + 2 * vm[3];
  s3 = -vm[6] + 3 * vm[5] - 3 * vm[4] + vm[3];
  b0 = fvs_beta7(s1, s2, s3);
  s1 = one6th * (vm[5] - 6 * vm[4] + 3 * vm[3] + 2 * vm[2]);
  s2 = vm[4] - 2 * vm[3] + vm[2];
  s3 = -vm[5] + 3 * vm[4] - 3 * vm[3] + vm[2];
  b1 = fvs_beta7(s1, s2, s3);
  s1 = one6th * (-2 * vm[4] - 3 * vm[3] + 6 * vm[2] - vm[1]);
  s3 = -vm[4] + 3 * vm[3] - 3 * vm[2] + vm[1];
  b2 = fvs_beta7(s1, s2, s3);
  s1 = one6th * (-11 * vm[3] + 18 * vm[2] - 9 * vm[1] + 2 * vm[0]);
  s2 = 2 * vm[3] - 5 * vm[2] + 4 * vm[1] - vm[0];
  s3 = -vm[3] + 3 * vm[2] - 3 * vm[1] + vm[0];
  b3 = fvs_beta7(s1, s2, s3);
  tau = (b0 - b3) * (b0 - b3);
  fvs_weights(c0, c1, c2, c3, tau, fvs_den(eps, b0), fvs_den(eps, b1), fvs_den(eps, b2), fvs_den(eps, b3), a0, a1, a2,
              a3);
  v0 = one12th * (-3 * vm[6] + 13 * vm[5] - 23 * vm[4] + 25 * vm[3]);
  v1 = one12th * (vm[5] - 5 * vm[4] + 13 * vm[3] + 3 * vm[2]);
  v2 = one12th * (-vm[4] + 7 * vm[3] + 7 * vm[2] - vm[1]);
  v3 = one12th * (3 * vm[3] + 13 * vm[2] - 5 * vm[1] + vm[0]);
  const T fm = (a0 * v0 + a1 * v1 + a2 * v2 + a3 * v3) / (a0 + a1 + a2 + a3);
  return fp + fm;
}

__device__ __forceinline__ double fvs_weno7(const double *vp, const double *vm, double eps) {
  return fvs_weno7_core<double>(vp, vm, eps);
}

// FP32 form.  beta ~ v^2 and tau ~ v^4, so the split fluxes of a minor species (|v| ~ 1e-11) or the
// energy flux of a coarse grid (|v| ~ 1e10) leave the FP32 range although the weights themselves
// (tau / (eps + beta)^2, scale-free as eps -> 0) are O(1).  The stencil is therefore scaled by the
// power of two 2^-E below its largest magnitude (exact), eps by 2^-2E, and the face value scaled back.
__device__ __forceinline__ float fvs_weno7(const float *vp, const float *vm, double eps) {
  float m = 0.f;
#pragma unroll
  for (int i = 0; i < 7; ++i) m = fmaxf(m, fmaxf(fabsf(vp[i]), fabsf(vm[i])));
  if (!(m > 0.f)) {  // all zero: the face value is 0 (or NaN, carried through)
    float z = 0.f;
#pragma unroll
    for (int i = 0; i < 7; ++i) z += vp[i] + vm[i];
    return z;
  }
  int ex = (__float_as_int(m) >> 23) & 0xff;  // biased exponent of m
  ex = ex < 1 ? 1 : (ex > 253 ? 253 : ex);
  const float inv = __int_as_float((254 - ex) << 23);  // 2^(127 - ex)
  const float scale = __int_as_float(ex << 23);        // 2^(ex - 127)
  float sp[7], sm[7];
#pragma unroll
  for (int i = 0; i < 7; ++i) {
    sp[i] = vp[i] * inv;
    sm[i] = vm[i] * inv;
  }
  const double id = (double)inv;
  const float e = (float)(eps * id * id);
  return fvs_weno7_core<float>(sp, sm, e) * scale;
}

}  // namespace ostc
