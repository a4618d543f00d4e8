// air_math.cuh -- per-face / per-node arithmetic of the calorically-perfect-air RHS, written once and
// instantiated for T = double (plain FP64 path) and T = float (mixed path).  The operation order of
// every expression follows the reference source it cites, so the FP64 instantiation reproduces the
// reference to rounding.
#pragma once

#include <cuda_runtime.h>

namespace ostc {

constexpr double kGamma = 1.4;
constexpr double kRuD = 8314.462618;
constexpr double kMwD = 28.9647;

template <typename T> __device__ __forceinline__ T tsqrt(T x);
template <> __device__ __forceinline__ double tsqrt<double>(double x) { return sqrt(x); }
template <> __device__ __forceinline__ float tsqrt<float>(float x) { return sqrtf(x); }
template <typename T> __device__ __forceinline__ T tabs(T x);
template <> __device__ __forceinline__ double tabs<double>(double x) { return fabs(x); }
template <> __device__ __forceinline__ float tabs<float>(float x) { return fabsf(x); }
template <typename T> __device__ __forceinline__ T tmin(T a, T b);
template <> __device__ __forceinline__ double tmin<double>(double a, double b) { return fmin(a, b); }
template <> __device__ __forceinline__ float tmin<float>(float a, float b) { return fminf(a, b); }
template <typename T> __device__ __forceinline__ T tmax(T a, T b);
template <> __device__ __forceinline__ double tmax<double>(double a, double b) { return fmax(a, b); }
template <> __device__ __forceinline__ float tmax<float>(float a, float b) { return fmaxf(a, b); }

// Sutherland viscosity (Transport.cu:6-9); always FP64 (it feeds the FP64 state path).
__device__ __forceinline__ double sutherland(double t) {
  return 1.7894e-5 * pow(t / 288.16, 1.5) * (288.16 + 110) / (t + 110);
}

// ------------------------------------------------------------------ characteristic WENO-Z

// Denominator (eps + beta)^2 of a WENO-Z weight.  The reference's WENO7 smoothness indicator beta2
// (AWENO.cu:236-238, 263-265) is not positive semi-definite, so eps + beta can pass through zero;
// in FP64 its square stays representable, in FP32 it can underflow to 0 and turn the weight into
// inf/inf.  The FP32 instantiation clamps the square at 1e-30 (the weight is then ~1e30 times the
// linear weight, i.e. that stencil is selected exactly as in FP64); FP64 is left untouched.
template <typename T> __device__ __forceinline__ T wden(T e);
template <> __device__ __forceinline__ double wden<double>(double e) { return e * e; }
template <> __device__ __forceinline__ float wden<float>(float e) { return fmaxf(e * e, 1e-30f); }

// Characteristic WENO5-Z interpolation of field l_row at i+1/2 from the 6 points i-2..i+3
// (AWENO.cu:156-210).  q(s, v) returns conservative variable v of stencil point s.
template <typename T, class Q>
__device__ __forceinline__ void weno5_char(const T *L, const Q &q, int l_row, T &vminus, T &vplus) {
  T v[6];
#pragma unroll
  for (int s = 0; s < 6; ++s) {
    T acc = T(0);
#pragma unroll
    for (int j = 0; j < 5; ++j) acc += L[l_row * 5 + j] * q(s, j);
    v[s] = acc;
  }
  T v0 = T(0.125) * (T(3) * v[0] - T(10) * v[1] + T(15) * v[2]);
  T v1 = T(0.125) * (-v[1] + T(6) * v[2] + T(3) * v[3]);
  T v2 = T(0.125) * (T(3) * v[2] + T(6) * v[3] - v[4]);
  const T th = T(13.0 / 12);
  T beta0 = th * (v[0] + v[2] - T(2) * v[1]) * (v[0] + v[2] - T(2) * v[1]) +
            T(0.25) * (v[0] + T(3) * v[2] - T(4) * v[1]) * (v[0] + T(3) * v[2] - T(4) * v[1]);
  T beta1 = th * (v[1] + v[3] - T(2) * v[2]) * (v[1] + v[3] - T(2) * v[2]) + T(0.25) * (v[3] - v[1]) * (v[3] - v[1]);
  T beta2 = th * (v[2] + v[4] - T(2) * v[3]) * (v[2] + v[4] - T(2) * v[3]) +
            T(0.25) * (T(3) * v[2] + v[4] - T(4) * v[3]) * (T(3) * v[2] + v[4] - T(4) * v[3]);
  T tau = (beta0 - beta2) * (beta0 - beta2);
  const T eps = T(1e-6), o16 = T(1.0 / 16), f8 = T(5.0 / 8), f16 = T(5.0 / 16);
  T a0 = o16 + o16 * tau / wden<T>(eps + beta0);
  T a1 = f8 + f8 * tau / wden<T>(eps + beta1);
  T a2 = f16 + f16 * tau / wden<T>(eps + beta2);
  vminus = (a0 * v0 + a1 * v1 + a2 * v2) / (a0 + a1 + a2);
  v0 = v1;
  v1 = v2;
  v2 = T(0.125) * (T(15) * v[3] - T(10) * v[4] + T(3) * v[5]);
  beta0 = th * (v[1] + v[3] - T(2) * v[2]) * (v[1] + v[3] - T(2) * v[2]) +
          T(0.25) * (v[1] + T(3) * v[3] - T(4) * v[2]) * (v[1] + T(3) * v[3] - T(4) * v[2]);
  beta1 = th * (v[2] + v[4] - T(2) * v[3]) * (v[2] + v[4] - T(2) * v[3]) + T(0.25) * (v[4] - v[2]) * (v[4] - v[2]);
  beta2 = th * (v[3] + v[5] - T(2) * v[4]) * (v[3] + v[5] - T(2) * v[4]) +
          T(0.25) * (T(3) * v[3] + v[5] - T(4) * v[4]) * (T(3) * v[3] + v[5] - T(4) * v[4]);
  tau = (beta0 - beta2) * (beta0 - beta2);
  a0 = f16 + f16 * tau / wden<T>(eps + beta0);
  a1 = f8 + f8 * tau / wden<T>(eps + beta1);
  a2 = o16 + o16 * tau / wden<T>(eps + beta2);
  vplus = (a0 * v0 + a1 * v1 + a2 * v2) / (a0 + a1 + a2);
}

// Characteristic WENO7-Z interpolation from the 8 points i-3..i+4 (AWENO.cu:212-280).
template <typename T, class Q>
__device__ __forceinline__ void weno7_char(const T *L, const Q &q, int l_row, T &vminus, T &vplus) {
  T v[8];
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    T acc = T(0);
#pragma unroll
    for (int j = 0; j < 5; ++j) acc += L[l_row * 5 + j] * q(s, j);
    v[s] = acc;
  }
  T v0 = T(0.0625) * (T(5) * v[3] + T(15) * v[4] - T(5) * v[5] + v[6]);
  T v1 = T(0.0625) * (-v[2] + T(9) * v[3] + T(9) * v[4] - v[5]);
  T v2 = T(0.0625) * (v[1] - T(5) * v[2] + T(15) * v[3] + T(5) * v[4]);
  T v3 = T(0.0625) * (T(-5) * v[0] + T(21) * v[1] - T(35) * v[2] + T(35) * v[3]);
  const T c = T(1.0 / 2880);
  T beta0 = c * (T(25729) * v[3] * v[3] + T(134241) * v[4] * v[4] + T(85641) * v[5] * v[5] -
                 T(6) * v[4] * (T(35047) * v[5] - T(9449) * v[6]) - T(47214) * v[5] * v[6] + T(6649) * v[6] * v[6] -
                 T(2) * v[3] * (T(57447) * v[4] - T(43107) * v[5] + T(11389) * v[6]));
  T beta1 = c * (T(6649) * v[2] * v[2] + T(41001) * v[3] * v[3] + T(33441) * v[4] * v[4] +
                 v[2] * (T(-30414) * v[3] + T(23094) * v[4] - T(5978) * v[5]) - T(19374) * v[4] * v[5] +
                 T(3169) * v[5] * v[5] + v[3] * (T(-70602) * v[4] + T(19014) * v[5]));
  T beta2 = c * (T(3169) * v[1] * v[1] + T(33441) * v[2] * v[2] + T(41001) * v[3] * v[3] - T(30414) * v[2] * v[3] +
                 T(6649) * v[3] * v[3] - T(2) * v[1] * (T(9687) * v[2] - T(9507) * v[3] + T(2989) * v[4]) +
                 v[2] * (T(-70602) * v[3] + T(23094) * v[4]));
  T beta3 = c * (T(6649) * v[0] * v[0] + T(85641) * v[1] * v[1] + T(134241) * v[2] * v[2] +
                 v[0] * (T(-47214) * v[1] + T(56694) * v[2] - T(22778) * v[3]) - T(114894) * v[2] * v[3] +
                 T(25729) * v[3] * v[3] + v[1] * (T(-210282) * v[2] + T(86214) * v[3]));
  T tau = (beta3 + T(5) * beta2 - T(5) * beta1 - beta0) * (beta3 + T(5) * beta2 - T(5) * beta1 - beta0);
  const T eps = T(1e-6), s7 = T(7.0 / 64), t5 = T(35.0 / 64), t1 = T(21.0 / 64), o1 = T(1.0 / 64);
  T a0 = s7 + s7 * tau / wden<T>(eps + beta0);
  T a1 = t5 + t5 * tau / wden<T>(eps + beta1);
  T a2 = t1 + t1 * tau / wden<T>(eps + beta2);
  T a3 = o1 + o1 * tau / wden<T>(eps + beta3);
  vminus = (a0 * v0 + a1 * v1 + a2 * v2 + a3 * v3) / (a0 + a1 + a2 + a3);
  v3 = v2;
  v2 = v1;
  v1 = v0;
  v0 = T(0.0625) * (T(35) * v[4] - T(35) * v[5] + T(21) * v[6] - T(5) * v[7]);
  beta0 = c * (T(25729) * v[4] * v[4] + T(134241) * v[5] * v[5] + T(85641) * v[6] * v[6] -
               T(6) * v[5] * (T(35047) * v[6] - T(9449) * v[7]) - T(47214) * v[6] * v[7] + T(6649) * v[7] * v[7] -
               T(2) * v[4] * (T(57447) * v[5] - T(43107) * v[6] + T(11389) * v[7]));
  beta1 = c * (T(6649) * v[3] * v[3] + T(41001) * v[4] * v[4] + T(33441) * v[5] * v[5] +
               v[3] * (T(-30414) * v[4] + T(23094) * v[5] - T(5978) * v[6]) - T(19374) * v[5] * v[6] +
               T(3169) * v[6] * v[6] + v[4] * (T(-70602) * v[5] + T(19014) * v[6]));
  beta2 = c * (T(3169) * v[2] * v[2] + T(33441) * v[3] * v[3] + T(41001) * v[4] * v[4] - T(30414) * v[3] * v[4] +
               T(6649) * v[4] * v[4] - T(2) * v[2] * (T(9687) * v[3] - T(9507) * v[4] + T(2989) * v[5]) +
               v[3] * (T(-70602) * v[4] + T(23094) * v[5]));
  beta3 = c * (T(6649) * v[1] * v[1] + T(85641) * v[2] * v[2] + T(134241) * v[3] * v[3] +
               v[1] * (T(-47214) * v[2] + T(56694) * v[3] - T(22778) * v[4]) - T(114894) * v[3] * v[4] +
               T(25729) * v[4] * v[4] + v[2] * (T(-210282) * v[3] + T(86214) * v[4]));
  tau = (beta3 + T(5) * beta2 - T(5) * beta1 - beta0) * (beta3 + T(5) * beta2 - T(5) * beta1 - beta0);
  a0 = o1 + o1 * tau / wden<T>(eps + beta0);
  a1 = t1 + t1 * tau / wden<T>(eps + beta1);
  a2 = t5 + t5 * tau / wden<T>(eps + beta2);
  a3 = s7 + s7 * tau / wden<T>(eps + beta3);
  vplus = (a0 * v0 + a1 * v1 + a2 * v2 + a3 * v3) / (a0 + a1 + a2 + a3);
}

// AWENO_interpolation<Air> (AWENO.cu:15-154).  NG = 3 (WENO5) or 4 (WENO7); q(s, v) for
// s in [0, 2*NG) is point i-NG+1+s, v = 0..4 conservative variables, v = 5 pressure.
// mt0/mt1: metric row of the sweep direction at i and i+1.  pl/pr: rho,u,v,w,p,rhoE.
template <int NG, typename T, class Q>
__device__ __forceinline__ void aweno_interp(const Q &q, const T *mt0, const T *mt1, T *pl, T *pr) {
  constexpr int cl = NG - 1, cr = NG;
  const T gm1 = T(kGamma - 1);
  const T l0 = q(cl, 0), r0 = q(cr, 0);
  const T sl = tsqrt(l0), sr = tsqrt(r0);
  const T rlc = sl / (sl + sr);
  const T rrc = sr / (sl + sr);
  const T um = rlc * q(cl, 1) / l0 + rrc * q(cr, 1) / r0;
  const T vm = rlc * q(cl, 2) / l0 + rrc * q(cr, 2) / r0;
  const T wm = rlc * q(cl, 3) / l0 + rrc * q(cr, 3) / r0;
  const T ekm = T(0.5) * (um * um + vm * vm + wm * wm);
  const T hl = (q(cl, 4) + q(cl, 5)) / l0;
  const T hr = (q(cr, 4) + q(cr, 5)) / r0;
  const T hm = rlc * hl + rrc * hr;
  const T cm2 = gm1 * (hm - ekm);
  const T cm = tsqrt(cm2);
  T kx = T(0.5) * (mt0[0] + mt1[0]);
  T ky = T(0.5) * (mt0[1] + mt1[1]);
  T kz = T(0.5) * (mt0[2] + mt1[2]);
  const T gradK = tsqrt(kx * kx + ky * ky + kz * kz);
  kx /= gradK;
  ky /= gradK;
  kz /= gradK;
  const T Uk = kx * um + ky * vm + kz * wm;
  const T alpha = gm1 * ekm;
  T L[25];
  L[0] = (alpha + Uk * cm) / cm2 * T(0.5);
  L[1] = -(gm1 * um + kx * cm) / cm2 * T(0.5);
  L[2] = -(gm1 * vm + ky * cm) / cm2 * T(0.5);
  L[3] = -(gm1 * wm + kz * cm) / cm2 * T(0.5);
  L[4] = gm1 / cm2 * T(0.5);
  L[5] = kx * (T(1) - alpha / cm2) - (kz * vm - ky * wm) / cm;
  L[6] = kx * gm1 * um / cm2;
  L[7] = (kx * gm1 * vm + kz * cm) / cm2;
  L[8] = (kx * gm1 * wm - ky * cm) / cm2;
  L[9] = -kx * gm1 / cm2;
  L[10] = ky * (T(1) - alpha / cm2) - (kx * wm - kz * um) / cm;
  L[11] = (ky * gm1 * um - kz * cm) / cm2;
  L[12] = ky * gm1 * vm / cm2;
  L[13] = (ky * gm1 * wm + kx * cm) / cm2;
  L[14] = -ky * gm1 / cm2;
  L[15] = kz * (T(1) - alpha / cm2) - (ky * um - kx * vm) / cm;
  L[16] = (kz * gm1 * um + ky * cm) / cm2;
  L[17] = (kz * gm1 * vm - kx * cm) / cm2;
  L[18] = kz * gm1 * wm / cm2;
  L[19] = -kz * gm1 / cm2;
  L[20] = (alpha - Uk * cm) / cm2 * T(0.5);
  L[21] = -(gm1 * um - kx * cm) / cm2 * T(0.5);
  L[22] = -(gm1 * vm - ky * cm) / cm2 * T(0.5);
  L[23] = -(gm1 * wm - kz * cm) / cm2 * T(0.5);
  L[24] = gm1 / cm2 * T(0.5);
  T vmi[5], vpl[5];
#pragma unroll
  for (int l = 0; l < 5; ++l) {
    if constexpr (NG == 3) {
      weno5_char<T>(L, q, l, vmi[l], vpl[l]);
    } else {
      weno7_char<T>(L, q, l, vmi[l], vpl[l]);
    }
  }
  T R[25];
  R[0] = T(1); R[1] = kx; R[2] = ky; R[3] = kz; R[4] = T(1);
  R[5] = um - kx * cm; R[6] = kx * um; R[7] = ky * um - kz * cm; R[8] = kz * um + ky * cm; R[9] = um + kx * cm;
  R[10] = vm - ky * cm; R[11] = kx * vm + kz * cm; R[12] = ky * vm; R[13] = kz * vm - kx * cm; R[14] = vm + ky * cm;
  R[15] = wm - kz * cm; R[16] = kx * wm - ky * cm; R[17] = ky * wm + kx * cm; R[18] = kz * wm; R[19] = wm + kz * cm;
  R[20] = hm - Uk * cm;
  R[21] = kx * alpha / gm1 + (kz * vm - ky * wm) * cm;
  R[22] = ky * alpha / gm1 + (kx * wm - kz * um) * cm;
  R[23] = kz * alpha / gm1 + (ky * um - kx * vm) * cm;
  R[24] = hm + Uk * cm;
  T ql[5], qr[5];
#pragma unroll
  for (int m = 0; m < 5; ++m) {
    T a = T(0), b = T(0);
#pragma unroll
    for (int n = 0; n < 5; ++n) {
      a += R[m * 5 + n] * vmi[n];
      b += R[m * 5 + n] * vpl[n];
    }
    ql[m] = a;
    qr[m] = b;
  }
  pl[0] = ql[0];
  pl[1] = ql[1] / ql[0];
  pl[2] = ql[2] / ql[0];
  pl[3] = ql[3] / ql[0];
  pl[4] = gm1 * (ql[4] - T(0.5) * (pl[1] * pl[1] + pl[2] * pl[2] + pl[3] * pl[3]) * ql[0]);
  pl[5] = ql[4];
  pr[0] = qr[0];
  pr[1] = qr[1] / qr[0];
  pr[2] = qr[2] / qr[0];
  pr[3] = qr[3] / qr[0];
  pr[4] = gm1 * (qr[4] - T(0.5) * (pr[1] * pr[1] + pr[2] * pr[2] + pr[3] * pr[3]) * qr[0]);
  pr[5] = qr[4];
}

// ------------------------------------------------------------------ Riemann solvers

// riemannSolver_ausmPlus<Air> (RiemannSolver.cuh:9-96)
template <typename T>
__device__ __forceinline__ void ausm_plus(const T *pl, const T *pr, const T *mt0, const T *mt1, T j0, T j1, T *fc) {
  const T k1 = T(0.5) * (j0 * mt0[0] + j1 * mt1[0]);
  const T k2 = T(0.5) * (j0 * mt0[1] + j1 * mt1[1]);
  const T k3 = T(0.5) * (j0 * mt0[2] + j1 * mt1[2]);
  const T gkj = tsqrt(k1 * k1 + k2 * k2 + k3 * k3);
  const T ul = (k1 * pl[1] + k2 * pl[2] + k3 * pl[3]) / gkj;
  const T ur = (k1 * pr[1] + k2 * pr[2] + k3 * pr[3]) / gkj;
  const T p_l = pl[4], p_r = pr[4], rho_l = pl[0], rho_r = pr[0];
  const T gam = T(kGamma);
  const T c = T(0.5) * (tsqrt(gam * p_l / rho_l) + tsqrt(gam * p_r / rho_r));
  const T mach_l = ul / c, mach_r = ur / c;
  T mlp, mrn, plp, prn;
  const T alpha = T(3 / 16.0);
  if (tabs(mach_l) > T(1)) {
    mlp = T(0.5) * (mach_l + tabs(mach_l));
    plp = mlp / mach_l;
  } else {
    const T a = (mach_l + T(1)) * (mach_l + T(1)) * T(0.25);
    const T b = (mach_l * mach_l - T(1)) * (mach_l * mach_l - T(1));
    mlp = a + T(0.125) * b;
    plp = a * (T(2) - mach_l) + alpha * mach_l * b;
  }
  if (tabs(mach_r) > T(1)) {
    mrn = T(0.5) * (mach_r - tabs(mach_r));
    prn = mrn / mach_r;
  } else {
    const T a = (mach_r - T(1)) * (mach_r - T(1)) * T(0.25);
    const T b = (mach_r * mach_r - T(1)) * (mach_r * mach_r - T(1));
    mrn = -a - T(0.125) * b;
    prn = a * (T(2) + mach_r) - alpha * mach_r * b;
  }
  const T p_coeff = plp * p_l + prn * p_r;
  const T m_half = mlp + mrn;
  const T mach_pos = T(0.5) * (m_half + tabs(m_half));
  const T mach_neg = T(0.5) * (m_half - tabs(m_half));
  const T mass_flux = c * (rho_l * mach_pos + rho_r * mach_neg);
  const T coeff = mass_flux * gkj;
  const T *s = mass_flux >= T(0) ? pl : pr;
  fc[0] = coeff;
  fc[1] = coeff * s[1] + p_coeff * k1;
  fc[2] = coeff * s[2] + p_coeff * k2;
  fc[3] = coeff * s[3] + p_coeff * k3;
  fc[4] = coeff * (s[5] + s[4]) / s[0];
}

// riemannSolver_hllc<Air> (RiemannSolver.cuh:98-230)
template <typename T>
__device__ __forceinline__ void hllc(const T *pl, const T *pr, const T *mt0, const T *mt1, T j0, T j1, T *fc) {
  const T gam = T(kGamma);
  const T sql = tsqrt(pl[0]), sqr = tsqrt(pr[0]);
  const T rl_c = sql / (sql + sqr);
  const T rr_c = sqr / (sql + sqr);
  const T ut = pl[1] * rl_c + pr[1] * rr_c;
  const T vt = pl[2] * rl_c + pr[2] * rr_c;
  const T wt = pl[3] * rl_c + pr[3] * rr_c;
  const T hl = (pl[5] + pl[4]) / pl[0];
  const T hr = (pr[5] + pr[4]) / pr[0];
  const T ht = hl * rl_c + hr * rr_c;
  const T ekt = T(0.5) * (ut * ut + vt * vt + wt * wt);
  const T ct = tsqrt((gam - T(1)) * (ht - ekt));
  const T kx = T(0.5) * (mt0[0] + mt1[0]);
  const T ky = T(0.5) * (mt0[1] + mt1[1]);
  const T kz = T(0.5) * (mt0[2] + mt1[2]);
  const T gradK = tsqrt(kx * kx + ky * ky + kz * kz);
  const T Ubar = (kx * ut + ky * vt + kz * wt) / gradK;
  const T jac = T(0.5) * (j0 + j1);
  const T Ul = kx * pl[1] + ky * pl[2] + kz * pl[3];
  const T cl = tsqrt(gam * pl[4] / pl[0]);
  const T sl = tmin(Ul / gradK - cl, Ubar - ct);
  if (sl >= T(0)) {
    const T rU = pl[0] * Ul;
    fc[0] = jac * rU;
    fc[1] = jac * (rU * pl[1] + pl[4] * kx);
    fc[2] = jac * (rU * pl[2] + pl[4] * ky);
    fc[3] = jac * (rU * pl[3] + pl[4] * kz);
    fc[4] = jac * ((pl[5] + pl[4]) * Ul);
    return;
  }
  const T Ur = kx * pr[1] + ky * pr[2] + kz * pr[3];
  const T cr = tsqrt(gam * pr[4] / pr[0]);
  const T sr = tmax(Ur / gradK + cr, Ubar + ct);
  if (sr < T(0)) {
    const T rU = pr[0] * Ur;
    fc[0] = jac * rU;
    fc[1] = jac * (rU * pr[1] + pr[4] * kx);
    fc[2] = jac * (rU * pr[2] + pr[4] * ky);
    fc[3] = jac * (rU * pr[3] + pr[4] * kz);
    fc[4] = jac * ((pr[5] + pr[4]) * Ur);
    return;
  }
  const T sm = ((pr[0] * Ur * (sr - Ur / gradK) - pl[0] * Ul * (sl - Ul / gradK)) / gradK + pl[4] - pr[4]) /
               (pr[0] * (sr - Ur / gradK) - pl[0] * (sl - Ul / gradK));
  const T pm = pl[0] * (sl - Ul / gradK) * (sm - Ul / gradK) + pl[4];
  if (sm >= T(0)) {
    const T pc = T(1) / (sl - sm);
    const T Q = jac * pc * sm * (sl * gradK - Ul) * pl[0];
    fc[0] = Q;
    const T dP = (sl * pm - sm * pl[4]) * pc * jac;
    fc[1] = Q * pl[1] + dP * kx;
    fc[2] = Q * pl[2] + dP * ky;
    fc[3] = Q * pl[3] + dP * kz;
    fc[4] = Q * pl[5] / pl[0] + pc * jac * (sl * pm * sm * gradK - sm * pl[4] * Ul);
  } else {
    const T pc = T(1) / (sr - sm);
    const T Q = jac * pc * sm * (sr * gradK - Ur) * pr[0];
    fc[0] = Q;
    const T dP = (sr * pm - sm * pr[4]) * pc * jac;
    fc[1] = Q * pr[1] + dP * kx;
    fc[2] = Q * pr[2] + dP * ky;
    fc[3] = Q * pr[3] + dP * kz;
    fc[4] = Q * pr[5] / pr[0] + pc * jac * (sr * pm * sm * gradK - sm * pr[4] * Ur);
  }
}

// Whole AWENO face flux: interpolation then the selected Riemann solver (InviscidScheme.cu:333-345).
template <int NG, int RS, typename T, class Q>
__device__ __forceinline__ void aweno_face_flux(const Q &q, const T *mt0, const T *mt1, T j0, T j1, T *fc) {
  T pl[6], pr[6];
  aweno_interp<NG, T>(q, mt0, mt1, pl, pr);
  if constexpr (RS == 4) {
    hllc<T>(pl, pr, mt0, mt1, j0, j1, fc);
  } else {
    ausm_plus<T>(pl, pr, mt0, mt1, j0, j1, fc);
  }
}

// Physical flux of one node for the central-difference correction (AWENO.cu:307-321).
// b: rho,u,v,w,p (bv 0..4); e: rho*E (cv 4); k: metric row of the sweep direction.
template <typename T>
__device__ __forceinline__ void node_flux(const T *b, T e, const T *k, T jac, T *f) {
  const T Uk = k[0] * b[1] + k[1] * b[2] + k[2] * b[3];
  const T rhoUk = b[0] * Uk;
  f[0] = rhoUk * jac;
  f[1] = jac * (rhoUk * b[1] + k[0] * b[4]);
  f[2] = jac * (rhoUk * b[2] + k[1] * b[4]);
  f[3] = jac * (rhoUk * b[3] + k[2] * b[4]);
  f[4] = jac * Uk * (e + b[4]);
}

// Central correction coefficients (AWENO.cu:327-350): dq += sum_m c_m (f(i+m) - f(i-m)), evaluated
// from the outermost pair inwards as the reference writes it.
template <int NG, typename T, class F>
__device__ __forceinline__ T cds_correction(const F &f, int l) {
  if constexpr (NG == 3) {
    const T c1 = T(-19.0 / 3840), c2 = T(13.0 / 320), c3 = T(-17.0 / 256);
    return c1 * (f(3, l) - f(-3, l)) + c2 * (f(2, l) - f(-2, l)) + c3 * (f(1, l) - f(-1, l));
  } else {
    const T c4 = T(-81.0 / 71680), c3 = T(1261.0 / 107520), c2 = T(-289.0 / 5120), c1 = T(421.0 / 5120);
    return c4 * (f(4, l) - f(-4, l)) + c3 * (f(3, l) - f(-3, l)) + c2 * (f(2, l) - f(-2, l)) +
           c1 * (f(1, l) - f(-1, l));
  }
}

}  // namespace ostc
