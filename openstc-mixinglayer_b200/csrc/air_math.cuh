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
// 1 / sqrt(x), from which the callers form sqrt(x) = x / sqrt(x) and 1 / x = (1 / sqrt(x))^2.  FP32:
// one reciprocal square root stands in for a square root and a division.  FP64 keeps the correctly
// rounded square root and division: with the reciprocal square root the FP64 sweeps ran 3 % faster,
// but the multi-block reference fixtures moved from inside the 1e-12 parity bar to 1.1-1.8e-12.
template <typename T> __device__ __forceinline__ T trsqrt(T x);
template <> __device__ __forceinline__ double trsqrt<double>(double x) { return 1.0 / sqrt(x); }
template <> __device__ __forceinline__ float trsqrt<float>(float x) { return rsqrtf(x); }
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

// Convex WENO-Z combination sum_k a_k v_k / sum_k a_k with a_k = d_k (1 + tau / D_k) and
// D_k = (eps + beta_k)^2 (AWENO.cu:193-197, 245-251).
// FP64: multiplying numerator and denominator by prod_k D_k leaves one division per combination
// instead of one per weight (products of three D_k stay far inside the FP64 range), and the two sides
// of a face share one division (finish).
// FP32: products of three D_k can underflow, so each weight keeps its own fast division.  The
// reference's WENO7 indicator beta2 (AWENO.cu:236-238, 263-265) is neither shift-invariant nor
// positive semi-definite, so eps + beta2 can pass through zero; in FP32 its square can underflow to
// 0, so D_k is floored at 1e-30 (the weight is then ~1e30 times the linear weight: that stencil is
// selected, as in FP64).
template <typename T> struct WenoComb;
template <> struct WenoComb<double> {
  // numerator and denominator of the combination
  static __device__ __forceinline__ void c3(double d0, double d1, double d2, double D0, double D1, double D2,
                                            double tau, double v0, double v1, double v2, double &num, double &den) {
    const double w0 = d0 * (D0 + tau) * (D1 * D2), w1 = d1 * (D1 + tau) * (D0 * D2), w2 = d2 * (D2 + tau) * (D0 * D1);
    num = w0 * v0 + w1 * v1 + w2 * v2;
    den = w0 + w1 + w2;
  }
  static __device__ __forceinline__ void c4(double d0, double d1, double d2, double d3, double D0, double D1,
                                            double D2, double D3, double tau, double v0, double v1, double v2,
                                            double v3, double &num, double &den) {
    const double a = D0 * D1, b = D2 * D3;
    const double w0 = d0 * (D0 + tau) * (D1 * b), w1 = d1 * (D1 + tau) * (D0 * b);
    const double w2 = d2 * (D2 + tau) * (a * D3), w3 = d3 * (D3 + tau) * (a * D2);
    num = w0 * v0 + w1 * v1 + w2 * v2 + w3 * v3;
    den = w0 + w1 + w2 + w3;
  }
  // the two sides' quotients from one division: a denominator is a sum of products of up to four
  // (eps + beta)^2 factors, so the product of two stays inside the FP64 range
  static __device__ __forceinline__ void finish(double nm, double dm, double np, double dp, double &vm, double &vp) {
    const double q = 1.0 / (dm * dp);
    vm = nm * dp * q;
    vp = np * dm * q;
  }
};
template <> struct WenoComb<float> {
  static __device__ __forceinline__ void c3(float d0, float d1, float d2, float D0, float D1, float D2, float tau,
                                            float v0, float v1, float v2, float &num, float &den) {
    const float a0 = d0 + d0 * __fdividef(tau, fmaxf(D0, 1e-30f)), a1 = d1 + d1 * __fdividef(tau, fmaxf(D1, 1e-30f));
    const float a2 = d2 + d2 * __fdividef(tau, fmaxf(D2, 1e-30f));
    num = a0 * v0 + a1 * v1 + a2 * v2;
    den = a0 + a1 + a2;
  }
  static __device__ __forceinline__ void c4(float d0, float d1, float d2, float d3, float D0, float D1, float D2,
                                            float D3, float tau, float v0, float v1, float v2, float v3, float &num,
                                            float &den) {
    const float a0 = d0 + d0 * __fdividef(tau, fmaxf(D0, 1e-30f)), a1 = d1 + d1 * __fdividef(tau, fmaxf(D1, 1e-30f));
    const float a2 = d2 + d2 * __fdividef(tau, fmaxf(D2, 1e-30f)), a3 = d3 + d3 * __fdividef(tau, fmaxf(D3, 1e-30f));
    num = a0 * v0 + a1 * v1 + a2 * v2 + a3 * v3;
    den = a0 + a1 + a2 + a3;
  }
  static __device__ __forceinline__ void finish(float nm, float dm, float np, float dp, float &vm, float &vp) {
    vm = __fdividef(nm, dm);
    vp = __fdividef(np, dp);
  }
};

// Characteristic WENO5-Z interpolation of one field at i+1/2 from the 6 points i-2..i+3
// (AWENO.cu:156-210).  Lr: the field's row of the left eigenvector matrix; q(s, v) returns
// conservative variable v of stencil point s.  Smoothness indicators, tau and the candidate
// interpolants are the reference's expressions; the weights go through WenoComb.
template <typename T, class Q>
__device__ __forceinline__ void weno5_char(const T *Lr, const Q &q, T &vminus, T &vplus) {
  T v[6];
#pragma unroll
  for (int s = 0; s < 6; ++s) {
    T acc = T(0);
#pragma unroll
    for (int j = 0; j < 5; ++j) acc += Lr[j] * q(s, j);
    v[s] = acc;
  }
  const T th = T(13.0 / 12), eps = T(1e-6), o16 = T(1.0 / 16), f8 = T(5.0 / 8), f16 = T(5.0 / 16);
  T nm, dm, np, dp;
  {
    const T v0 = T(0.125) * (T(3) * v[0] - T(10) * v[1] + T(15) * v[2]);
    const T v1 = T(0.125) * (-v[1] + T(6) * v[2] + T(3) * v[3]);
    const T v2 = T(0.125) * (T(3) * v[2] + T(6) * v[3] - v[4]);
    const T beta0 = th * (v[0] + v[2] - T(2) * v[1]) * (v[0] + v[2] - T(2) * v[1]) +
                    T(0.25) * (v[0] + T(3) * v[2] - T(4) * v[1]) * (v[0] + T(3) * v[2] - T(4) * v[1]);
    const T beta1 = th * (v[1] + v[3] - T(2) * v[2]) * (v[1] + v[3] - T(2) * v[2]) + T(0.25) * (v[3] - v[1]) * (v[3] - v[1]);
    const T beta2 = th * (v[2] + v[4] - T(2) * v[3]) * (v[2] + v[4] - T(2) * v[3]) +
                    T(0.25) * (T(3) * v[2] + v[4] - T(4) * v[3]) * (T(3) * v[2] + v[4] - T(4) * v[3]);
    const T tau = (beta0 - beta2) * (beta0 - beta2);
    WenoComb<T>::c3(o16, f8, f16, (eps + beta0) * (eps + beta0), (eps + beta1) * (eps + beta1),
                    (eps + beta2) * (eps + beta2), tau, v0, v1, v2, nm, dm);
  }
  {
    const T v0 = T(0.125) * (-v[1] + T(6) * v[2] + T(3) * v[3]);
    const T v1 = T(0.125) * (T(3) * v[2] + T(6) * v[3] - v[4]);
    const T v2 = T(0.125) * (T(15) * v[3] - T(10) * v[4] + T(3) * v[5]);
    const T beta0 = th * (v[1] + v[3] - T(2) * v[2]) * (v[1] + v[3] - T(2) * v[2]) +
                    T(0.25) * (v[1] + T(3) * v[3] - T(4) * v[2]) * (v[1] + T(3) * v[3] - T(4) * v[2]);
    const T beta1 = th * (v[2] + v[4] - T(2) * v[3]) * (v[2] + v[4] - T(2) * v[3]) + T(0.25) * (v[4] - v[2]) * (v[4] - v[2]);
    const T beta2 = th * (v[3] + v[5] - T(2) * v[4]) * (v[3] + v[5] - T(2) * v[4]) +
                    T(0.25) * (T(3) * v[3] + v[5] - T(4) * v[4]) * (T(3) * v[3] + v[5] - T(4) * v[4]);
    const T tau = (beta0 - beta2) * (beta0 - beta2);
    WenoComb<T>::c3(f16, f8, o16, (eps + beta0) * (eps + beta0), (eps + beta1) * (eps + beta1),
                    (eps + beta2) * (eps + beta2), tau, v0, v1, v2, np, dp);
  }
  WenoComb<T>::finish(nm, dm, np, dp, vminus, vplus);
}

// Characteristic WENO7-Z interpolation from the 8 points i-3..i+4 (AWENO.cu:212-280).  beta2 keeps
// the reference's expression exactly (see WenoComb above).
template <typename T>
__device__ __forceinline__ void weno7_betas(const T *v, T &b0, T &b1, T &b2, T &b3) {
  const T c = T(1.0 / 2880);
  b0 = c * (T(25729) * v[3] * v[3] + T(134241) * v[4] * v[4] + T(85641) * v[5] * v[5] -
            T(6) * v[4] * (T(35047) * v[5] - T(9449) * v[6]) - T(47214) * v[5] * v[6] + T(6649) * v[6] * v[6] -
            T(2) * v[3] * (T(57447) * v[4] - T(43107) * v[5] + T(11389) * v[6]));
  b1 = c * (T(6649) * v[2] * v[2] + T(41001) * v[3] * v[3] + T(33441) * v[4] * v[4] +
            v[2] * (T(-30414) * v[3] + T(23094) * v[4] - T(5978) * v[5]) - T(19374) * v[4] * v[5] +
            T(3169) * v[5] * v[5] + v[3] * (T(-70602) * v[4] + T(19014) * v[5]));
  b2 = c * (T(3169) * v[1] * v[1] + T(33441) * v[2] * v[2] + T(41001) * v[3] * v[3] - T(30414) * v[2] * v[3] +
            T(6649) * v[3] * v[3] - T(2) * v[1] * (T(9687) * v[2] - T(9507) * v[3] + T(2989) * v[4]) +
            v[2] * (T(-70602) * v[3] + T(23094) * v[4]));
  b3 = c * (T(6649) * v[0] * v[0] + T(85641) * v[1] * v[1] + T(134241) * v[2] * v[2] +
            v[0] * (T(-47214) * v[1] + T(56694) * v[2] - T(22778) * v[3]) - T(114894) * v[2] * v[3] +
            T(25729) * v[3] * v[3] + v[1] * (T(-210282) * v[2] + T(86214) * v[3]));
}

template <typename T, class Q>
__device__ __forceinline__ void weno7_char(const T *Lr, const Q &q, T &vminus, T &vplus) {
  T v[8];
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    T acc = T(0);
#pragma unroll
    for (int j = 0; j < 5; ++j) acc += Lr[j] * q(s, j);
    v[s] = acc;
  }
  const T eps = T(1e-6), s7 = T(7.0 / 64), t5 = T(35.0 / 64), t1 = T(21.0 / 64), o1 = T(1.0 / 64);
  T nm, dm, np, dp;
  {
    const T v0 = T(0.0625) * (T(5) * v[3] + T(15) * v[4] - T(5) * v[5] + v[6]);
    const T v1 = T(0.0625) * (-v[2] + T(9) * v[3] + T(9) * v[4] - v[5]);
    const T v2 = T(0.0625) * (v[1] - T(5) * v[2] + T(15) * v[3] + T(5) * v[4]);
    const T v3 = T(0.0625) * (T(-5) * v[0] + T(21) * v[1] - T(35) * v[2] + T(35) * v[3]);
    T b0, b1, b2, b3;
    weno7_betas<T>(v, b0, b1, b2, b3);
    const T tau = (b3 + T(5) * b2 - T(5) * b1 - b0) * (b3 + T(5) * b2 - T(5) * b1 - b0);
    WenoComb<T>::c4(s7, t5, t1, o1, (eps + b0) * (eps + b0), (eps + b1) * (eps + b1), (eps + b2) * (eps + b2),
                    (eps + b3) * (eps + b3), tau, v0, v1, v2, v3, nm, dm);
  }
  {
    const T v1 = T(0.0625) * (T(5) * v[3] + T(15) * v[4] - T(5) * v[5] + v[6]);
    const T v2 = T(0.0625) * (-v[2] + T(9) * v[3] + T(9) * v[4] - v[5]);
    const T v3 = T(0.0625) * (v[1] - T(5) * v[2] + T(15) * v[3] + T(5) * v[4]);
    const T v0 = T(0.0625) * (T(35) * v[4] - T(35) * v[5] + T(21) * v[6] - T(5) * v[7]);
    T b0, b1, b2, b3;
    weno7_betas<T>(v + 1, b0, b1, b2, b3);
    const T tau = (b3 + T(5) * b2 - T(5) * b1 - b0) * (b3 + T(5) * b2 - T(5) * b1 - b0);
    WenoComb<T>::c4(o1, t1, t5, s7, (eps + b0) * (eps + b0), (eps + b1) * (eps + b1), (eps + b2) * (eps + b2),
                    (eps + b3) * (eps + b3), tau, v0, v1, v2, v3, np, dp);
  }
  WenoComb<T>::finish(nm, dm, np, dp, vminus, vplus);
}

// AWENO_interpolation<Air> (AWENO.cu:15-154).  NG = 3 (WENO5) or 4 (WENO7); q(s, v) for
// s in [0, 2*NG) is point i-NG+1+s, v = 0..4 conservative variables, v = 5 pressure.
// mt0/mt1: metric row of the sweep direction at i and i+1.  pl/pr: rho,u,v,w,p,rhoE.
// The left eigenvector matrix is built one row per characteristic field and the right one column
// by column, so only one row/column is live at a time; the reference's divisions by cm2, cm,
// gradK and rho are replaced by multiplications with their reciprocals.  The back projection
// accumulates field by field in the reference's summation order.
template <int NG, typename T, class Q>
__device__ __forceinline__ void aweno_interp(const Q &q, const T *mt0, const T *mt1, T *pl, T *pr) {
  constexpr int cl = NG - 1, cr = NG;
  const T gm1 = T(kGamma - 1), igm1 = T(1.0 / (kGamma - 1));
  const T l0 = q(cl, 0), r0 = q(cr, 0);
  const T rsl = trsqrt(l0), rsr = trsqrt(r0);
  const T sl = l0 * rsl, sr = r0 * rsr;
  const T isum = T(1) / (sl + sr);
  const T rlc = sl * isum, rrc = sr * isum;
  const T il0 = rsl * rsl, ir0 = rsr * rsr;
  const T um = rlc * q(cl, 1) * il0 + rrc * q(cr, 1) * ir0;
  const T vm = rlc * q(cl, 2) * il0 + rrc * q(cr, 2) * ir0;
  const T wm = rlc * q(cl, 3) * il0 + rrc * q(cr, 3) * ir0;
  const T ekm = T(0.5) * (um * um + vm * vm + wm * wm);
  const T hl = (q(cl, 4) + q(cl, 5)) * il0;
  const T hr = (q(cr, 4) + q(cr, 5)) * ir0;
  const T hm = rlc * hl + rrc * hr;
  const T cm2 = gm1 * (hm - ekm);
  const T icm = trsqrt(cm2);
  const T cm = cm2 * icm, icm2 = icm * icm;
  T kx = T(0.5) * (mt0[0] + mt1[0]);
  T ky = T(0.5) * (mt0[1] + mt1[1]);
  T kz = T(0.5) * (mt0[2] + mt1[2]);
  const T igk = trsqrt(kx * kx + ky * ky + kz * kz);
  kx *= igk;
  ky *= igk;
  kz *= igk;
  const T Uk = kx * um + ky * vm + kz * wm;
  const T alpha = gm1 * ekm;
  const T h2 = T(0.5) * icm2;
  T ql[5] = {T(0), T(0), T(0), T(0), T(0)}, qr[5] = {T(0), T(0), T(0), T(0), T(0)};
#pragma unroll
  for (int l = 0; l < 5; ++l) {
    T Lr[5], Rc[5];
    if (l == 0) {
      Lr[0] = (alpha + Uk * cm) * h2;
      Lr[1] = -(gm1 * um + kx * cm) * h2;
      Lr[2] = -(gm1 * vm + ky * cm) * h2;
      Lr[3] = -(gm1 * wm + kz * cm) * h2;
      Lr[4] = gm1 * h2;
      Rc[0] = T(1); Rc[1] = um - kx * cm; Rc[2] = vm - ky * cm; Rc[3] = wm - kz * cm; Rc[4] = hm - Uk * cm;
    } else if (l == 1) {
      Lr[0] = kx * (T(1) - alpha * icm2) - (kz * vm - ky * wm) * icm;
      Lr[1] = kx * gm1 * um * icm2;
      Lr[2] = (kx * gm1 * vm + kz * cm) * icm2;
      Lr[3] = (kx * gm1 * wm - ky * cm) * icm2;
      Lr[4] = -kx * gm1 * icm2;
      Rc[0] = kx; Rc[1] = kx * um; Rc[2] = kx * vm + kz * cm; Rc[3] = kx * wm - ky * cm;
      Rc[4] = kx * alpha * igm1 + (kz * vm - ky * wm) * cm;
    } else if (l == 2) {
      Lr[0] = ky * (T(1) - alpha * icm2) - (kx * wm - kz * um) * icm;
      Lr[1] = (ky * gm1 * um - kz * cm) * icm2;
      Lr[2] = ky * gm1 * vm * icm2;
      Lr[3] = (ky * gm1 * wm + kx * cm) * icm2;
      Lr[4] = -ky * gm1 * icm2;
      Rc[0] = ky; Rc[1] = ky * um - kz * cm; Rc[2] = ky * vm; Rc[3] = ky * wm + kx * cm;
      Rc[4] = ky * alpha * igm1 + (kx * wm - kz * um) * cm;
    } else if (l == 3) {
      Lr[0] = kz * (T(1) - alpha * icm2) - (ky * um - kx * vm) * icm;
      Lr[1] = (kz * gm1 * um + ky * cm) * icm2;
      Lr[2] = (kz * gm1 * vm - kx * cm) * icm2;
      Lr[3] = kz * gm1 * wm * icm2;
      Lr[4] = -kz * gm1 * icm2;
      Rc[0] = kz; Rc[1] = kz * um + ky * cm; Rc[2] = kz * vm - kx * cm; Rc[3] = kz * wm;
      Rc[4] = kz * alpha * igm1 + (ky * um - kx * vm) * cm;
    } else {
      Lr[0] = (alpha - Uk * cm) * h2;
      Lr[1] = -(gm1 * um - kx * cm) * h2;
      Lr[2] = -(gm1 * vm - ky * cm) * h2;
      Lr[3] = -(gm1 * wm - kz * cm) * h2;
      Lr[4] = gm1 * h2;
      Rc[0] = T(1); Rc[1] = um + kx * cm; Rc[2] = vm + ky * cm; Rc[3] = wm + kz * cm; Rc[4] = hm + Uk * cm;
    }
    T vmi, vpl;
    if constexpr (NG == 3) {
      weno5_char<T>(Lr, q, vmi, vpl);
    } else {
      weno7_char<T>(Lr, q, vmi, vpl);
    }
#pragma unroll
    for (int m = 0; m < 5; ++m) {
      ql[m] += Rc[m] * vmi;
      qr[m] += Rc[m] * vpl;
    }
  }
  const T iqq = T(1) / (ql[0] * qr[0]);
  const T iql = qr[0] * iqq, iqr = ql[0] * iqq;
  pl[0] = ql[0];
  pl[1] = ql[1] * iql;
  pl[2] = ql[2] * iql;
  pl[3] = ql[3] * iql;
  pl[4] = gm1 * (ql[4] - T(0.5) * (pl[1] * pl[1] + pl[2] * pl[2] + pl[3] * pl[3]) * ql[0]);
  pl[5] = ql[4];
  pr[0] = qr[0];
  pr[1] = qr[1] * iqr;
  pr[2] = qr[2] * iqr;
  pr[3] = qr[3] * iqr;
  pr[4] = gm1 * (qr[4] - T(0.5) * (pr[1] * pr[1] + pr[2] * pr[2] + pr[3] * pr[3]) * qr[0]);
  pr[5] = qr[4];
}

// ------------------------------------------------------------------ Riemann solvers

// riemannSolver_ausmPlus<Air> (RiemannSolver.cuh:9-96); divisions by the face-normal magnitude,
// sound speed and densities go through reciprocals.
template <typename T>
__device__ __forceinline__ void ausm_plus(const T *pl, const T *pr, const T *mt0, const T *mt1, T j0, T j1, T *fc) {
  const T k1 = T(0.5) * (j0 * mt0[0] + j1 * mt1[0]);
  const T k2 = T(0.5) * (j0 * mt0[1] + j1 * mt1[1]);
  const T k3 = T(0.5) * (j0 * mt0[2] + j1 * mt1[2]);
  const T k2s = k1 * k1 + k2 * k2 + k3 * k3;
  const T igkj = trsqrt(k2s);
  const T gkj = k2s * igkj;
  const T ul = (k1 * pl[1] + k2 * pl[2] + k3 * pl[3]) * igkj;
  const T ur = (k1 * pr[1] + k2 * pr[2] + k3 * pr[3]) * igkj;
  const T p_l = pl[4], p_r = pr[4], rho_l = pl[0], rho_r = pr[0];
  const T gam = T(kGamma);
  const T irl = T(1) / rho_l, irr = T(1) / rho_r;
  const T c = T(0.5) * (tsqrt(gam * p_l * irl) + tsqrt(gam * p_r * irr));
  const T ic = T(1) / c;
  const T mach_l = ul * ic, mach_r = ur * ic;
  T mlp, mrn, plp, prn;
  const T alpha = T(3 / 16.0);
  if (tabs(mach_l) > T(1)) {
    mlp = T(0.5) * (mach_l + tabs(mach_l));
    plp = mach_l > T(0) ? T(1) : T(0);
  } else {
    const T a = (mach_l + T(1)) * (mach_l + T(1)) * T(0.25);
    const T b = (mach_l * mach_l - T(1)) * (mach_l * mach_l - T(1));
    mlp = a + T(0.125) * b;
    plp = a * (T(2) - mach_l) + alpha * mach_l * b;
  }
  if (tabs(mach_r) > T(1)) {
    mrn = T(0.5) * (mach_r - tabs(mach_r));
    prn = mach_r < T(0) ? T(1) : T(0);
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
  const bool left = mass_flux >= T(0);
  const T *s = left ? pl : pr;
  fc[0] = coeff;
  fc[1] = coeff * s[1] + p_coeff * k1;
  fc[2] = coeff * s[2] + p_coeff * k2;
  fc[3] = coeff * s[3] + p_coeff * k3;
  fc[4] = coeff * (s[5] + s[4]) * (left ? irl : irr);
}

// riemannSolver_hllc<Air> (RiemannSolver.cuh:98-230), with shared reciprocals.
template <typename T>
__device__ __forceinline__ void hllc(const T *pl, const T *pr, const T *mt0, const T *mt1, T j0, T j1, T *fc) {
  const T gam = T(kGamma);
  const T rsl = trsqrt(pl[0]), rsr = trsqrt(pr[0]);
  const T sql = pl[0] * rsl, sqr = pr[0] * rsr;
  const T isq = T(1) / (sql + sqr);
  const T rl_c = sql * isq;
  const T rr_c = sqr * isq;
  const T ut = pl[1] * rl_c + pr[1] * rr_c;
  const T vt = pl[2] * rl_c + pr[2] * rr_c;
  const T wt = pl[3] * rl_c + pr[3] * rr_c;
  const T irl = rsl * rsl, irr = rsr * rsr;
  const T hl = (pl[5] + pl[4]) * irl;
  const T hr = (pr[5] + pr[4]) * irr;
  const T ht = hl * rl_c + hr * rr_c;
  const T ekt = T(0.5) * (ut * ut + vt * vt + wt * wt);
  const T ct = tsqrt((gam - T(1)) * (ht - ekt));
  const T kx = T(0.5) * (mt0[0] + mt1[0]);
  const T ky = T(0.5) * (mt0[1] + mt1[1]);
  const T kz = T(0.5) * (mt0[2] + mt1[2]);
  const T k2s = kx * kx + ky * ky + kz * kz;
  const T igk = trsqrt(k2s);
  const T gradK = k2s * igk;
  const T Ubar = (kx * ut + ky * vt + kz * wt) * igk;
  const T jac = T(0.5) * (j0 + j1);
  const T Ul = kx * pl[1] + ky * pl[2] + kz * pl[3];
  const T Ur = kx * pr[1] + ky * pr[2] + kz * pr[3];
  const T unl = Ul * igk, unr = Ur * igk;
  const T cl = tsqrt(gam * pl[4] * irl);
  const T sl = tmin(unl - cl, Ubar - ct);
  if (sl >= T(0)) {
    const T rU = pl[0] * Ul;
    fc[0] = jac * rU;
    fc[1] = jac * (rU * pl[1] + pl[4] * kx);
    fc[2] = jac * (rU * pl[2] + pl[4] * ky);
    fc[3] = jac * (rU * pl[3] + pl[4] * kz);
    fc[4] = jac * ((pl[5] + pl[4]) * Ul);
    return;
  }
  const T cr = tsqrt(gam * pr[4] * irr);
  const T sr = tmax(unr + cr, Ubar + ct);
  if (sr < T(0)) {
    const T rU = pr[0] * Ur;
    fc[0] = jac * rU;
    fc[1] = jac * (rU * pr[1] + pr[4] * kx);
    fc[2] = jac * (rU * pr[2] + pr[4] * ky);
    fc[3] = jac * (rU * pr[3] + pr[4] * kz);
    fc[4] = jac * ((pr[5] + pr[4]) * Ur);
    return;
  }
  const T sm = ((pr[0] * Ur * (sr - unr) - pl[0] * Ul * (sl - unl)) * igk + pl[4] - pr[4]) /
               (pr[0] * (sr - unr) - pl[0] * (sl - unl));
  const T pm = pl[0] * (sl - unl) * (sm - unl) + pl[4];
  const bool left = sm >= T(0);
  const T *q = left ? pl : pr;
  const T sk = left ? sl : sr, Uk = left ? Ul : Ur, irk = left ? irl : irr;
  const T pc = T(1) / (sk - sm);
  const T Q = jac * pc * sm * (sk * gradK - Uk) * q[0];
  fc[0] = Q;
  const T dP = (sk * pm - sm * q[4]) * pc * jac;
  fc[1] = Q * q[1] + dP * kx;
  fc[2] = Q * q[2] + dP * ky;
  fc[3] = Q * q[3] + dP * kz;
  fc[4] = Q * q[5] * irk + pc * jac * (sk * pm * sm * gradK - sm * q[4] * Uk);
}

// riemannSolver_laxFriedrich<Air> (RiemannSolver.cuh:420-460): face-averaged metric, the larger
// spectral radius of the two sides.
template <typename T>
__device__ __forceinline__ void lax_friedrichs(const T *pl, const T *pr, const T *mt0, const T *mt1, T j0, T j1,
                                               T *fc) {
  const T kx = T(0.5) * (mt0[0] + mt1[0]);
  const T ky = T(0.5) * (mt0[1] + mt1[1]);
  const T kz = T(0.5) * (mt0[2] + mt1[2]);
  const T gradK = tsqrt(kx * kx + ky * ky + kz * kz);
  const T Ukl = pl[1] * kx + pl[2] * ky + pl[3] * kz;
  const T Ukr = pr[1] * kx + pr[2] * ky + pr[3] * kz;
  const T cl = tsqrt(T(kGamma) * pl[4] / pl[0]);
  const T cr = tsqrt(T(kGamma) * pr[4] / pr[0]);
  const T sr = tmax(tabs(Ukl) + cl * gradK, tabs(Ukr) + cr * gradK);
  const T hj = T(0.25) * (j0 + j1);
  const T rUl = pl[0] * Ukl, rUr = pr[0] * Ukr;
  fc[0] = (rUl + rUr - sr * (pr[0] - pl[0])) * hj;
  fc[1] = (rUl * pl[1] + rUr * pr[1] + kx * (pl[4] + pr[4]) - sr * (pr[1] * pr[0] - pl[1] * pl[0])) * hj;
  fc[2] = (rUl * pl[2] + rUr * pr[2] + ky * (pl[4] + pr[4]) - sr * (pr[2] * pr[0] - pl[2] * pl[0])) * hj;
  fc[3] = (rUl * pl[3] + rUr * pr[3] + kz * (pl[4] + pr[4]) - sr * (pr[3] * pr[0] - pl[3] * pl[0])) * hj;
  fc[4] = ((pl[5] + pl[4]) * Ukl + (pr[5] + pr[4]) * Ukr - sr * (pr[5] - pl[5])) * hj;
}

// Harten entropy-fix threshold of one node (compute_entropy_fix_delta<Air>, InviscidScheme.cu:417-456):
// factor * (|U| + |V| (+ |W|) + c * mean |grad xi|).  m: the 9 metric entries of the node, b: rho..p.
template <typename T>
__device__ __forceinline__ T entropy_fix_delta(const T *m, const T *b, T factor, bool dim3) {
  const T U = tabs(b[1] * m[0] + b[2] * m[1] + b[3] * m[2]);
  const T V = tabs(b[1] * m[3] + b[2] * m[4] + b[3] * m[5]);
  const T W = tabs(b[1] * m[6] + b[2] * m[7] + b[3] * m[8]);
  const T kx = tsqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
  const T ky = tsqrt(m[3] * m[3] + m[4] * m[4] + m[5] * m[5]);
  const T kz = tsqrt(m[6] * m[6] + m[7] * m[7] + m[8] * m[8]);
  const T c = tsqrt(T(kGamma) * b[4] / b[0]);
  if (!dim3) return factor * (U + V + c * T(0.5) * (kx + ky));
  return factor * (U + V + W + c * (kx + ky + kz) / T(3));
}

// riemannSolver_Roe<Air> (RiemannSolver.cuh:279-417): the half sum of the two sides' physical fluxes
// (each with its own node's metric and Jacobian, compute_half_sum_left_right_flux :232-277) plus
// the Roe dissipation with Harten's entropy fix on |lambda| below the face-averaged threshold.
template <typename T>
__device__ __forceinline__ void roe(const T *pl, const T *pr, const T *mt0, const T *mt1, T j0, T j1, T d0, T d1,
                                    T *fc) {
  {
    const T jx = j0 * mt0[0], jy = j0 * mt0[1], jz = j0 * mt0[2];
    const T Uk = pl[1] * jx + pl[2] * jy + pl[3] * jz;
    const T co = Uk * pl[0];
    fc[0] = T(0.5) * co;
    fc[1] = T(0.5) * (co * pl[1] + pl[4] * jx);
    fc[2] = T(0.5) * (co * pl[2] + pl[4] * jy);
    fc[3] = T(0.5) * (co * pl[3] + pl[4] * jz);
    fc[4] = T(0.5) * Uk * (pl[4] + pl[5]);
  }
  {
    const T jx = j1 * mt1[0], jy = j1 * mt1[1], jz = j1 * mt1[2];
    const T Uk = pr[1] * jx + pr[2] * jy + pr[3] * jz;
    const T co = Uk * pr[0];
    fc[0] += T(0.5) * co;
    fc[1] += T(0.5) * (co * pr[1] + pr[4] * jx);
    fc[2] += T(0.5) * (co * pr[2] + pr[4] * jy);
    fc[3] += T(0.5) * (co * pr[3] + pr[4] * jz);
    fc[4] += T(0.5) * Uk * (pr[4] + pr[5]);
  }
  const T dl = tsqrt(pl[0]), dr = tsqrt(pr[0]);
  const T inv = T(1) / (dl + dr);
  const T u = (dl * pl[1] + dr * pr[1]) * inv;
  const T v = (dl * pl[2] + dr * pr[2]) * inv;
  const T w = (dl * pl[3] + dr * pr[3]) * inv;
  const T ek = T(0.5) * (u * u + v * v + w * w);
  const T hl = (pl[5] + pl[4]) / pl[0];
  const T hr = (pr[5] + pr[4]) / pr[0];
  const T h = (dl * hl + dr * hr) * inv;
  const T gm1 = T(kGamma - 1);
  const T c = tsqrt(gm1 * (h - ek));
  T kx = T(0.5) * (mt0[0] + mt1[0]);
  T ky = T(0.5) * (mt0[1] + mt1[1]);
  T kz = T(0.5) * (mt0[2] + mt1[2]);
  const T gradK = tsqrt(kx * kx + ky * ky + kz * kz);
  T Uk = kx * u + ky * v + kz * w;
  T ch[3] = {Uk - gradK * c, Uk, Uk + gradK * c};
  const T da = T(0.5) * (d0 + d1);
#pragma unroll
  for (int n = 0; n < 3; ++n) {
    ch[n] = tabs(ch[n]);
    if (ch[n] < da) ch[n] = T(0.5) * (ch[n] * ch[n] / da + da);
  }
  const T igk = T(1) / gradK;
  kx *= igk;
  ky *= igk;
  kz *= igk;
  Uk *= igk;
  const T ja = T(0.5) * (j0 + j1);
  const T q0 = ja * (pr[0] - pl[0]);
  const T q1 = ja * (pr[0] * pr[1] - pl[0] * pl[1]);
  const T q2 = ja * (pr[0] * pr[2] - pl[0] * pl[2]);
  const T q3 = ja * (pr[0] * pr[3] - pl[0] * pl[3]);
  const T q4 = ja * (pr[5] - pl[5]);
  const T ic = T(1) / c;
  T c1 = gm1 * (ek * q0 - u * q1 - v * q2 - w * q3 + q4) * ic * ic;
  T c2 = (kx * q1 + ky * q2 + kz * q3 - Uk * q0) * ic;
  const T c3 = q0 - c1;
  const T L0 = T(0.5) * (c1 - c2);
  const T L1 = kx * c3 - ((kz * v - ky * w) * q0 - kz * q2 + ky * q3) * ic;
  const T L2 = ky * c3 - ((kx * w - kz * u) * q0 - kx * q3 + kz * q1) * ic;
  const T L3 = kz * c3 - ((ky * u - kx * v) * q0 - ky * q1 + kx * q2) * ic;
  const T L4 = T(0.5) * (c1 + c2);
  const T b0 = -ch[0] * L0, b1 = -ch[1] * L1, b2 = -ch[1] * L2, b3 = -ch[1] * L3, b4 = -ch[2] * L4;
  const T c0 = kx * b1 + ky * b2 + kz * b3;
  c1 = c0 + b0 + b4;
  c2 = c * (b4 - b0);
  fc[0] += T(0.5) * c1;
  fc[1] += T(0.5) * (u * c1 + kx * c2 - c * (kz * b2 - ky * b3));
  fc[2] += T(0.5) * (v * c1 + ky * c2 - c * (kx * b3 - kz * b1));
  fc[3] += T(0.5) * (w * c1 + kz * c2 - c * (ky * b1 - kx * b2));
  fc[4] += T(0.5) * (h * c1 + Uk * c2 - c * c * c0 / gm1 +
                     c * ((kz * v - ky * w) * b1 + (kx * w - kz * u) * b2 + (ky * u - kx * v) * b3));
}

// ------------------------------------------------------------------ primitive reconstruction

// minmod with the reference's sign convention sgn(0) = +1 (Limiter.cuh:13-16, gxl_lib/Math.hpp:13-15).
template <typename T>
__device__ __forceinline__ T minmod(T a, T b) {
  const T sa = a < T(0) ? T(-1) : T(1), sb = b < T(0) ? T(-1) : T(1);
  return T(0.5) * (sa + sb) * tmin(tabs(a), tabs(b));
}

// Left/right primitive states at i+1/2 from nodes i-1, i, i+1, i+2 (v(m, l), m = -1..2), then the total
// energy of each side (reconstruction<Air>, InviscidScheme.cu:163-215; first_order_reconstruct,
// MUSCL_reconstruct (kappa = 1/3), NND2_reconstruct, Reconstruction.cu:5-45).
template <typename T, class V>
__device__ __forceinline__ void pv_reconstruct(const V &v, int recon, T *pl, T *pr) {
#pragma unroll
  for (int l = 0; l < 5; ++l) {
    const T a = v(0, l), bq = v(1, l);
    if (recon == 2 || recon == 3) {
      const T di = a - v(-1, l), di1 = bq - a, di2 = v(2, l) - bq;
      if (recon == 2) {
        const T k1 = T(1) - T(1.0 / 3.0), k2 = T(1) + T(1.0 / 3.0);
        pl[l] = a + T(0.25) * (k1 * minmod(di, di1) + k2 * minmod(di1, di));
        pr[l] = bq - T(0.25) * (k1 * minmod(di2, di1) + k2 * minmod(di1, di2));
      } else {
        pl[l] = a + T(0.5) * minmod(di, di1);
        pr[l] = bq - T(0.5) * minmod(di1, di2);
      }
    } else {
      pl[l] = a;
      pr[l] = bq;
    }
  }
  const T el = T(0.5) * (pl[1] * pl[1] + pl[2] * pl[2] + pl[3] * pl[3]);
  const T er = T(0.5) * (pr[1] * pr[1] + pr[2] * pr[2] + pr[3] * pr[3]);
  pl[5] = el * pl[0] + pl[4] / T(kGamma - 1);
  pr[5] = er * pr[0] + pr[4] / T(kGamma - 1);
}

// Whole AWENO face flux: interpolation then the selected Riemann solver (InviscidScheme.cu:333-345).
template <int NG, int RS, typename T, class Q>
__device__ __forceinline__ void aweno_face_flux(const Q &q, const T *mt0, const T *mt1, T j0, T j1, T *fc) {
  T pl[6], pr[6];
  aweno_interp<NG, T>(q, mt0, mt1, pl, pr);
  if constexpr (RS == 4) {
    hllc<T>(pl, pr, mt0, mt1, j0, j1, fc);
  } else if constexpr (RS == 1) {
    lax_friedrichs<T>(pl, pr, mt0, mt1, j0, j1, fc);
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
