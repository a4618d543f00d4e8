// pv_mix.cuh -- the primitive-reconstruction inviscid path for multi-component mixtures
// (compute_convective_term_pv / Roe_compute_inviscid_flux with MixtureModel Mixture or FR,
// InviscidScheme.cu:12-215, 369-548): 1st-order / MUSCL / NND2 reconstruction of rho, u, v, w, p and
// the mass fractions, the mixture total energy and gamma of each side from NASA-7 thermo at the side's
// temperature (reconstruction<mixture>, :163-215), and the mixture branches of AUSM+, HLLC and Roe
// (RiemannSolver.cuh:9-417).  Lax-Friedrichs has no mixture form in the reference (its
// riemannSolver_laxFriedrich<mixture> only prints) and is refused on the host.
//
// Two kernels per sweep direction: k_pv_mix_face computes every face flux of the block (one thread per
// face, face f between nodes f and f + 1 along the sweep, f = -1 .. n-1) into a face array laid out
// [l][face] with i fastest, and k_pv_mix_diff differences the faces of every node into dq.  FP64.
#pragma once

namespace ostc {

// reconstructed state: rho, u, v, w, p, Y_1..Y_ns at [0, nv), rho E at [nv], gamma at [nv + 1]
template <int NS> struct PvMix {
  static constexpr int V = 5 + Spec<NS>::A + 2;
};

// reconstruction<mixture> (InviscidScheme.cu:163-215) of the face between stencil nodes 1 and 2 of
// st[4][nv] (nodes f-1 .. f+2; the primitive reconstructions run with ngg = 2, Parameter.cpp:194-248);
// minmod keeps the reference's sgn(0) = +1 (air_math.cuh).
template <int NS>
__device__ __forceinline__ void pv_reconstruct_mix(const double (*st)[5 + Spec<NS>::A], int nv, int recon, double *pl,
                                                   double *pr) {
  const int ns = nv - 5;
  const double k1 = 1.0 - 1.0 / 3.0, k2 = 1.0 + 1.0 / 3.0;
  for (int l = 0; l < nv; ++l) {
    const double a = st[1][l], bq = st[2][l];
    if (recon == 2 || recon == 3) {
      const double di = a - st[0][l], di1 = bq - a, di2 = st[3][l] - bq;
      if (recon == 2) {
        pl[l] = a + 0.25 * (k1 * minmod(di, di1) + k2 * minmod(di1, di));
        pr[l] = bq - 0.25 * (k1 * minmod(di2, di1) + k2 * minmod(di1, di2));
      } else {
        pl[l] = a + 0.5 * minmod(di, di1);
        pr[l] = bq - 0.5 * minmod(di1, di2);
      }
    } else {
      pl[l] = a;
      pr[l] = bq;
    }
  }
  double el = 0.5 * (pl[1] * pl[1] + pl[2] * pl[2] + pl[3] * pl[3]);
  double er = 0.5 * (pr[1] * pr[1] + pr[2] * pr[2] + pr[3] * pr[3]);
  double mw_inv_l = 0, mw_inv_r = 0;
  for (int l = 0; l < ns; ++l) {
    mw_inv_l += pl[5 + l] / c_mix.mw[l];
    mw_inv_r += pr[5 + l] / c_mix.mw[l];
  }
  const double t_l = pl[4] / (pl[0] * kRuD * mw_inv_l);
  const double t_r = pr[4] / (pr[0] * kRuD * mw_inv_r);
  double hl[Spec<NS>::A], hr[Spec<NS>::A], cpl_i[Spec<NS>::A], cpr_i[Spec<NS>::A];
  mix_h_cp<NS>(t_l, hl, cpl_i);
  mix_h_cp<NS>(t_r, hr, cpr_i);
  double cpl = 0, cpr = 0, cvl = 0, cvr = 0;
  for (int l = 0; l < ns; ++l) {
    cpl += cpl_i[l] * pl[l + 5];
    cpr += cpr_i[l] * pr[l + 5];
    cvl += pl[l + 5] * (cpl_i[l] - kRuD / c_mix.mw[l]);
    cvr += pr[l + 5] * (cpr_i[l] - kRuD / c_mix.mw[l]);
    el += hl[l] * pl[l + 5];
    er += hr[l] * pr[l + 5];
  }
  pl[nv] = pl[0] * el - pl[4];
  pr[nv] = pr[0] * er - pr[4];
  pl[nv + 1] = cpl / cvl;
  pr[nv + 1] = cpr / cvr;
}

// riemannSolver_ausmPlus<mixture> (RiemannSolver.cuh:9-96): the air steps with each side's gamma and the
// species convected with the upwind side's mass fractions.
template <int NS>
__device__ __forceinline__ void ausm_mix(const double *pl, const double *pr, const double *mt0, const double *mt1,
                                         double j0, double j1, int nv, double *fc) {
  const double k1 = 0.5 * (j0 * mt0[0] + j1 * mt1[0]);
  const double k2 = 0.5 * (j0 * mt0[1] + j1 * mt1[1]);
  const double k3 = 0.5 * (j0 * mt0[2] + j1 * mt1[2]);
  const double gkj = sqrt(k1 * k1 + k2 * k2 + k3 * k3);
  const double ul = (k1 * pl[1] + k2 * pl[2] + k3 * pl[3]) / gkj;
  const double ur = (k1 * pr[1] + k2 * pr[2] + k3 * pr[3]) / gkj;
  const double p_l = pl[4], p_r = pr[4], rho_l = pl[0], rho_r = pr[0];
  const double c = 0.5 * (sqrt(pl[nv + 1] * p_l / rho_l) + sqrt(pr[nv + 1] * p_r / rho_r));
  const double mach_l = ul / c, mach_r = ur / c;
  double mlp, mrn, plp, prn;
  const double alpha = 3 / 16.0;
  if (fabs(mach_l) > 1) {
    mlp = 0.5 * (mach_l + fabs(mach_l));
    plp = mlp / mach_l;
  } else {
    const double a = (mach_l + 1) * (mach_l + 1) * 0.25;
    const double b = (mach_l * mach_l - 1) * (mach_l * mach_l - 1);
    mlp = a + 0.125 * b;
    plp = a * (2 - mach_l) + alpha * mach_l * b;
  }
  if (fabs(mach_r) > 1) {
    mrn = 0.5 * (mach_r - fabs(mach_r));
    prn = mrn / mach_r;
  } else {
    const double a = (mach_r - 1) * (mach_r - 1) * 0.25;
    const double b = (mach_r * mach_r - 1) * (mach_r * mach_r - 1);
    mrn = -a - 0.125 * b;
    prn = a * (2 + mach_r) - alpha * mach_r * b;
  }
  const double p_coeff = plp * p_l + prn * p_r;
  const double m_half = mlp + mrn;
  const double mach_pos = 0.5 * (m_half + fabs(m_half));
  const double mach_neg = 0.5 * (m_half - fabs(m_half));
  const double mass_flux = c * (rho_l * mach_pos + rho_r * mach_neg);
  const double coeff = mass_flux * gkj;
  const double *q = mass_flux >= 0 ? pl : pr;
  fc[0] = coeff;
  fc[1] = coeff * q[1] + p_coeff * k1;
  fc[2] = coeff * q[2] + p_coeff * k2;
  fc[3] = coeff * q[3] + p_coeff * k3;
  fc[4] = coeff * (q[nv] + q[4]) / q[0];
  for (int l = 5; l < nv; ++l) fc[l] = coeff * q[l];
}

// Roe-averaged mixture temperature, gamma, speed of sound, molecular weight and species enthalpies
// (riemannSolver_hllc / riemannSolver_Roe mixture branches, RiemannSolver.cuh:118-137, 316-336); the HLLC
// form divides the weighted temperature sum once, the Roe form scales it by 1 / (sqrt rho_l + sqrt rho_r).
template <int NS>
__device__ __forceinline__ void roe_mixture_sound(const double *svm, double tl, double tr, double wl, double wr,
                                                  double wsum_inv, bool hllc_form, int ns, double &gamma, double &c,
                                                  double &mw, double *h_i) {
  double mw_inv = 0;
  for (int l = 0; l < ns; ++l) mw_inv += svm[l] / c_mix.mw[l];
  const double t = hllc_form ? (wl * tl + wr * tr) / (kRuD * mw_inv) : (wl * tl + wr * tr) * wsum_inv / (kRuD * mw_inv);
  double cp_i[Spec<NS>::A];
  mix_h_cp<NS>(t, h_i, cp_i);
  double cv = 0, cp = 0;
  for (int l = 0; l < ns; ++l) {
    cp += cp_i[l] * svm[l];
    cv += svm[l] * (cp_i[l] - kRuD / c_mix.mw[l]);
  }
  gamma = cp / cv;
  c = sqrt(gamma * kRuD * mw_inv * t);
  mw = 1.0 / mw_inv;
}

// riemannSolver_hllc<mixture> (RiemannSolver.cuh:98-230)
template <int NS>
__device__ __forceinline__ void hllc_mix(const double *pl, const double *pr, const double *mt0, const double *mt1,
                                         double j0, double j1, int nv, double *fc) {
  const int ns = nv - 5;
  const double rl_c = sqrt(pl[0]) / (sqrt(pl[0]) + sqrt(pr[0])), rr_c = sqrt(pr[0]) / (sqrt(pl[0]) + sqrt(pr[0]));
  const double u_t = pl[1] * rl_c + pr[1] * rr_c, v_t = pl[2] * rl_c + pr[2] * rr_c, w_t = pl[3] * rl_c + pr[3] * rr_c;
  double svm[Spec<NS>::A];
  for (int l = 0; l < ns; ++l) svm[l] = rl_c * pl[l + 5] + rr_c * pr[l + 5];
  double gamma, c_t, mw, h_i[Spec<NS>::A];
  roe_mixture_sound<NS>(svm, pl[4] / pl[0], pr[4] / pr[0], rl_c, rr_c, 0.0, true, ns, gamma, c_t, mw, h_i);
  const double kx = 0.5 * (mt0[0] + mt1[0]), ky = 0.5 * (mt0[1] + mt1[1]), kz = 0.5 * (mt0[2] + mt1[2]);
  const double gradK = sqrt(kx * kx + ky * ky + kz * kz);
  const double U_t = (kx * u_t + ky * v_t + kz * w_t) / gradK;
  const double jac_ave = 0.5 * (j0 + j1);
  const double Ul = kx * pl[1] + ky * pl[2] + kz * pl[3];
  const double cl = sqrt(pl[nv + 1] * pl[4] / pl[0]);
  const double sl = fmin(Ul / gradK - cl, U_t - c_t);
  if (sl >= 0) {
    const double rhoUk = pl[0] * Ul;
    fc[0] = jac_ave * rhoUk;
    fc[1] = jac_ave * (rhoUk * pl[1] + pl[4] * kx);
    fc[2] = jac_ave * (rhoUk * pl[2] + pl[4] * ky);
    fc[3] = jac_ave * (rhoUk * pl[3] + pl[4] * kz);
    fc[4] = jac_ave * ((pl[nv] + pl[4]) * Ul);
    for (int l = 5; l < nv; ++l) fc[l] = jac_ave * rhoUk * pl[l];
    return;
  }
  const double Ur = kx * pr[1] + ky * pr[2] + kz * pr[3];
  const double cr = sqrt(pr[nv + 1] * pr[4] / pr[0]);
  const double sr = fmax(Ur / gradK + cr, U_t + c_t);
  if (sr < 0) {
    const double rhoUk = pr[0] * Ur;
    fc[0] = jac_ave * rhoUk;
    fc[1] = jac_ave * (rhoUk * pr[1] + pr[4] * kx);
    fc[2] = jac_ave * (rhoUk * pr[2] + pr[4] * ky);
    fc[3] = jac_ave * (rhoUk * pr[3] + pr[4] * kz);
    fc[4] = jac_ave * ((pr[nv] + pr[4]) * Ur);
    for (int l = 5; l < nv; ++l) fc[l] = jac_ave * rhoUk * pr[l];
    return;
  }
  const double sm = ((pr[0] * Ur * (sr - Ur / gradK) - pl[0] * Ul * (sl - Ul / gradK)) / gradK + pl[4] - pr[4]) /
                    (pr[0] * (sr - Ur / gradK) - pl[0] * (sl - Ul / gradK));
  const double pm = pl[0] * (sl - Ul / gradK) * (sm - Ul / gradK) + pl[4];
  const double *q = sm >= 0 ? pl : pr;
  const double s = sm >= 0 ? sl : sr, Uq = sm >= 0 ? Ul : Ur;
  const double pCoeff = 1.0 / (s - sm);
  const double QCoeff = jac_ave * pCoeff * sm * (s * gradK - Uq) * q[0];
  fc[0] = QCoeff;
  const double dP = (s * pm - sm * q[4]) * pCoeff * jac_ave;
  fc[1] = QCoeff * q[1] + dP * kx;
  fc[2] = QCoeff * q[2] + dP * ky;
  fc[3] = QCoeff * q[3] + dP * kz;
  fc[4] = QCoeff * q[nv] / q[0] + pCoeff * jac_ave * (s * pm * sm * gradK - sm * q[4] * Uq);
  for (int l = 5; l < nv; ++l) fc[l] = QCoeff * q[l];
}

// compute_half_sum_left_right_flux + riemannSolver_Roe<mixture> (RiemannSolver.cuh:232-417); d0, d1:
// the entropy-fix thresholds of the face's two nodes.
template <int NS>
__device__ __forceinline__ void roe_mix(const double *pl, const double *pr, const double *mt0, const double *mt1,
                                        double j0, double j1, double d0, double d1, int nv, double *fc) {
  const int ns = nv - 5;
  double JacKx = j0 * mt0[0], JacKy = j0 * mt0[1], JacKz = j0 * mt0[2];
  double Uk = pl[1] * JacKx + pl[2] * JacKy + pl[3] * JacKz;
  double coeff = Uk * pl[0];
  fc[0] = 0.5 * coeff;
  fc[1] = 0.5 * (coeff * pl[1] + pl[4] * JacKx);
  fc[2] = 0.5 * (coeff * pl[2] + pl[4] * JacKy);
  fc[3] = 0.5 * (coeff * pl[3] + pl[4] * JacKz);
  fc[4] = 0.5 * Uk * (pl[4] + pl[nv]);
  for (int l = 5; l < nv; ++l) fc[l] = 0.5 * coeff * pl[l];
  JacKx = j1 * mt1[0];
  JacKy = j1 * mt1[1];
  JacKz = j1 * mt1[2];
  Uk = pr[1] * JacKx + pr[2] * JacKy + pr[3] * JacKz;
  coeff = Uk * pr[0];
  fc[0] += 0.5 * coeff;
  fc[1] += 0.5 * (coeff * pr[1] + pr[4] * JacKx);
  fc[2] += 0.5 * (coeff * pr[2] + pr[4] * JacKy);
  fc[3] += 0.5 * (coeff * pr[3] + pr[4] * JacKz);
  fc[4] += 0.5 * Uk * (pr[4] + pr[nv]);
  for (int l = 5; l < nv; ++l) fc[l] += 0.5 * coeff * pr[l];

  const double dl = sqrt(pl[0]), dr = sqrt(pr[0]);
  const double inv_den = 1.0 / (dl + dr);
  const double u = (dl * pl[1] + dr * pr[1]) * inv_den;
  const double v = (dl * pl[2] + dr * pr[2]) * inv_den;
  const double w = (dl * pl[3] + dr * pr[3]) * inv_den;
  const double ek = 0.5 * (u * u + v * v + w * w);
  const double hl = (pl[nv] + pl[4]) / pl[0];
  const double hr = (pr[nv] + pr[4]) / pr[0];
  const double h = (dl * hl + dr * hr) * inv_den;
  double svm[Spec<NS>::A];
  for (int l = 0; l < ns; ++l) svm[l] = (dl * pl[l + 5] + dr * pr[l + 5]) * inv_den;
  double gamma, c, mw, h_i[Spec<NS>::A];
  roe_mixture_sound<NS>(svm, pl[4] / pl[0], pr[4] / pr[0], dl, dr, inv_den, false, ns, gamma, c, mw, h_i);
  double kx = 0.5 * (mt0[0] + mt1[0]), ky = 0.5 * (mt0[1] + mt1[1]), kz = 0.5 * (mt0[2] + mt1[2]);
  const double gradK = sqrt(kx * kx + ky * ky + kz * kz);
  double Ukk = kx * u + ky * v + kz * w;
  double ch3[3] = {Ukk - gradK * c, Ukk, Ukk + gradK * c};
  const double ed = 0.5 * (d0 + d1);
  for (int q = 0; q < 3; ++q) {
    ch3[q] = fabs(ch3[q]);
    if (ch3[q] < ed) ch3[q] = 0.5 * (ch3[q] * ch3[q] / ed + ed);
  }
  kx /= gradK;
  ky /= gradK;
  kz /= gradK;
  Ukk /= gradK;
  const double jac_ave = 0.5 * (j0 + j1);
  double dq[5 + Spec<NS>::A];
  dq[0] = jac_ave * (pr[0] - pl[0]);
  for (int l = 1; l < nv; ++l) dq[l] = jac_ave * (pr[0] * pr[l] - pl[0] * pl[l]);
  dq[4] = jac_ave * (pr[nv] - pl[nv]);
  double c1 = (gamma - 1) * (ek * dq[0] - u * dq[1] - v * dq[2] - w * dq[3] + dq[4]) / (c * c);
  double c2 = (kx * dq[1] + ky * dq[2] + kz * dq[3] - Ukk * dq[0]) / c;
  for (int l = 0; l < ns; ++l) c1 += (mw / c_mix.mw[l] - h_i[l] * (gamma - 1) / (c * c)) * dq[l + 5];
  double c3 = dq[0] - c1;
  double LDq[5 + Spec<NS>::A];
  LDq[0] = 0.5 * (c1 - c2);
  LDq[1] = kx * c3 - ((kz * v - ky * w) * dq[0] - kz * dq[2] + ky * dq[3]) / c;
  LDq[2] = ky * c3 - ((kx * w - kz * u) * dq[0] - kx * dq[3] + kz * dq[1]) / c;
  LDq[3] = kz * c3 - ((ky * u - kx * v) * dq[0] - ky * dq[1] + kx * dq[2]) / c;
  LDq[4] = 0.5 * (c1 + c2);
  for (int l = 0; l < ns; ++l) LDq[l + 5] = dq[l + 5] - svm[l] * dq[0];
  double *b = dq;
  b[0] = -ch3[0] * LDq[0];
  for (int l = 1; l < nv; ++l) b[l] = -ch3[1] * LDq[l];
  b[4] = -ch3[2] * LDq[4];
  const double c0 = kx * b[1] + ky * b[2] + kz * b[3];
  c1 = c0 + b[0] + b[4];
  c2 = c * (b[4] - b[0]);
  c3 = 0;
  for (int l = 0; l < ns; ++l) c3 += (h_i[l] - mw / c_mix.mw[l] * c * c / (gamma - 1)) * b[l + 5];
  fc[0] += 0.5 * c1;
  fc[1] += 0.5 * (u * c1 + kx * c2 - c * (kz * b[2] - ky * b[3]));
  fc[2] += 0.5 * (v * c1 + ky * c2 - c * (kx * b[3] - kz * b[1]));
  fc[3] += 0.5 * (w * c1 + kz * c2 - c * (ky * b[1] - kx * b[2]));
  fc[4] += 0.5 * (h * c1 + Ukk * c2 - c * c * c0 / (gamma - 1) +
                  c * ((kz * v - ky * w) * b[1] + (kx * w - kz * u) * b[2] + (ky * u - kx * v) * b[3]) + c3);
  for (int l = 0; l < ns; ++l) fc[5 + l] += 0.5 * (b[l + 5] + svm[l] * c1);
}

// compute_entropy_fix_delta<mixture> (InviscidScheme.cu:417-456) over nodes -1 .. m of every direction,
// with the node's mixture speed of sound; into efd (padded layout).
__global__ void k_efix_mix(DevBlock b, DevState s, double factor, double *__restrict__ efd) {
  const int ex = b.mx + 2, ey = b.my + 2, ez = b.mz > 1 ? b.mz + 2 : 1;
  const long long tot = (long long)ex * ey * ez;
  const long long P = b.plane;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < tot; n += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(n % ex) - 1;
    const long long r = n / ex;
    const int j = (int)(r % ey) - 1, k = b.mz > 1 ? (int)(r / ey) - 1 : 0;
    const long long p = b.id(i, j, k);
    double m[9];
    for (int q = 0; q < 9; ++q) m[q] = b.met[q * P + p];
    const double u = s.bv[P + p], v = s.bv[2 * P + p], w = s.bv[3 * P + p];
    const double U = fabs(u * m[0] + v * m[1] + w * m[2]);
    const double V = fabs(u * m[3] + v * m[4] + w * m[5]);
    const double W = fabs(u * m[6] + v * m[7] + w * m[8]);
    const double kx = sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
    const double ky = sqrt(m[3] * m[3] + m[4] * m[4] + m[5] * m[5]);
    const double kz = sqrt(m[6] * m[6] + m[7] * m[7] + m[8] * m[8]);
    const double c = s.acs[p];
    efd[p] = b.mz == 1 ? factor * (U + V + c * 0.5 * (kx + ky)) : factor * (U + V + W + c * (kx + ky + kz) / 3.0);
  }
}

// Faces of sweep DIR: face f (between nodes f and f+1, f = -1 .. n-1) sits at index f + 1 along the
// sweep in an (mx + [DIR==0]) x (my + [DIR==1]) x (mz + [DIR==2]) array, i fastest; fcb[l * count + id].
template <int DIR>
__host__ __device__ __forceinline__ long long pv_face_count(const DevBlock &b) {
  return (long long)(b.mx + (DIR == 0)) * (b.my + (DIR == 1)) * (b.mz + (DIR == 2));
}

template <int NS, int DIR>
__global__ void __launch_bounds__(128) k_pv_mix_face(DevBlock b, DevState s, int nv, int recon, int rs,
                                                   const double *__restrict__ efd, double *__restrict__ fcb) {
  const int ex = b.mx + (DIR == 0), ey = b.my + (DIR == 1);
  const long long nf = pv_face_count<DIR>(b);
  const long long P = b.plane;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < nf; n += (long long)gridDim.x * blockDim.x) {
    int i = (int)(n % ex);
    const long long r = n / ex;
    int j = (int)(r % ey), k = (int)(r / ey);
    // face index along the sweep starts at -1
    if (DIR == 0) i -= 1;
    else if (DIR == 1) j -= 1;
    else k -= 1;
    const int e0 = DIR == 0, e1 = DIR == 1, e2 = DIR == 2;
    double st[4][5 + Spec<NS>::A];
    for (int m = 0; m < 4; ++m) {
      const long long p = b.id(i + (m - 1) * e0, j + (m - 1) * e1, k + (m - 1) * e2);
      for (int l = 0; l < 5; ++l) st[m][l] = s.bv[l * P + p];
      for (int l = 0; l < nv - 5; ++l) st[m][5 + l] = s.sv[l * P + p];
    }
    const long long p0 = b.id(i, j, k), p1 = b.id(i + e0, j + e1, k + e2);
    double mt0[3], mt1[3];
    for (int q = 0; q < 3; ++q) {
      mt0[q] = b.met[(DIR * 3 + q) * P + p0];
      mt1[q] = b.met[(DIR * 3 + q) * P + p1];
    }
    double pl[PvMix<NS>::V], pr[PvMix<NS>::V], fc[5 + Spec<NS>::A];
    pv_reconstruct_mix<NS>(st, nv, recon, pl, pr);
    if (rs == 2) roe_mix<NS>(pl, pr, mt0, mt1, b.jac[p0], b.jac[p1], efd[p0], efd[p1], nv, fc);
    else if (rs == 4) hllc_mix<NS>(pl, pr, mt0, mt1, b.jac[p0], b.jac[p1], nv, fc);
    else ausm_mix<NS>(pl, pr, mt0, mt1, b.jac[p0], b.jac[p1], nv, fc);
    for (int l = 0; l < nv; ++l) fcb[l * nf + n] = fc[l];
  }
}

// dq -= fc(i+1/2) - fc(i-1/2) for every node of sweep DIR (compute_convective_term_pv_1D's last step).
template <int DIR>
__global__ void k_pv_mix_diff(DevBlock b, int nv, const double *__restrict__ fcb, double *__restrict__ dq) {
  const long long nf = pv_face_count<DIR>(b);
  const int ex = b.mx + (DIR == 0), ey = b.my + (DIR == 1);
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < b.n; n += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(n % b.mx);
    const long long r = n / b.mx;
    const int j = (int)(r % b.my), k = (int)(r / b.my);
    // face f of this node's right side is f = node index; stored at index node + 1 along the sweep
    const int fi = DIR == 0 ? i + 1 : i, fj = DIR == 1 ? j + 1 : j, fk = DIR == 2 ? k + 1 : k;
    const long long fr = ((long long)fk * ey + fj) * ex + fi;
    const long long fl = fr - (DIR == 0 ? 1 : DIR == 1 ? (long long)ex : (long long)ex * ey);
    for (int l = 0; l < nv; ++l) dq[l * b.n + n] -= fcb[l * nf + fr] - fcb[l * nf + fl];
  }
}

}  // namespace ostc
