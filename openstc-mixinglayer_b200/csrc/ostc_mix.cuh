// ostc_mix.cuh -- kernels of the multi-component path (species = 1; included by ostc_b200.cu after
// DevBlock/DevState).  Per RK stage (RK.cuh:112-172): the chemical source initialises dq, the
// flux-split WENO7 sweeps and the viscous sweeps accumulate into it, the update kernel combines the
// stage and solves the temperature, the boundary faces fill the ghosts, and the properties kernel
// recomputes gamma, c, mu, lambda and rho*D over the padded block.
#pragma once

#include "mix_math.cuh"

namespace ostc {

// compute_cv_from_bv_1_point<mixture> (FieldOperation.cuh:78-105, total energy :17-32)
template <int NS>
__device__ __forceinline__ void mix_cv_from_bv_node(const DevBlock &b, const DevState &s, long long p) {
  const long long P = b.plane;
  const int ns = OSTC_NS;
  const double rho = s.bv[p], u = s.bv[P + p], v = s.bv[2 * P + p], w = s.bv[3 * P + p];
  s.cv[p] = rho;
  s.cv[P + p] = rho * u;
  s.cv[2 * P + p] = rho * v;
  s.cv[3 * P + p] = rho * w;
  double h[Spec<NS>::A];
  mix_h_cp<NS, double>(s.bv[5 * P + p], h, nullptr);
  double te = 0.5 * (u * u + v * v + w * w);
  for (int l = 0; l < ns; ++l) {
    const double y = s.sv[l * P + p];
    s.cv[(5 + l) * P + p] = rho * y;
    te += h[l] * y;
  }
  te *= rho;
  te -= s.bv[4 * P + p];
  s.cv[4 * P + p] = te;
}

// update_physical_properties<mixture> over every padded node (FieldOperation.cuh:107-134), with the
// node's state read in FP64 and the properties evaluated in T (FP32 in the mixed precision mode).
// FP32 at four resident blocks (128 registers) measured 1.4 ms per step faster than uncapped; FP64
// is fastest uncapped.
template <int NS, typename T>
__global__ void __launch_bounds__(128, sizeof(T) == 8 ? 1 : 4) k_mix_props(DevBlock b, DevState s) {
  const long long P = b.plane;
  const int ns = OSTC_NS;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < P; p += (long long)gridDim.x * blockDim.x) {
    const double rho = s.bv[p];
    if (!(rho > 0)) continue;  // padding columns of the row pitch carry no state
    T y[Spec<NS>::A], rd[Spec<NS>::A];
    for (int l = 0; l < ns; ++l) y[l] = (T)s.sv[l * P + p];
    T g, a, mu, cd;
    mix_properties<NS, T>((T)rho, (T)s.bv[4 * P + p], (T)s.bv[5 * P + p], y, g, a, mu, cd, rd);
    s.gam[p] = g;
    s.acs[p] = a;
    s.mul[p] = mu;
    s.cond[p] = cd;
    for (int l = 0; l < ns; ++l) s.rhod[l * P + p] = rd[l];
  }
}

// conservative variables from bv and sv over the padded block (initialisation, RK.cuh:37-45)
template <int NS>
__global__ void k_mix_init_cv(DevBlock b, DevState s) {
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < b.plane; p += (long long)gridDim.x * blockDim.x)
    if (s.bv[p] > 0) mix_cv_from_bv_node<NS>(b, s, p);
}

// compute_source<FR> (SourceTerm.cuh:11-35) as the first contribution to dq: dq[5+l] = J omega_l
// (finite rate) or 0, dq[0..4] = 0.
template <int NS>
__global__ void __launch_bounds__(128, 4) k_mix_source(DevBlock b, DevState s, double *__restrict__ dq, int nv,
                                                     int finite_rate) {
  if (NS > 0) nv = 5 + NS;
  const long long P = b.plane;
  const int ns = OSTC_NS;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < b.n; n += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(n % b.mx);
    const long long r = n / b.mx;
    const int j = (int)(r % b.my), k = (int)(r / b.my);
    const long long p = b.id(i, j, k);
    for (int l = 0; l < 5; ++l) dq[l * b.n + n] = 0.0;
    if (finite_rate) {
      double y[Spec<NS>::A], om[Spec<NS>::A];
      for (int l = 0; l < ns; ++l) y[l] = s.sv[l * P + p];
      mix_chemistry<NS>(s.bv[p], s.bv[5 * P + p], y, om);
      const double jac = b.jac[p];
      for (int l = 0; l < ns; ++l) dq[(5 + l) * b.n + n] = jac * om[l];
    } else {
      for (int l = 5; l < nv; ++l) dq[l * b.n + n] = 0.0;
    }
  }
}

// Point-implicit chemistry (chem mode 1, an extension of the RK3 path): after the fluxes, add the
// chemical source J omega to dq and replace the species part by the solution of
// (I - dt J_chem) x = dq_species (EPI + solve_chem_system, FiniteRateChem.cu:233-254, 302-357, with the
// stage's global dt), one cell per thread, every cell of the block in one launch.
template <int NS>
__global__ void __launch_bounds__(128, 4) k_mix_chem_epi(DevBlock b, DevState s, double *__restrict__ dq,
                                                       const double *dtp) {
  const long long P = b.plane;
  const int ns = OSTC_NS;
  const double dt = *dtp;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < b.n; n += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(n % b.mx);
    const long long r = n / b.mx;
    const int j = (int)(r % b.my), k = (int)(r / b.my);
    const long long p = b.id(i, j, k);
    double y[Spec<NS>::A], om[Spec<NS>::A], jc[Spec<NS>::A * Spec<NS>::A], rhs[Spec<NS>::A];
    for (int l = 0; l < ns; ++l) y[l] = s.sv[l * P + p];
    for (int l = 0; l < ns * ns; ++l) jc[l] = 0.0;
    mix_chemistry<NS>(s.bv[p], s.bv[5 * P + p], y, om, jc);
    const double jac = b.jac[p];
    for (int l = 0; l < ns; ++l) rhs[l] = dq[(5 + l) * b.n + n] + jac * om[l];
    for (int m = 0; m < ns; ++m)
      for (int q = 0; q < ns; ++q) jc[m * ns + q] = (m == q ? 1.0 : 0.0) - dt * jc[m * ns + q];
    mix_lu_solve<NS>(jc, rhs);
    for (int l = 0; l < ns; ++l) dq[(5 + l) * b.n + n] = rhs[l];
  }
}

// ------------------------------------------------------------------ flux-split WENO7 sweeps

// Tile geometry of the sweeps: TD faces along the sweep direction (TD-1 nodes finalised per tile),
// and for the y / z sweeps TXL consecutive i per tile (coalesced rows).
template <int DIR> struct FvsTile {
  static constexpr int TXL = DIR == 0 ? 1 : 8;
  static constexpr int TD = DIR == 0 ? 128 : 16;
  static constexpr int NST = TD + 7;  // staged nodes: stencils of 8 nodes around TD faces
};

template <int DIR, typename T>
__host__ __device__ constexpr size_t fvs_smem_bytes(int nv) {
  return (size_t)FvsTile<DIR>::NST * FvsTile<DIR>::TXL * nv * 2 * sizeof(T);
}

// compute_convective_term_weno_x/_y/_z (WENO.cu:8-461) for inviscid_scheme 72 (characteristic,
// compute_weno_flux_ch method 1, WENO.cu:722-758, 899-965, 1119-1142) or 71 (component-wise,
// compute_weno_flux_cp, :1455-1536).  Every node's split fluxes F+- (compute_flux, :697-720) are
// computed once into shared memory; each thread then forms one face flux from the 8-node stencil,
// and after a barrier the node threads difference neighbouring faces into dq.  T is the arithmetic
// type of the fluxes (FP32 in the mixed precision mode: state read in FP64, dq accumulated in FP64).
// Resident blocks per SM (measured on the 384 x 192 x 96 layer): FP64 4; FP32 8 (64 registers, some
// spills; 6, 7 and 8 blocks ran the mixed step in 79.5, 77.0 and 76.9 ms against 84.6 ms at 4).
template <int DIR, int NS, typename T>
__global__ void __launch_bounds__(FvsTile<DIR>::TD * FvsTile<DIR>::TXL, sizeof(T) == 8 ? 4 : 8) k_fvs(DevBlock b, DevState s,
                                                                               double *__restrict__ dq, int nv,
                                                                               int scheme) {
  constexpr int TXL = FvsTile<DIR>::TXL, TD = FvsTile<DIR>::TD, NST = FvsTile<DIR>::NST;
  extern __shared__ __align__(16) unsigned char mix_smem[];
  T *fsm = reinterpret_cast<T *>(mix_smem);
  T *Fp = fsm;                        // [NST][TXL][nv]
  T *Fm = fsm + NST * TXL * nv;       // [NST][TXL][nv]
  const int lane = DIR == 0 ? 0 : (int)threadIdx.x;
  const int t = DIR == 0 ? (int)threadIdx.x : (int)threadIdx.y;
  const int ns = OSTC_NS;
  if (NS > 0) nv = 5 + NS;
  const long long P = b.plane;
  const int nd = DIR == 0 ? b.mx : DIR == 1 ? b.my : b.mz;
  const int start = (DIR == 0 ? blockIdx.x : blockIdx.y) * (TD - 1);
  int i0, j0, k0;  // coordinates of this lane's line
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
  const T half = T(0.5);
  // stage split fluxes of nodes start-4 .. start+TD+2
  if (lane_ok) {
    for (int st = t; st < NST; st += TD) {
      const int n = start - 4 + st;
      if (n > nd + 3) continue;
      const long long p = pid(n);
      T Q[Spec<NS>::A + 5];
      for (int l = 0; l < nv; ++l) Q[l] = (T)s.cv[l * P + p];
      const T pk = (T)s.bv[4 * P + p];
      const T c = (T)(s.acs ? s.acs[p] : sqrt(kGamma * (kRuD / kMwD) * s.bv[5 * P + p]));
      const T k0m = (T)b.met[(DIR * 3 + 0) * P + p], k1m = (T)b.met[(DIR * 3 + 1) * P + p],
              k2m = (T)b.met[(DIR * 3 + 2) * P + p];
      const T jac = (T)b.jac[p];
      const T Uk = (Q[1] * k0m + Q[2] * k1m + Q[3] * k2m) / Q[0];
      const T cg = c * tsqrt(k0m * k0m + k1m * k1m + k2m * k2m);
      const T l0 = tabs(Uk) + cg;
      T *fp = Fp + ((long long)st * TXL + lane) * nv, *fm = Fm + ((long long)st * TXL + lane) * nv;
      fp[0] = half * jac * (Uk * Q[0] + l0 * Q[0]);
      fp[1] = half * jac * (Uk * Q[1] + pk * k0m + l0 * Q[1]);
      fp[2] = half * jac * (Uk * Q[2] + pk * k1m + l0 * Q[2]);
      fp[3] = half * jac * (Uk * Q[3] + pk * k2m + l0 * Q[3]);
      fp[4] = half * jac * (Uk * (Q[4] + pk) + l0 * Q[4]);
      fm[0] = half * jac * (Uk * Q[0] - l0 * Q[0]);
      fm[1] = half * jac * (Uk * Q[1] + pk * k0m - l0 * Q[1]);
      fm[2] = half * jac * (Uk * Q[2] + pk * k1m - l0 * Q[2]);
      fm[3] = half * jac * (Uk * Q[3] + pk * k2m - l0 * Q[3]);
      fm[4] = half * jac * (Uk * (Q[4] + pk) - l0 * Q[4]);
      for (int l = 5; l < nv; ++l) {
        fp[l] = half * jac * (Uk * Q[l] + l0 * Q[l]);
        fm[l] = half * jac * (Uk * Q[l] - l0 * Q[l]);
      }
    }
  }
  __syncthreads();
  const int n = start - 1 + t;  // left node of this thread's face
  const bool face_ok = lane_ok && n < nd;
  T fc[Spec<NS>::A + 5];
  for (int l = 0; l < kMV; ++l) fc[l] = T(0);
  auto FP = [&](int m, int l) -> T { return Fp[((long long)(t + m) * TXL + lane) * nv + l]; };
  auto FM = [&](int m, int l) -> T { return Fm[((long long)(t + m) * TXL + lane) * nv + l]; };
  if (face_ok && scheme == 71) {
    const long long pl = pid(n), pr = pid(n + 1);
    const double j1 = b.jac[pl], j2 = b.jac[pr];
    double a[3];
    for (int q = 0; q < 3; ++q) a[q] = b.met[(DIR * 3 + q) * P + pl] * j1 + b.met[(DIR * 3 + q) * P + pr] * j2;
    const double eps_ref = 1e-20 * c_mix.weno_eps_scale * 0.25 * (a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
    const double e1 = eps_ref * c_mix.v_ref * c_mix.v_ref;
    const double e2 = e1 * c_mix.v_ref * c_mix.v_ref;
    for (int l = 0; l < nv; ++l) {
      const double e = (l >= 1 && l <= 3) ? e1 : (l == 4 ? e2 : eps_ref);
      T vp[7], vm[7];
      for (int m = 0; m < 7; ++m) {
        vp[m] = FP(m, l);
        vm[m] = FM(m + 1, l);
      }
      fc[l] = fvs_weno7(vp, vm, e);
    }
  } else if (face_ok) {
    // Roe-averaged mixture eigensystem at the face (WENO.cu:747-821)
    const long long pl = pid(n), pr = pid(n + 1);
    T cvl[Spec<NS>::A + 5], cvr[Spec<NS>::A + 5];
    for (int l = 0; l < nv; ++l) {
      cvl[l] = (T)s.cv[l * P + pl];
      cvr[l] = (T)s.cv[l * P + pr];
    }
    const T p_l = (T)s.bv[4 * P + pl], p_r = (T)s.bv[4 * P + pr];
    const T rli = T(1) / cvl[0], rri = T(1) / cvr[0];
    const T sl = tsqrt(cvl[0]), sr = tsqrt(cvr[0]);
    const T rlc = sl / (sl + sr), rrc = sr / (sl + sr);
    const T um = rlc * cvl[1] * rli + rrc * cvr[1] * rri;
    const T vm_ = rlc * cvl[2] * rli + rrc * cvr[2] * rri;
    const T wm = rlc * cvl[3] * rli + rrc * cvr[3] * rri;
    const T ekm = half * (um * um + vm_ * vm_ + wm * wm);
    const T hm = rlc * ((cvl[4] + p_l) * rli) + rrc * ((cvr[4] + p_r) * rri);
    T svm[Spec<NS>::A], hi[Spec<NS>::A], cpi[Spec<NS>::A], al[Spec<NS>::A];
    T mw_inv = 0;
    for (int l = 0; l < ns; ++l) {
      svm[l] = rlc * cvl[l + 5] * rli + rrc * cvr[l + 5] * rri;
      mw_inv += svm[l] / (T)c_mix.mw[l];
    }
    const T tm = (rlc * (p_l * rli) + rrc * (p_r * rri)) / (T(kRuD) * mw_inv);
    mix_h_cp<NS, T>(tm, hi, cpi);
    T cp = 0, cvt = 0;
    for (int l = 0; l < ns; ++l) {
      cp += svm[l] * cpi[l];
      cvt += svm[l] * (cpi[l] - (T)c_mix.ru_mw[l]);
    }
    const T gamma = cp / cvt;
    const T cm = tsqrt(gamma * T(kRuD) * mw_inv * tm);
    const T gm1 = gamma - 1;
    const double jld = b.jac[pl], jrd = b.jac[pr];
    const double kxJd = b.met[(DIR * 3 + 0) * P + pl] * jld + b.met[(DIR * 3 + 0) * P + pr] * jrd;
    const double kyJd = b.met[(DIR * 3 + 1) * P + pl] * jld + b.met[(DIR * 3 + 1) * P + pr] * jrd;
    const double kzJd = b.met[(DIR * 3 + 2) * P + pl] * jld + b.met[(DIR * 3 + 2) * P + pr] * jrd;
    const double eps = 1e-40 * c_mix.weno_eps_scale * 0.25 * (kxJd * kxJd + kyJd * kyJd + kzJd * kzJd);
    const T jlr = (T)(jld + jrd);
    T kx = (T)kxJd / jlr, ky = (T)kyJd / jlr, kz = (T)kzJd / jlr;
    const T gradK = tsqrt(kx * kx + ky * ky + kz * kz);
    kx /= gradK;
    ky /= gradK;
    kz /= gradK;
    const T Ukb = kx * um + ky * vm_ + kz * wm;
    const T alpha = gm1 * ekm;
    const T c2i = T(1) / (cm * cm);
    for (int l = 0; l < ns; ++l) {
      al[l] = gamma * T(kRuD) / (T)c_mix.mw[l] * tm - (gamma - 1) * hi[l];
      al[l] *= c2i;
    }
    // The species columns of the five flow rows of L are cs_l * al[q] (cs = 1/2, -kx, -ky, -kz, 1/2):
    // their products with the split fluxes share one sum per stencil node, formed once for all rows.
    T sp[7], sm[7];
    for (int m = 0; m < 7; ++m) {
      T a = 0, bq = 0;
      for (int q = 0; q < ns; ++q) {
        a += al[q] * FP(m, 5 + q);
        bq += al[q] * FM(m + 1, 5 + q);
      }
      sp[m] = a;
      sm[m] = bq;
    }
    T fch[Spec<NS>::A + 5];
    for (int l = 0; l < 5; ++l) {
      T cs = half, L[5];
      if (l == 0) {
        L[0] = (alpha + Ukb * cm) * c2i * half;
        L[1] = -(gm1 * um + kx * cm) * c2i * half;
        L[2] = -(gm1 * vm_ + ky * cm) * c2i * half;
        L[3] = -(gm1 * wm + kz * cm) * c2i * half;
        L[4] = gm1 * c2i * half;
      } else if (l == 1) {
        cs = -kx;
        L[0] = kx * (1 - alpha * c2i) - (kz * vm_ - ky * wm) / cm;
        L[1] = kx * gm1 * um * c2i;
        L[2] = (kx * gm1 * vm_ + kz * cm) * c2i;
        L[3] = (kx * gm1 * wm - ky * cm) * c2i;
        L[4] = -kx * gm1 * c2i;
      } else if (l == 2) {
        cs = -ky;
        L[0] = ky * (1 - alpha * c2i) - (kx * wm - kz * um) / cm;
        L[1] = (ky * gm1 * um - kz * cm) * c2i;
        L[2] = ky * gm1 * vm_ * c2i;
        L[3] = (ky * gm1 * wm + kx * cm) * c2i;
        L[4] = -ky * gm1 * c2i;
      } else if (l == 3) {
        cs = -kz;
        L[0] = kz * (1 - alpha * c2i) - (ky * um - kx * vm_) / cm;
        L[1] = (kz * gm1 * um + ky * cm) * c2i;
        L[2] = (kz * gm1 * vm_ - kx * cm) * c2i;
        L[3] = kz * gm1 * wm * c2i;
        L[4] = -kz * gm1 * c2i;
      } else {
        L[0] = (alpha - Ukb * cm) * c2i * half;
        L[1] = -(gm1 * um - kx * cm) * c2i * half;
        L[2] = -(gm1 * vm_ - ky * cm) * c2i * half;
        L[3] = -(gm1 * wm - kz * cm) * c2i * half;
        L[4] = gm1 * c2i * half;
      }
      T vp[7], vmn[7];
      for (int m = 0; m < 7; ++m) {
        T a = 0, bq = 0;
        for (int q = 0; q < 5; ++q) {
          a += L[q] * FP(m, q);
          bq += L[q] * FM(m + 1, q);
        }
        vp[m] = a + cs * sp[m];
        vmn[m] = bq + cs * sm[m];
      }
      fch[l] = fvs_weno7(vp, vmn, eps);
    }
    for (int l = 0; l < ns; ++l) {
      T vp[7], vmn[7];
      for (int m = 0; m < 7; ++m) {
        vp[m] = -svm[l] * FP(m, 0) + FP(m, 5 + l);
        vmn[m] = -svm[l] * FM(m + 1, 0) + FM(m + 1, 5 + l);
      }
      fch[5 + l] = fvs_weno7(vp, vmn, eps);
    }
    fc[0] = fch[0] + kx * fch[1] + ky * fch[2] + kz * fch[3] + fch[4];
    fc[1] = (um - kx * cm) * fch[0] + kx * um * fch[1] + (ky * um - kz * cm) * fch[2] + (kz * um + ky * cm) * fch[3] +
            (um + kx * cm) * fch[4];
    fc[2] = (vm_ - ky * cm) * fch[0] + (kx * vm_ + kz * cm) * fch[1] + ky * vm_ * fch[2] +
            (kz * vm_ - kx * cm) * fch[3] + (vm_ + ky * cm) * fch[4];
    fc[3] = (wm - kz * cm) * fch[0] + (kx * wm - ky * cm) * fch[1] + (ky * wm + kx * cm) * fch[2] + kz * wm * fch[3] +
            (wm + kz * cm) * fch[4];
    const T hc = hm - cm * cm / gm1;
    fc[4] = (hm - Ukb * cm) * fch[0] + (kx * hc + (kz * vm_ - ky * wm) * cm) * fch[1] +
            (ky * hc + (kx * wm - kz * um) * cm) * fch[2] + (kz * hc + (ky * um - kx * vm_) * cm) * fch[3] +
            (hm + Ukb * cm) * fch[4];
    T add = 0;
    const T ca = fch[0] + kx * fch[1] + ky * fch[2] + kz * fch[3] + fch[4];
    for (int l = 0; l < ns; ++l) {
      fc[5 + l] = svm[l] * ca + fch[l + 5];
      add += al[l] * fch[l + 5];
    }
    fc[4] -= add * cm * cm / gm1;
  }
  __syncthreads();  // every thread is done with the staged fluxes: reuse them for the face fluxes
  T *fcs = fsm;  // [TD][TXL][nv]
  for (int l = 0; l < nv; ++l) fcs[((long long)t * TXL + lane) * nv + l] = fc[l];
  __syncthreads();
  if (face_ok && t >= 1) {
    const long long q = DIR == 0 ? b.iq(n, j0, k0) : DIR == 1 ? b.iq(i0, n, k0) : b.iq(i0, j0, n);
    for (int l = 0; l < nv; ++l)
      dq[l * b.n + q] -= (double)(fc[l] - fcs[((long long)(t - 1) * TXL + lane) * nv + l]);
  }
}

// ------------------------------------------------------------------ viscous sweeps (mixtures)

// compute_fv/gv/hv_2nd_order<mixture, Laminar> (ViscousScheme.cuh:24-318 and its y / z twins) at the
// face between node p0 and its neighbour p0 + e[d]: stress, Fourier conduction with the mixture
// conductivity, mixture-averaged species diffusion with the correction velocity and its enthalpy flux.
// The node differences of each gradient are taken in FP64 (they cancel the leading digits); the
// chain rule and the fluxes run in T.
template <bool DIM3, int NS, typename T>
__device__ __forceinline__ void mix_visc_face(const DevBlock &b, const DevState &s, long long p0, int d, int nv,
                                              T *fv) {
  const long long P = b.plane;
  const long long st[3] = {1, b.pitch, (long long)b.pitch * b.sy};
  const long long p1 = b.chk(p0 + st[d]);
  const T half = T(0.5);
  T m[9];
  for (int r = 0; r < 9; ++r) m[r] = (T)(0.5 * (b.met[r * P + p0] + b.met[r * P + p1]));
  // gradient of plane B at the face: 2-point normal difference, 4-point averages across
  auto grad = [&](const double *B, T *out) {
    T g[3];
    for (int c = 0; c < 3; ++c) {
      if (c == d) {
        g[c] = (T)(B[p1] - B[p0]);
      } else if (c == 2 && !DIM3) {
        g[c] = T(0);
      } else {
        const long long a = st[c];
        g[c] = (T)(0.25 * (B[p0 + a] - B[p0 - a] + B[p1 + a] - B[p1 - a]));
      }
    }
    out[0] = g[0] * m[0] + g[1] * m[3] + g[2] * m[6];
    out[1] = g[0] * m[1] + g[1] * m[4] + g[2] * m[7];
    out[2] = g[0] * m[2] + g[1] * m[5] + g[2] * m[8];
  };
  T gu[3], gv[3], gw[3], gt[3];
  grad(s.bv + P, gu);
  grad(s.bv + 2 * P, gv);
  grad(s.bv + 3 * P, gw);
  grad(s.bv + 5 * P, gt);
  const T mul = (T)(0.5 * (s.mul[p0] + s.mul[p1]));
  const T txx = mul * (4 * gu[0] - 2 * gv[1] - 2 * gw[2]) / T(3);
  const T tyy = mul * (4 * gv[1] - 2 * gu[0] - 2 * gw[2]) / T(3);
  const T tzz = mul * (4 * gw[2] - 2 * gu[0] - 2 * gv[1]) / T(3);
  const T txy = mul * (gu[1] + gv[0]);
  const T txz = mul * (gu[2] + gw[0]);
  const T tyz = mul * (gv[2] + gw[1]);
  const double j0 = b.jac[p0], j1 = b.jac[p1];
  const T nx = (T)(0.5 * (b.met[(d * 3 + 0) * P + p0] * j0 + b.met[(d * 3 + 0) * P + p1] * j1));
  const T ny = (T)(0.5 * (b.met[(d * 3 + 1) * P + p0] * j0 + b.met[(d * 3 + 1) * P + p1] * j1));
  const T nz = (T)(0.5 * (b.met[(d * 3 + 2) * P + p0] * j0 + b.met[(d * 3 + 2) * P + p1] * j1));
  fv[0] = 0;
  fv[1] = nx * txx + ny * txy + nz * txz;
  fv[2] = nx * txy + ny * tyy + nz * tyz;
  fv[3] = nx * txz + ny * tyz + nz * tzz;
  const T um = (T)(0.5 * (s.bv[P + p0] + s.bv[P + p1]));
  const T vm = (T)(0.5 * (s.bv[2 * P + p0] + s.bv[2 * P + p1]));
  const T wm = (T)(0.5 * (s.bv[3 * P + p0] + s.bv[3 * P + p1]));
  const T cond = (T)(0.5 * (s.cond[p0] + s.cond[p1]));
  fv[4] = um * fv[1] + vm * fv[2] + wm * fv[3] + cond * (nx * gt[0] + ny * gt[1] + nz * gt[2]);
  const int ns = OSTC_NS;
  T dif[Spec<NS>::A], yk[Spec<NS>::A], ddf[Spec<NS>::A];
  T sgw = 0, srdy = 0, corr = 0, mwt = 0;
  for (int l = 0; l < ns; ++l) {
    const double *Y = s.sv + (long long)l * P;
    yk[l] = (T)(0.5 * (Y[p0] + Y[p1]));
    dif[l] = (T)(0.5 * (s.rhod[l * P + p0] + s.rhod[l * P + p1]));
    T gy[3];
    grad(Y, gy);
    const T gdy = nx * gy[0] + ny * gy[1] + nz * gy[2];
    ddf[l] = gdy;
    corr += dif[l] * gdy;
    sgw += gdy / (T)c_mix.mw[l];
    mwt += yk[l] / (T)c_mix.mw[l];
    srdy += dif[l] * yk[l];
  }
  mwt = T(1) / mwt;
  corr -= mwt * srdy * sgw;
  T h[Spec<NS>::A];
  mix_h_cp<NS, T>((T)(0.5 * (s.bv[5 * P + p0] + s.bv[5 * P + p1])), h, nullptr);
  for (int l = 0; l < ns; ++l) {
    const T flux = dif[l] * (ddf[l] - mwt * yk[l] * sgw) - yk[l] * corr;
    fv[5 + l] = flux;
    fv[4] += h[l] * flux;
  }
}

// viscous_flux_fv/gv/hv (SchemeSelector.cuh:69-154) for mixtures: one thread per face of the tile,
// then dq += fv(i+1/2) - fv(i-1/2) through shared memory; tiles as the flux-split sweeps.
template <int DIR, bool DIM3, int NS, typename T>
__global__ void __launch_bounds__(FvsTile<DIR>::TD * FvsTile<DIR>::TXL, sizeof(T) == 8 ? 4 : 5) k_mix_visc(DevBlock b, DevState s,
                                                                                    double *__restrict__ dq, int nv) {
  if (NS > 0) nv = 5 + NS;
  constexpr int TXL = FvsTile<DIR>::TXL, TD = FvsTile<DIR>::TD;
  extern __shared__ __align__(16) unsigned char mix_smem[];
  T *fsm = reinterpret_cast<T *>(mix_smem);
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
  const bool face_ok = i0 < b.mx && n < nd;
  T fv[Spec<NS>::A + 5];
  for (int l = 0; l < kMV; ++l) fv[l] = T(0);
  if (face_ok) {
    const long long p0 = DIR == 0 ? b.id(n, j0, k0) : DIR == 1 ? b.id(i0, n, k0) : b.id(i0, j0, n);
    mix_visc_face<DIM3, NS, T>(b, s, p0, DIR, nv, fv);
  }
  for (int l = 0; l < nv; ++l) fsm[((long long)t * TXL + lane) * nv + l] = fv[l];
  __syncthreads();
  if (face_ok && t >= 1) {
    const long long q = DIR == 0 ? b.iq(n, j0, k0) : DIR == 1 ? b.iq(i0, n, k0) : b.iq(i0, j0, n);
    for (int l = 0; l < nv; ++l)
      dq[l * b.n + q] += (double)(fv[l] - fsm[((long long)(t - 1) * TXL + lane) * nv + l]);
  }
}

// update_cv_and_bv_rk<mixture> (RK.cuh:230-284) with compute_temperature_and_pressure
// (FieldOperation.cu:3-40): the Newton iteration starts from the stage-input temperature.  With dtl
// (per-node local time steps, interior-indexed) the step of each node is dtl[n] instead of *dtp: the
// steady driver's update_cv_and_bv (FieldOperation.cuh:189-232) with ca = 0, cb = cc = 1 and the state
// updated in place (in = qn = out).
template <int NS>
__global__ void __launch_bounds__(128, 4) k_mix_update(DevBlock b, DevState in, DevState qn, DevState out,
                                                     const double *__restrict__ dq, const double *dtp, double ca,
                                                     double cb, double cc, int nv, unsigned *flags,
                                                     const double *__restrict__ dtl = nullptr) {
  if (NS > 0) nv = 5 + NS;
  const long long P = b.plane;
  const int ns = OSTC_NS;
  const double dt = dtl ? 0.0 : *dtp;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < b.n; n += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(n % b.mx);
    const long long r = n / b.mx;
    const int j = (int)(r % b.my), k = (int)(r / b.my);
    const long long p = b.id(i, j, k);
    const double dtj = (dtl ? dtl[n] : dt) / b.jac[p];
    double c[Spec<NS>::A + 5];
    for (int l = 0; l < nv; ++l) {
      c[l] = ca * qn.cv[l * P + p] + cb * in.cv[l * P + p] + cc * dtj * dq[l * b.n + n];
    }
    if (b.mz == 1) c[3] = 0;
    for (int l = 0; l < nv; ++l) out.cv[l * P + p] = c[l];
    const double rho = c[0];
    const double di = 1.0 / rho;
    const double u = c[1] * di, v = c[2] * di, w = c[3] * di;
    out.bv[p] = rho;
    out.bv[P + p] = u;
    out.bv[2 * P + p] = v;
    out.bv[3 * P + p] = w;
    double y[Spec<NS>::A];
    for (int l = 0; l < ns; ++l) {
      y[l] = c[5 + l] * di;
      out.sv[l * P + p] = y[l];
    }
    const double e = c[4] / rho - 0.5 * (u * u + v * v + w * w);
    double pr;
    const double t = mix_temperature<NS>(rho, e, in.bv[5 * P + p], y, pr);
    out.bv[4 * P + p] = pr;
    out.bv[5 * P + p] = t;
    if (!(rho > 0) || !(pr > 0) || !(t > 0)) atomicOr(flags, (rho != rho || pr != pr || t != t) ? 2u : 1u);
  }
}

}  // namespace ostc
