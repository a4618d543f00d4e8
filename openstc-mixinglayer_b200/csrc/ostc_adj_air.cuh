// ostc_adj_air.cuh -- vector-Jacobian product of the calorically-perfect-air right-hand side
// (ostc_rhs_vjp on the AWENO path): cv_bar = (d dq / d cv)^T dq_bar at the current state.  The
// reference has no adjoint.  Every term of the forward sweep is a function of a few stencil nodes'
// cv, so its transposed Jacobian is assembled from local derivatives:
//   1. face fluxes (AWENO_interpolation + Riemann solver, AWENO.cu:15-154, RiemannSolver.cuh:9-230):
//      the face's adjoint (dq_bar of its two nodes) times d F_face / d cv of each of the 2 NG stencil
//      nodes, by forward-mode Dual evaluations of the same templated face code (aweno_face_flux), one
//      seeded conservative variable per evaluation;
//   2. the central correction (CDSPart1D, AWENO.cu:307-350): per node, the adjoint of its physical
//      flux collected from the nodes whose correction reads it, times d f_node / d cv (Dual);
//   3. viscous faces (viscous_flux_fv/gv/hv, ViscousScheme.cuh:24-911): d F_v / d cv of the up to ten
//      nodes the face's gradients read, through u, v, w, T (equation of state) and the Sutherland
//      viscosity of each node (analytic node derivatives, Dual face evaluations);
//   4. ghost fills in reverse face order (apply_outflow / apply_periodic): a ghost's cv adjoint moves
//      to the node it was copied from (a ghost's cv is its source's cv).
// Evaluations are FP64 (the plain path's adjoint).  Accumulation into the node planes uses atomicAdd
// where several threads reach one node, so results are reproducible to rounding, not bitwise.
#pragma once

#include "dual.cuh"

namespace ostc {

template <> __device__ __forceinline__ Dual trsqrt<Dual>(Dual x) { return 1.0 / ad::sqrt(x); }
template <> __device__ __forceinline__ Dual tabs<Dual>(Dual x) { return ad::fabs(x); }
template <> __device__ __forceinline__ Dual tmin<Dual>(Dual a, Dual b) { return b < a ? b : a; }
template <> __device__ __forceinline__ Dual tmax<Dual>(Dual a, Dual b) { return b > a ? b : a; }

// The FP64 weight combination (same products of the D_k) on dual numbers.
template <> struct WenoComb<Dual> {
  static __device__ __forceinline__ void c3(Dual d0, Dual d1, Dual d2, Dual D0, Dual D1, Dual D2, Dual tau, Dual v0,
                                            Dual v1, Dual v2, Dual &num, Dual &den) {
    const Dual w0 = d0 * (D0 + tau) * (D1 * D2), w1 = d1 * (D1 + tau) * (D0 * D2), w2 = d2 * (D2 + tau) * (D0 * D1);
    num = w0 * v0 + w1 * v1 + w2 * v2;
    den = w0 + w1 + w2;
  }
  static __device__ __forceinline__ void c4(Dual d0, Dual d1, Dual d2, Dual d3, Dual D0, Dual D1, Dual D2, Dual D3,
                                            Dual tau, Dual v0, Dual v1, Dual v2, Dual v3, Dual &num, Dual &den) {
    const Dual a = D0 * D1, b = D2 * D3;
    const Dual w0 = d0 * (D0 + tau) * (D1 * b), w1 = d1 * (D1 + tau) * (D0 * b);
    const Dual w2 = d2 * (D2 + tau) * (a * D3), w3 = d3 * (D3 + tau) * (a * D2);
    num = w0 * v0 + w1 * v1 + w2 * v2 + w3 * v3;
    den = w0 + w1 + w2 + w3;
  }
  static __device__ __forceinline__ void finish(Dual nm, Dual dm, Dual np, Dual dp, Dual &vm, Dual &vp) {
    vm = nm / dm;
    vp = np / dp;
  }
};

// d p / d cv of one node (p = (gamma - 1)(rho E - |m|^2 / (2 rho))).
__device__ __forceinline__ void air_dp_dcv(const double *cv, double *dp) {
  const double ir = 1.0 / cv[0], u = cv[1] * ir, v = cv[2] * ir, w = cv[3] * ir;
  const double g1 = kGamma - 1;
  dp[0] = g1 * 0.5 * (u * u + v * v + w * w);
  dp[1] = -g1 * u;
  dp[2] = -g1 * v;
  dp[3] = -g1 * w;
  dp[4] = g1;
}

// Node index along a sweep: node c of direction DIR through the other two interior indices.
template <int DIR>
__device__ __forceinline__ long long sweep_id(const DevBlock &b, int c, int o1, int o2) {
  return DIR == 0 ? b.id(c, o1, o2) : DIR == 1 ? b.id(o1, c, o2) : b.id(o1, o2, c);
}
template <int DIR>
__device__ __forceinline__ long long sweep_iq(const DevBlock &b, int c, int o1, int o2) {
  return DIR == 0 ? b.iq(c, o1, o2) : DIR == 1 ? b.iq(o1, c, o2) : b.iq(o1, o2, c);
}
// Thread t of a sweep over `span` sweep positions starting at c0 and all interior (o1, o2).
template <int DIR>
__device__ __forceinline__ void sweep_pos(const DevBlock &b, long long t, int span, int c0, int &c, int &o1, int &o2) {
  if (DIR == 0) {
    c = c0 + (int)(t % span);
    const long long r = t / span;
    o1 = (int)(r % b.my);
    o2 = (int)(r / b.my);
  } else {
    o1 = (int)(t % b.mx);
    const long long r = t / b.mx;
    c = c0 + (int)(r % span);
    o2 = (int)(r / span);
  }
}

// 1. Face fluxes of direction DIR (faces c + 1/2, c = -1 .. n - 1): every face thread turns its face
// adjoint into cv adjoints of its 2 NG stencil nodes.  The forward sweep subtracts F(c + 1/2) from
// dq of node c and adds it to node c + 1.
template <int DIR, int NG, int RS>
__global__ void __launch_bounds__(128) k_adj_air_face(DevBlock b, DevState s, const double *__restrict__ dqb,
                                                      double *__restrict__ acv) {
  const long long P = b.plane;
  const int nd = DIR == 0 ? b.mx : DIR == 1 ? b.my : b.mz;
  const long long other = DIR == 0 ? (long long)b.my * b.mz : DIR == 1 ? (long long)b.mx * b.mz : (long long)b.mx * b.my;
  const long long nf = (long long)(nd + 1) * other;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nf; t += (long long)gridDim.x * blockDim.x) {
    int c, o1, o2;
    sweep_pos<DIR>(b, t, nd + 1, -1, c, o1, o2);
    double fb[5];
    bool any = false;
#pragma unroll
    for (int l = 0; l < 5; ++l) {
      double a = 0.0;
      if (c >= 0) a -= dqb[l * b.n + sweep_iq<DIR>(b, c, o1, o2)];
      if (c + 1 < nd) a += dqb[l * b.n + sweep_iq<DIR>(b, c + 1, o1, o2)];
      fb[l] = a;
      any = any || a != 0.0;
    }
    if (!any) continue;
    double cv[2 * NG][5], pr[2 * NG];
    long long pid[2 * NG];
#pragma unroll
    for (int st = 0; st < 2 * NG; ++st) {
      pid[st] = sweep_id<DIR>(b, c - NG + 1 + st, o1, o2);
#pragma unroll
      for (int l = 0; l < 5; ++l) cv[st][l] = s.cv[l * P + pid[st]];
      pr[st] = s.bv[4 * P + pid[st]];
    }
    const long long pl = pid[NG - 1], prr = pid[NG];
    Dual mt0[3], mt1[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      mt0[q] = Dual(b.met[(DIR * 3 + q) * P + pl]);
      mt1[q] = Dual(b.met[(DIR * 3 + q) * P + prr]);
    }
    const Dual j0(b.jac[pl]), j1(b.jac[prr]);
#pragma unroll 1
    for (int st = 0; st < 2 * NG; ++st) {
      double dp[5];
      air_dp_dcv(cv[st], dp);
#pragma unroll 1
      for (int v = 0; v < 5; ++v) {
        auto q = [&](int sn, int vv) -> Dual {
          if (vv < 5) return Dual(cv[sn][vv], (sn == st && vv == v) ? 1.0 : 0.0);
          return Dual(pr[sn], sn == st ? dp[v] : 0.0);
        };
        Dual fc[5];
        aweno_face_flux<NG, RS, Dual>(q, mt0, mt1, j0, j1, fc);
        double g = 0.0;
#pragma unroll
        for (int l = 0; l < 5; ++l) g += fb[l] * fc[l].d;
        if (g != 0.0) atomicAdd(acv + v * P + pid[st], g);
      }
    }
  }
}

// 2. Central correction of direction DIR: node n (sweep positions -NG .. n + NG - 1) collects the
// adjoint of its physical flux from every node c = n -+ m whose correction reads it (c interior and
// c < n - 2 NG, as the forward sweep applies it), then maps it to its cv.  One thread per node.
template <int DIR, int NG>
__global__ void __launch_bounds__(128) k_adj_air_cds(DevBlock b, DevState s, const double *__restrict__ dqb,
                                                     double *__restrict__ acv) {
  const long long P = b.plane;
  const int nd = DIR == 0 ? b.mx : DIR == 1 ? b.my : b.mz;
  const long long other = DIR == 0 ? (long long)b.my * b.mz : DIR == 1 ? (long long)b.mx * b.mz : (long long)b.mx * b.my;
  const int span = nd + 2 * NG;
  const long long nn = (long long)span * other;
  // coefficients of f(c + m) - f(c - m), m = 1 .. NG (cds_correction)
  double cm[5];
  if (NG == 3) {
    cm[1] = -17.0 / 256; cm[2] = 13.0 / 320; cm[3] = -19.0 / 3840;
  } else {
    cm[1] = 421.0 / 5120; cm[2] = -289.0 / 5120; cm[3] = 1261.0 / 107520; cm[4] = -81.0 / 71680;
  }
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nn; t += (long long)gridDim.x * blockDim.x) {
    int n, o1, o2;
    sweep_pos<DIR>(b, t, span, -NG, n, o1, o2);
    double fb[5] = {0, 0, 0, 0, 0};
    bool any = false;
#pragma unroll
    for (int m = 1; m <= NG; ++m) {
      const int cu = n - m, cd = n + m;  // node n is f(cu + m) for cu, f(cd - m) for cd
      const bool use_u = cu >= 0 && cu < nd && cu < nd - 2 * NG;
      const bool use_d = cd >= 0 && cd < nd && cd < nd - 2 * NG;
#pragma unroll
      for (int l = 0; l < 5; ++l) {
        if (use_u) fb[l] += cm[m] * dqb[l * b.n + sweep_iq<DIR>(b, cu, o1, o2)];
        if (use_d) fb[l] -= cm[m] * dqb[l * b.n + sweep_iq<DIR>(b, cd, o1, o2)];
      }
      any = any || use_u || use_d;
    }
    if (!any) continue;
    const long long p = sweep_id<DIR>(b, n, o1, o2);
    double cv[5];
#pragma unroll
    for (int l = 0; l < 5; ++l) cv[l] = s.cv[l * P + p];
    double dp[5];
    air_dp_dcv(cv, dp);
    const double pn = s.bv[4 * P + p];
    const Dual k[3] = {Dual(b.met[(DIR * 3 + 0) * P + p]), Dual(b.met[(DIR * 3 + 1) * P + p]),
                       Dual(b.met[(DIR * 3 + 2) * P + p])};
    const Dual jac(b.jac[p]);
#pragma unroll 1
    for (int v = 0; v < 5; ++v) {
      Dual q[5];
#pragma unroll
      for (int l = 0; l < 5; ++l) q[l] = Dual(cv[l], l == v ? 1.0 : 0.0);
      const Dual ir = 1.0 / q[0];
      const Dual bb[5] = {q[0], q[1] * ir, q[2] * ir, q[3] * ir, Dual(pn, dp[v])};
      Dual f[5];
      node_flux<Dual>(bb, q[4], k, jac, f);
      double g = 0.0;
#pragma unroll
      for (int l = 0; l < 5; ++l) g += fb[l] * f[l].d;
      acv[v * P + p] += g;  // one thread per node in this launch
    }
  }
}

// 3. Viscous faces of direction DIR (faces c + 1/2, c = -1 .. n - 1; the forward adds F_v(c + 1/2) to
// dq of node c and subtracts it from node c + 1, components 1..4).  The face reads u, v, w, T, mu of
// the nodes {0, e_d} x {0, +-e_c} (c != d; c = 2 only in 3-D); each of them is seeded per conserved
// variable with the analytic node derivatives of u, v, w, T = p W / (rho R_u) and Sutherland's mu.
template <int DIR, bool DIM3>
__global__ void __launch_bounds__(128) k_adj_air_visc(DevBlock b, DevState s, const double *__restrict__ dqb,
                                                      double prandtl, double *__restrict__ acv) {
  const long long P = b.plane;
  const int nd = DIR == 0 ? b.mx : DIR == 1 ? b.my : b.mz;
  const long long other = DIR == 0 ? (long long)b.my * b.mz : DIR == 1 ? (long long)b.mx * b.mz : (long long)b.mx * b.my;
  const long long nf = (long long)(nd + 1) * other;
  const long long st3[3] = {1, b.pitch, (long long)b.pitch * b.sy};
  constexpr int NN = DIM3 ? 10 : 6;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nf; t += (long long)gridDim.x * blockDim.x) {
    int c, o1, o2;
    sweep_pos<DIR>(b, t, nd + 1, -1, c, o1, o2);
    double fb[4];
    bool any = false;
#pragma unroll
    for (int l = 0; l < 4; ++l) {
      double a = 0.0;
      if (c >= 0) a += dqb[(l + 1) * b.n + sweep_iq<DIR>(b, c, o1, o2)];
      if (c + 1 < nd) a -= dqb[(l + 1) * b.n + sweep_iq<DIR>(b, c + 1, o1, o2)];
      fb[l] = a;
      any = any || a != 0.0;
    }
    if (!any) continue;
    const long long p0 = sweep_id<DIR>(b, c, o1, o2);
    // the stencil nodes (padded offsets from p0)
    long long off[NN];
    {
      int n = 0;
      off[n++] = 0;
      off[n++] = st3[DIR];
#pragma unroll
      for (int cc = 0; cc < 3; ++cc) {
        if (cc == DIR || (cc == 2 && !DIM3)) continue;
        off[n++] = st3[cc];
        off[n++] = -st3[cc];
        off[n++] = st3[DIR] + st3[cc];
        off[n++] = st3[DIR] - st3[cc];
      }
    }
    const Dual ipr(1.0 / prandtl);
    const Dual vref[3] = {Dual(0.0), Dual(0.0), Dual(0.0)};
    auto Mt = [&](int r, int sd) -> Dual {
      const long long p = p0 + (sd ? st3[DIR] : 0);
      return Dual(r == 9 ? b.jac[p] : b.met[r * P + p]);
    };
#pragma unroll 1
    for (int sn = 0; sn < NN; ++sn) {
      const long long ps = b.chk(p0 + off[sn]);
      double cv[5];
#pragma unroll
      for (int l = 0; l < 5; ++l) cv[l] = s.cv[l * P + ps];
      const double ir = 1.0 / cv[0];
      const double u = cv[1] * ir, v = cv[2] * ir, w = cv[3] * ir;
      const double tt = s.bv[5 * P + ps], mu = s.mul[ps];
      const double rgas = kRuD / kMwD, pn = s.bv[4 * P + ps];
      double dp[5];
      air_dp_dcv(cv, dp);
      const double dmu_dt = mu * (1.5 / tt - 1.0 / (tt + 110.0));
#pragma unroll 1
      for (int vv = 0; vv < 5; ++vv) {
        // derivatives of (u, v, w, T, mu) of node sn along cv_vv
        double dq[5];
        dq[0] = vv == 0 ? -u * ir : vv == 1 ? ir : 0.0;
        dq[1] = vv == 0 ? -v * ir : vv == 2 ? ir : 0.0;
        dq[2] = vv == 0 ? -w * ir : vv == 3 ? ir : 0.0;
        dq[3] = (dp[vv] - (vv == 0 ? pn * ir : 0.0)) * ir / rgas;
        dq[4] = dmu_dt * dq[3];
        auto V = [&](int q, int di, int dj, int dk) -> Dual {
          const long long p = b.chk(p0 + di * st3[0] + dj * st3[1] + dk * st3[2]);
          const double val = q == 0 ? s.bv[P + p] : q == 1 ? s.bv[2 * P + p] : q == 2 ? s.bv[3 * P + p]
                           : q == 3 ? s.bv[5 * P + p] : s.mul[p];
          return Dual(val, p == ps ? dq[q] : 0.0);
        };
        Dual fv[4];
        viscous_face<Dual, DIM3>(DIR, V, Mt, ipr, vref, fv);
        double g = 0.0;
#pragma unroll
        for (int l = 0; l < 4; ++l) g += fb[l] * fv[l].d;
        if (g != 0.0) atomicAdd(acv + vv * P + ps, g);
      }
    }
  }
}

// 4. Ghost fills in reverse (apply_outflow / apply_periodic, BoundCond.cuh:205-233, 1443-1486) on the
// cv adjoint planes: each ghost's adjoint moves to the node it was copied from.
__global__ void __launch_bounds__(128) k_adj_air_bc_face(DevBlock b, double *acv, DevFace f) {
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
    long long po = pb;
    if (f.type == kPeriodic) {
      const int ext[3] = {b.mx, b.my, b.mz};
      int oth[3] = {idx[0], idx[1], idx[2]};
      oth[f.face] = f.direction < 0 ? ext[f.face] - 1 : 0;
      po = b.id(oth[0], oth[1], oth[2]);
    }
    for (int g = b.g; g >= 1; --g) {
      const long long pg = b.chk(pb + g * dstep);
      const long long ps = b.chk(f.type == kPeriodic ? po + g * dstep : pb);
#pragma unroll
      for (int l = 0; l < 5; ++l) {
        acv[l * P + ps] += acv[l * P + pg];
        acv[l * P + pg] = 0.0;
      }
    }
  }
}

}  // namespace ostc
