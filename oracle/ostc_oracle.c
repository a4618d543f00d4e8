/*
 * ostc_oracle.c -- serial FP64 CPU restatement of the OpenSTC RHS + SSP-RK3 hot path for
 * calorically perfect air.  TEST INFRASTRUCTURE: only tests/, the smoke check and bench.py's CPU
 * baseline use it, and only as the checker / timed CPU baseline.
 *
 * Parity pin: the reference ships no tests or golden vectors for this path and runs only as CUDA, so
 * its own FP64 build (oracle/ref/build_ref.sh: the reference sources compiled for sm_100a with a
 * single-rank MPI subset, driven through its Driver and RK3 by oracle/ref/ref_harness.cu) produced
 * the fixtures in tests/golden/ (tests/golden/make_golden.py).  This restatement matches them to
 * ~1e-14 relative after 20-100 SSP-RK3 steps (tests/test_golden.py).
 *
 * Build (see oracle/Makefile): gcc -O2 -ffp-contract=off -fPIC -shared.  Contraction is disabled so
 * that every product/sum is rounded exactly as written, like the reference's source order.
 */
#include "ostc_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* Constants.h:18,26,31-35 */
#define GAMMA_AIR 1.4
#define R_U 8314.462618
#define MW_AIR 28.9647

typedef struct {
  int type, face, direction;
  int rs[3], re[3];
  double density, u, v, w, pressure, temperature, acoustic_speed, gamma, entropy, mw;
  int wall_adiabatic;
  double y[16];
  int inflow_type;
  double delta_omega, lower[6], y_lower[16];
} face_t;

struct orc_ctx {
  orc_case c;
  int mx, my, mz, g, dim;
  int sx, sy, sz;   /* padded extents of state arrays (ngg ghosts) */
  long P;
  int cx, cy, cz;   /* padded extents of coordinate arrays (ngg+1 ghosts, Mesh.cpp:229-231) */
  long PC;
  double *x, *y, *z;
  double *jac, *met; /* met: 9 SoA planes of P */
  double *cv, *bv, *mul, *qn, *dq, *dtl;
  /* mixtures: ns species, nv = 5 + ns conservative variables; per-node properties over the padded
   * block (update_physical_properties, FieldOperation.cuh:107-140) */
  int ns, nv;
  double *sv, *cond, *rhod, *cpm, *gam, *acs;
  double dt_cur; /* dt of the current step (point-implicit chemistry) */
  /* steady driver: inviscid spectral radii per interior node [N][3] (local_time_step), chemical
   * source Jacobian per node (chem_src_jac: [N][ns][ns] for EPI, [N][ns] for DA), DPLUR iterates */
  double *srad, *cj, *dq0, *dqk;
  /* dual time stepping: previous physical step's cv (qn1, padded), the BDF2 source q* (interior), the
   * inner iteration's stored (rho, |V|, p, T), the physical step count and the inner-iteration count */
  double *qn1, *qstar, *inlast;
  int dual_step, inner, dual_init;
  double res_scale_inner[4];
  face_t f[16];
  int nf;
  double t;
};

#define ID(o, i, j, k) ((((long)(k) + (o)->g) * (o)->sy + ((j) + (o)->g)) * (o)->sx + ((i) + (o)->g))
#define IC(o, i, j, k) ((((long)(k) + (o)->g + 1) * (o)->cy + ((j) + (o)->g + 1)) * (o)->cx + ((i) + (o)->g + 1))
#define IQ(o, i, j, k) ((((long)(k)) * (o)->my + (j)) * (o)->mx + (i))
#define M(o, r, c, p) ((o)->met[(long)((r) - 1) * 3 * (o)->P + (long)((c) - 1) * (o)->P + (p)])

static double sutherland(double t) { /* Transport.cu:6-9 */
  return 1.7894e-5 * pow(t / 288.16, 1.5) * (288.16 + 110) / (t + 110);
}

/* ---------------------------------------------------------------- geometry (host side) */

/* Mesh::init_ghost_grid for a single block without inner/parallel faces (Mesh.cpp:893-1043). */
static void ghost_grid(orc_ctx *o) {
  const int mx = o->mx, my = o->my, mz = o->mz, ngg = o->g;
  double *X = o->x, *Y = o->y, *Z = o->z;
#define XX(i, j, k) X[IC(o, i, j, k)]
#define YY(i, j, k) Y[IC(o, i, j, k)]
#define ZZ(i, j, k) Z[IC(o, i, j, k)]
  for (int k = 0; k < mz; ++k)
    for (int j = 0; j < my; ++j) {
      for (int i = -1; i >= -ngg - 1; --i) {
        XX(i, j, k) = 2 * XX(0, j, k) - XX(-i, j, k);
        YY(i, j, k) = 2 * YY(0, j, k) - YY(-i, j, k);
        ZZ(i, j, k) = 2 * ZZ(0, j, k) - ZZ(-i, j, k);
      }
      for (int i = mx; i < mx + ngg + 1; ++i) {
        XX(i, j, k) = 2 * XX(mx - 1, j, k) - XX(2 * (mx - 1) - i, j, k);
        YY(i, j, k) = 2 * YY(mx - 1, j, k) - YY(2 * (mx - 1) - i, j, k);
        ZZ(i, j, k) = 2 * ZZ(mx - 1, j, k) - ZZ(2 * (mx - 1) - i, j, k);
      }
    }
  for (int k = 0; k < mz; ++k)
    for (int i = 0; i < mx; ++i) {
      for (int j = -1; j >= -ngg - 1; --j) {
        XX(i, j, k) = 2 * XX(i, 0, k) - XX(i, -j, k);
        YY(i, j, k) = 2 * YY(i, 0, k) - YY(i, -j, k);
        ZZ(i, j, k) = 2 * ZZ(i, 0, k) - ZZ(i, -j, k);
      }
      for (int j = my; j < my + ngg + 1; ++j) {
        XX(i, j, k) = 2 * XX(i, my - 1, k) - XX(i, 2 * (my - 1) - j, k);
        YY(i, j, k) = 2 * YY(i, my - 1, k) - YY(i, 2 * (my - 1) - j, k);
        ZZ(i, j, k) = 2 * ZZ(i, my - 1, k) - ZZ(i, 2 * (my - 1) - j, k);
      }
    }
  if (o->dim == 3) {
    for (int j = 0; j < my; ++j)
      for (int i = 0; i < mx; ++i) {
        for (int k = -1; k >= -ngg - 1; --k) {
          XX(i, j, k) = 2 * XX(i, j, 0) - XX(i, j, -k);
          YY(i, j, k) = 2 * YY(i, j, 0) - YY(i, j, -k);
          ZZ(i, j, k) = 2 * ZZ(i, j, 0) - ZZ(i, j, -k);
        }
        for (int k = mz; k < mz + ngg + 1; ++k) {
          XX(i, j, k) = 2 * XX(i, j, mz - 1) - XX(i, j, 2 * (mz - 1) - k);
          YY(i, j, k) = 2 * YY(i, j, mz - 1) - YY(i, j, 2 * (mz - 1) - k);
          ZZ(i, j, k) = 2 * ZZ(i, j, mz - 1) - ZZ(i, j, 2 * (mz - 1) - k);
        }
      }
  } else {
    for (int j = 0; j < my; ++j)
      for (int i = 0; i < mx; ++i) {
        for (int k = -1; k >= -ngg - 1; --k) {
          XX(i, j, k) = XX(i, j, 0);
          YY(i, j, k) = YY(i, j, 0);
          ZZ(i, j, k) = ZZ(i, j, 0) + k;
        }
        for (int k = mz; k < mz + ngg + 1; ++k) {
          XX(i, j, k) = XX(i, j, mz - 1);
          YY(i, j, k) = YY(i, j, mz - 1);
          ZZ(i, j, k) = ZZ(i, j, mz - 1) + k - mz + 1;
        }
      }
  }
}

/* edges and corners by the parallelogram rule (Mesh.cpp:968-1036), after the face layers and the
 * interface layers (Mesh.cpp:962-967) */
static void ghost_grid_edges(orc_ctx *o) {
  const int mx = o->mx, my = o->my, mz = o->mz, ngg = o->g;
  double *X = o->x, *Y = o->y, *Z = o->z;
#define XX(i, j, k) X[IC(o, i, j, k)]
#define YY(i, j, k) Y[IC(o, i, j, k)]
#define ZZ(i, j, k) Z[IC(o, i, j, k)]
    for (int i = 1; i <= ngg + 1; ++i)
    for (int j = 1; j <= ngg + 1; ++j)
      for (int k = 0; k < mz; ++k) {
        const int i1 = -i, j1 = -j, i2 = mx - 1 + i, j2 = my - 1 + j;
        double *A[3] = {X, Y, Z};
        for (int q = 0; q < 3; ++q) {
          double *C = A[q];
          C[IC(o, i1, j1, k)] = C[IC(o, i1, 0, k)] + C[IC(o, 0, j1, k)] - C[IC(o, 0, 0, k)];
          C[IC(o, i2, j2, k)] = C[IC(o, i2, my - 1, k)] + C[IC(o, mx - 1, j2, k)] - C[IC(o, mx - 1, my - 1, k)];
          C[IC(o, i1, j2, k)] = C[IC(o, i1, my - 1, k)] + C[IC(o, 0, j2, k)] - C[IC(o, 0, my - 1, k)];
          C[IC(o, i2, j1, k)] = C[IC(o, i2, 0, k)] + C[IC(o, mx - 1, j1, k)] - C[IC(o, mx - 1, 0, k)];
        }
      }
  for (int i = 1; i <= ngg + 1; ++i)
    for (int j = 0; j < my; ++j)
      for (int k = 1; k <= ngg + 1; ++k) {
        const int i1 = -i, k1 = -k, i2 = mx - 1 + i, k2 = mz - 1 + k;
        double *A[3] = {X, Y, Z};
        for (int q = 0; q < 3; ++q) {
          double *C = A[q];
          C[IC(o, i1, j, k1)] = C[IC(o, i1, j, 0)] + C[IC(o, 0, j, k1)] - C[IC(o, 0, j, 0)];
          C[IC(o, i2, j, k2)] = C[IC(o, i2, j, mz - 1)] + C[IC(o, mx - 1, j, k2)] - C[IC(o, mx - 1, j, mz - 1)];
          C[IC(o, i1, j, k2)] = C[IC(o, i1, j, mz - 1)] + C[IC(o, 0, j, k2)] - C[IC(o, 0, j, mz - 1)];
          C[IC(o, i2, j, k1)] = C[IC(o, i2, j, 0)] + C[IC(o, mx - 1, j, k1)] - C[IC(o, mx - 1, j, 0)];
        }
      }
  for (int i = -ngg - 1; i <= mx + ngg; ++i)
    for (int j = 1; j <= ngg + 1; ++j)
      for (int k = 1; k <= ngg + 1; ++k) {
        const int j1 = -j, k1 = -k, j2 = my - 1 + j, k2 = mz - 1 + k;
        double *A[3] = {X, Y, Z};
        for (int q = 0; q < 3; ++q) {
          double *C = A[q];
          C[IC(o, i, j1, k1)] = C[IC(o, i, j1, 0)] + C[IC(o, i, 0, k1)] - C[IC(o, i, 0, 0)];
          C[IC(o, i, j2, k2)] = C[IC(o, i, j2, mz - 1)] + C[IC(o, i, my - 1, k2)] - C[IC(o, i, my - 1, mz - 1)];
          C[IC(o, i, j1, k2)] = C[IC(o, i, j1, mz - 1)] + C[IC(o, i, 0, k2)] - C[IC(o, i, 0, mz - 1)];
          C[IC(o, i, j2, k1)] = C[IC(o, i, j2, 0)] + C[IC(o, i, my - 1, k1)] - C[IC(o, i, my - 1, 0)];
        }
      }
#undef XX
#undef YY
#undef ZZ
}

/* One node of Block::compute_jac_metric (Mesh.cpp:241-503).  (fi,fj,fk) is the neighbour whose values
 * are copied when the Jacobian is not positive. */
static void metric_node(orc_ctx *o, int i, int j, int k, int fi, int fj, int fk) {
  const double *X = o->x, *Y = o->y, *Z = o->z;
  const double dxd1 = (X[IC(o, i + 1, j, k)] - X[IC(o, i - 1, j, k)]) * 0.5;
  const double dyd1 = (Y[IC(o, i + 1, j, k)] - Y[IC(o, i - 1, j, k)]) * 0.5;
  const double dzd1 = (Z[IC(o, i + 1, j, k)] - Z[IC(o, i - 1, j, k)]) * 0.5;
  const double dxd2 = (X[IC(o, i, j + 1, k)] - X[IC(o, i, j - 1, k)]) * 0.5;
  const double dyd2 = (Y[IC(o, i, j + 1, k)] - Y[IC(o, i, j - 1, k)]) * 0.5;
  const double dzd2 = (Z[IC(o, i, j + 1, k)] - Z[IC(o, i, j - 1, k)]) * 0.5;
  const double dxd3 = (X[IC(o, i, j, k + 1)] - X[IC(o, i, j, k - 1)]) * 0.5;
  const double dyd3 = (Y[IC(o, i, j, k + 1)] - Y[IC(o, i, j, k - 1)]) * 0.5;
  const double dzd3 = (Z[IC(o, i, j, k + 1)] - Z[IC(o, i, j, k - 1)]) * 0.5;
  const double jac = dxd1 * dyd2 * dzd3 + dxd2 * dyd3 * dzd1 + dxd3 * dyd1 * dzd2 - dxd1 * dyd3 * dzd2 -
                     dxd2 * dyd1 * dzd3 - dxd3 * dyd2 * dzd1;
  const long p = ID(o, i, j, k);
  if (jac <= 0) {
    const long q = ID(o, fi, fj, fk);
    o->jac[p] = o->jac[q];
    for (int r = 0; r < 9; ++r) o->met[r * o->P + p] = o->met[r * o->P + q];
    return;
  }
  o->jac[p] = jac;
  M(o, 1, 1, p) = (dyd2 * dzd3 - dyd3 * dzd2) / jac;
  M(o, 1, 2, p) = (dxd3 * dzd2 - dxd2 * dzd3) / jac;
  M(o, 1, 3, p) = (dxd2 * dyd3 - dxd3 * dyd2) / jac;
  M(o, 2, 1, p) = (dyd3 * dzd1 - dyd1 * dzd3) / jac;
  M(o, 2, 2, p) = (dxd1 * dzd3 - dxd3 * dzd1) / jac;
  M(o, 2, 3, p) = (dxd3 * dyd1 - dxd1 * dyd3) / jac;
  M(o, 3, 1, p) = (dyd1 * dzd2 - dyd2 * dzd1) / jac;
  M(o, 3, 2, p) = (dxd2 * dzd1 - dxd1 * dzd2) / jac;
  M(o, 3, 3, p) = (dxd1 * dyd2 - dxd2 * dyd1) / jac;
}

static void compute_metric(orc_ctx *o) {
  const int mx = o->mx, my = o->my, mz = o->mz, ngg = o->g;
  for (int i = 1; i < mx - 1; ++i)
    for (int j = 1; j < my - 1; ++j) {
      int k0 = 1, k1 = mz - 1;
      if (mz == 1) { k0 = 0; k1 = 1; }
      for (int k = k0; k < k1; ++k) metric_node(o, i, j, k, i, j, k);
    }
  for (int i = 1; i < mx - 1; ++i)
    for (int j = 1; j < my - 1; ++j)
      for (int k = 0; k >= -ngg; --k) metric_node(o, i, j, k, i, j, k + 1);
  for (int i = 1; i < mx - 1; ++i)
    for (int j = 1; j < my - 1; ++j)
      for (int k = mz - 1; k < mz + ngg; ++k) metric_node(o, i, j, k, i, j, k - 1);
  for (int i = 1; i < mx - 1; ++i)
    for (int j = 0; j >= -ngg; --j)
      for (int k = -ngg; k < mz + ngg; ++k) metric_node(o, i, j, k, i, j + 1, k);
  for (int i = 1; i < mx - 1; ++i)
    for (int j = my - 1; j < my + ngg; ++j)
      for (int k = -ngg; k < mz + ngg; ++k) metric_node(o, i, j, k, i, j - 1, k);
  for (int i = 0; i >= -ngg; --i)
    for (int j = -ngg; j < my + ngg; ++j)
      for (int k = -ngg; k < mz + ngg; ++k) metric_node(o, i, j, k, i + 1, j, k);
  for (int i = mx - 1; i < mx + ngg; ++i)
    for (int j = -ngg; j < my + ngg; ++j)
      for (int k = -ngg; k < mz + ngg; ++k) metric_node(o, i, j, k, i - 1, j, k);
}

/* Boundary::register_boundary (Mesh.cpp:14-32). */
static void register_face(orc_ctx *o, const orc_face_in *in, face_t *f) {
  const int ngg = o->g, dim = o->dim;
  f->rs[0] = in->raw[0]; f->re[0] = in->raw[1];
  f->rs[1] = in->raw[2]; f->re[1] = in->raw[3];
  f->rs[2] = in->raw[4]; f->re[2] = in->raw[5];
  f->face = 0;
  f->direction = 1;
  for (int i = 0; i < dim; ++i) {
    if (f->rs[i] == f->re[i]) {
      f->face = i;
      if (f->rs[i] == 0) f->direction = -1;
      break;
    }
  }
  for (int i = 0; i < dim; ++i) {
    if (i == f->face) continue;
    if (f->re[i] < f->rs[i]) { int t = f->re[i]; f->re[i] = f->rs[i]; f->rs[i] = t; }
    f->rs[i] -= ngg;
    f->re[i] += ngg;
  }
  if (dim == 2) { f->rs[2] = -ngg; f->re[2] = ngg; }
  f->type = in->type;
  f->density = in->density; f->u = in->u; f->v = in->v; f->w = in->w;
  f->pressure = in->pressure; f->temperature = in->temperature;
  f->acoustic_speed = in->acoustic_speed; f->gamma = in->gamma; f->entropy = in->entropy; f->mw = in->mw;
  f->wall_adiabatic = in->wall_adiabatic;
  memcpy(f->y, in->y, sizeof(f->y));
  f->inflow_type = in->inflow_type;
  f->delta_omega = in->delta_omega;
  memcpy(f->lower, in->lower, sizeof(f->lower));
  memcpy(f->y_lower, in->y_lower, sizeof(f->y_lower));
}

/* ---------------------------------------------------------------- pointwise helpers */

/* compute_cv_from_bv_1_point + compute_total_energy<Air> (FieldOperation.cuh:17-38,78-105). */
static void mix_h_cp(const orc_chem *ch, double t, double *h, double *cp);
#define FVS_MAXV (5 + ORC_MAX_SPEC)

static void cv_from_bv(orc_ctx *o, long p) {
  const long P = o->P;
  const double rho = o->bv[p];
  o->cv[p] = rho;
  o->cv[P + p] = rho * o->bv[P + p];
  o->cv[2 * P + p] = rho * o->bv[2 * P + p];
  o->cv[3 * P + p] = rho * o->bv[3 * P + p];
  const double u = o->bv[P + p], v = o->bv[2 * P + p], w = o->bv[3 * P + p];
  const double V2 = u * u + v * v + w * w;
  double te = 0.5 * V2;
  if (o->ns) {
    /* compute_total_energy<mixture> (FieldOperation.cuh:17-32): rho (sum h_k Y_k + V^2/2) - p */
    double h[ORC_MAX_SPEC];
    mix_h_cp(o->c.chem, o->bv[5 * P + p], h, NULL);
    for (int l = 0; l < o->ns; ++l) {
      o->cv[(5 + l) * P + p] = rho * o->sv[l * P + p];
      te += h[l] * o->sv[l * P + p];
    }
    te *= rho;
    te -= o->bv[4 * P + p];
  } else {
    te *= rho;
    te += o->bv[4 * P + p] / (GAMMA_AIR - 1);
  }
  o->cv[4 * P + p] = te;
}

/* ---------------------------------------------------------------- AWENO inviscid flux */

/* Characteristic WENO5-Z interpolation of one characteristic field (AWENO.cu:156-210).
 * st: 6 stencil points (i-2..i+3), 7 values each (5 cv, p, T). */
static void weno5_char(const double *L, const double st[][7], int l_row, double *vminus, double *vplus) {
  double v[6] = {0, 0, 0, 0, 0, 0};
  for (int s = 0; s < 6; ++s)
    for (int j = 0; j < 5; ++j) v[s] += L[l_row * 5 + j] * st[s][j];
  double v0 = 0.125 * (3 * v[0] - 10 * v[1] + 15 * v[2]);
  double v1 = 0.125 * (-v[1] + 6 * v[2] + 3 * v[3]);
  double v2 = 0.125 * (3 * v[2] + 6 * v[3] - v[4]);
  const double th = 13.0 / 12;
  double beta0 = th * (v[0] + v[2] - 2 * v[1]) * (v[0] + v[2] - 2 * v[1]) +
                 0.25 * (v[0] + 3 * v[2] - 4 * v[1]) * (v[0] + 3 * v[2] - 4 * v[1]);
  double beta1 = th * (v[1] + v[3] - 2 * v[2]) * (v[1] + v[3] - 2 * v[2]) + 0.25 * (v[3] - v[1]) * (v[3] - v[1]);
  double beta2 = th * (v[2] + v[4] - 2 * v[3]) * (v[2] + v[4] - 2 * v[3]) +
                 0.25 * (3 * v[2] + v[4] - 4 * v[3]) * (3 * v[2] + v[4] - 4 * v[3]);
  double tau = (beta0 - beta2) * (beta0 - beta2);
  const double eps = 1e-6, o16 = 1.0 / 16, f8 = 5.0 / 8, f16 = 5.0 / 16;
  double a0 = o16 + o16 * tau / ((eps + beta0) * (eps + beta0));
  double a1 = f8 + f8 * tau / ((eps + beta1) * (eps + beta1));
  double a2 = f16 + f16 * tau / ((eps + beta2) * (eps + beta2));
  *vminus = (a0 * v0 + a1 * v1 + a2 * v2) / (a0 + a1 + a2);
  v0 = v1;
  v1 = v2;
  v2 = 0.125 * (15 * v[3] - 10 * v[4] + 3 * v[5]);
  beta0 = th * (v[1] + v[3] - 2 * v[2]) * (v[1] + v[3] - 2 * v[2]) +
          0.25 * (v[1] + 3 * v[3] - 4 * v[2]) * (v[1] + 3 * v[3] - 4 * v[2]);
  beta1 = th * (v[2] + v[4] - 2 * v[3]) * (v[2] + v[4] - 2 * v[3]) + 0.25 * (v[4] - v[2]) * (v[4] - v[2]);
  beta2 = th * (v[3] + v[5] - 2 * v[4]) * (v[3] + v[5] - 2 * v[4]) +
          0.25 * (3 * v[3] + v[5] - 4 * v[4]) * (3 * v[3] + v[5] - 4 * v[4]);
  tau = (beta0 - beta2) * (beta0 - beta2);
  a0 = f16 + f16 * tau / ((eps + beta0) * (eps + beta0));
  a1 = f8 + f8 * tau / ((eps + beta1) * (eps + beta1));
  a2 = o16 + o16 * tau / ((eps + beta2) * (eps + beta2));
  *vplus = (a0 * v0 + a1 * v1 + a2 * v2) / (a0 + a1 + a2);
}

/* Characteristic WENO7-Z interpolation (AWENO.cu:212-280).  st: 8 points (i-3..i+4). */
static void weno7_char(const double *L, const double st[][7], int l_row, double *vminus, double *vplus) {
  double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int s = 0; s < 8; ++s)
    for (int j = 0; j < 5; ++j) v[s] += L[l_row * 5 + j] * st[s][j];
  double v0 = 0.0625 * (5 * v[3] + 15 * v[4] - 5 * v[5] + v[6]);
  double v1 = 0.0625 * (-v[2] + 9 * v[3] + 9 * v[4] - v[5]);
  double v2 = 0.0625 * (v[1] - 5 * v[2] + 15 * v[3] + 5 * v[4]);
  double v3 = 0.0625 * (-5 * v[0] + 21 * v[1] - 35 * v[2] + 35 * v[3]);
  const double c = 1.0 / 2880;
  double beta0 = c * (25729 * v[3] * v[3] + 134241 * v[4] * v[4] + 85641 * v[5] * v[5] -
                      6 * v[4] * (35047 * v[5] - 9449 * v[6]) - 47214 * v[5] * v[6] + 6649 * v[6] * v[6] -
                      2 * v[3] * (57447 * v[4] - 43107 * v[5] + 11389 * v[6]));
  double beta1 = c * (6649 * v[2] * v[2] + 41001 * v[3] * v[3] + 33441 * v[4] * v[4] +
                      v[2] * (-30414 * v[3] + 23094 * v[4] - 5978 * v[5]) - 19374 * v[4] * v[5] +
                      3169 * v[5] * v[5] + v[3] * (-70602 * v[4] + 19014 * v[5]));
  double beta2 = c * (3169 * v[1] * v[1] + 33441 * v[2] * v[2] + 41001 * v[3] * v[3] - 30414 * v[2] * v[3] +
                      6649 * v[3] * v[3] - 2 * v[1] * (9687 * v[2] - 9507 * v[3] + 2989 * v[4]) +
                      v[2] * (-70602 * v[3] + 23094 * v[4]));
  double beta3 = c * (6649 * v[0] * v[0] + 85641 * v[1] * v[1] + 134241 * v[2] * v[2] +
                      v[0] * (-47214 * v[1] + 56694 * v[2] - 22778 * v[3]) - 114894 * v[2] * v[3] +
                      25729 * v[3] * v[3] + v[1] * (-210282 * v[2] + 86214 * v[3]));
  double tau = (beta3 + 5 * beta2 - 5 * beta1 - beta0) * (beta3 + 5 * beta2 - 5 * beta1 - beta0);
  const double eps = 1e-6, s7 = 7.0 / 64, t5 = 35.0 / 64, t1 = 21.0 / 64, o1 = 1.0 / 64;
  double a0 = s7 + s7 * tau / ((eps + beta0) * (eps + beta0));
  double a1 = t5 + t5 * tau / ((eps + beta1) * (eps + beta1));
  double a2 = t1 + t1 * tau / ((eps + beta2) * (eps + beta2));
  double a3 = o1 + o1 * tau / ((eps + beta3) * (eps + beta3));
  *vminus = (a0 * v0 + a1 * v1 + a2 * v2 + a3 * v3) / (a0 + a1 + a2 + a3);
  v3 = v2;
  v2 = v1;
  v1 = v0;
  v0 = 0.0625 * (35 * v[4] - 35 * v[5] + 21 * v[6] - 5 * v[7]);
  beta0 = c * (25729 * v[4] * v[4] + 134241 * v[5] * v[5] + 85641 * v[6] * v[6] -
               6 * v[5] * (35047 * v[6] - 9449 * v[7]) - 47214 * v[6] * v[7] + 6649 * v[7] * v[7] -
               2 * v[4] * (57447 * v[5] - 43107 * v[6] + 11389 * v[7]));
  beta1 = c * (6649 * v[3] * v[3] + 41001 * v[4] * v[4] + 33441 * v[5] * v[5] +
               v[3] * (-30414 * v[4] + 23094 * v[5] - 5978 * v[6]) - 19374 * v[5] * v[6] +
               3169 * v[6] * v[6] + v[4] * (-70602 * v[5] + 19014 * v[6]));
  beta2 = c * (3169 * v[2] * v[2] + 33441 * v[3] * v[3] + 41001 * v[4] * v[4] - 30414 * v[3] * v[4] +
               6649 * v[4] * v[4] - 2 * v[2] * (9687 * v[3] - 9507 * v[4] + 2989 * v[5]) +
               v[3] * (-70602 * v[4] + 23094 * v[5]));
  beta3 = c * (6649 * v[1] * v[1] + 85641 * v[2] * v[2] + 134241 * v[3] * v[3] +
               v[1] * (-47214 * v[2] + 56694 * v[3] - 22778 * v[4]) - 114894 * v[3] * v[4] +
               25729 * v[4] * v[4] + v[2] * (-210282 * v[3] + 86214 * v[4]));
  tau = (beta3 + 5 * beta2 - 5 * beta1 - beta0) * (beta3 + 5 * beta2 - 5 * beta1 - beta0);
  a0 = o1 + o1 * tau / ((eps + beta0) * (eps + beta0));
  a1 = t1 + t1 * tau / ((eps + beta1) * (eps + beta1));
  a2 = t5 + t5 * tau / ((eps + beta2) * (eps + beta2));
  a3 = s7 + s7 * tau / ((eps + beta3) * (eps + beta3));
  *vplus = (a0 * v0 + a1 * v1 + a2 * v2 + a3 * v3) / (a0 + a1 + a2 + a3);
}

/* AWENO_interpolation<Air> (AWENO.cu:15-154): Roe average at i+1/2, characteristic WENO of cv,
 * back projection; returns the left/right primitive states (rho,u,v,w,p) and total energy.
 * st holds 2*ngg points centred so that st[ngg-1] is i and st[ngg] is i+1; mt: metric row of the
 * direction at i and i+1. */
static void aweno_interp(const double st[][7], int ngg, int recon, const double mt[2][3], double pl[6],
                         double pr[6]) {
  const double *cvl = st[ngg - 1], *cvr = st[ngg];
  const double rlc = sqrt(cvl[0]) / (sqrt(cvl[0]) + sqrt(cvr[0]));
  const double rrc = sqrt(cvr[0]) / (sqrt(cvl[0]) + sqrt(cvr[0]));
  const double um = rlc * cvl[1] / cvl[0] + rrc * cvr[1] / cvr[0];
  const double vm = rlc * cvl[2] / cvl[0] + rrc * cvr[2] / cvr[0];
  const double wm = rlc * cvl[3] / cvl[0] + rrc * cvr[3] / cvr[0];
  const double ekm = 0.5 * (um * um + vm * vm + wm * wm);
  const double gm1 = GAMMA_AIR - 1;
  const double hl = (cvl[4] + cvl[5]) / cvl[0];
  const double hr = (cvr[4] + cvr[5]) / cvr[0];
  const double hm = rlc * hl + rrc * hr;
  const double cm2 = gm1 * (hm - ekm);
  const double cm = sqrt(cm2);
  double kx = 0.5 * (mt[0][0] + mt[1][0]);
  double ky = 0.5 * (mt[0][1] + mt[1][1]);
  double kz = 0.5 * (mt[0][2] + mt[1][2]);
  const double gradK = sqrt(kx * kx + ky * ky + kz * kz);
  kx /= gradK;
  ky /= gradK;
  kz /= gradK;
  const double Uk = kx * um + ky * vm + kz * wm;
  const double alpha = gm1 * ekm;
  double L[25];
  L[0] = (alpha + Uk * cm) / cm2 * 0.5;
  L[1] = -(gm1 * um + kx * cm) / cm2 * 0.5;
  L[2] = -(gm1 * vm + ky * cm) / cm2 * 0.5;
  L[3] = -(gm1 * wm + kz * cm) / cm2 * 0.5;
  L[4] = gm1 / cm2 * 0.5;
  L[5] = kx * (1 - alpha / cm2) - (kz * vm - ky * wm) / cm;
  L[6] = kx * gm1 * um / cm2;
  L[7] = (kx * gm1 * vm + kz * cm) / cm2;
  L[8] = (kx * gm1 * wm - ky * cm) / cm2;
  L[9] = -kx * gm1 / cm2;
  L[10] = ky * (1 - alpha / cm2) - (kx * wm - kz * um) / cm;
  L[11] = (ky * gm1 * um - kz * cm) / cm2;
  L[12] = ky * gm1 * vm / cm2;
  L[13] = (ky * gm1 * wm + kx * cm) / cm2;
  L[14] = -ky * gm1 / cm2;
  L[15] = kz * (1 - alpha / cm2) - (ky * um - kx * vm) / cm;
  L[16] = (kz * gm1 * um + ky * cm) / cm2;
  L[17] = (kz * gm1 * vm - kx * cm) / cm2;
  L[18] = kz * gm1 * wm / cm2;
  L[19] = -kz * gm1 / cm2;
  L[20] = (alpha - Uk * cm) / cm2 * 0.5;
  L[21] = -(gm1 * um - kx * cm) / cm2 * 0.5;
  L[22] = -(gm1 * vm - ky * cm) / cm2 * 0.5;
  L[23] = -(gm1 * wm - kz * cm) / cm2 * 0.5;
  L[24] = gm1 / cm2 * 0.5;
  double vmi[5] = {0}, vpl[5] = {0};
  for (int l = 0; l < 5; ++l) {
    if (recon == 4) weno5_char(L, st + (ngg - 3), l, &vmi[l], &vpl[l]);
    else if (recon == 5) weno7_char(L, st + (ngg - 4), l, &vmi[l], &vpl[l]);
  }
  double R[25];
  R[0] = 1.0; R[1] = kx; R[2] = ky; R[3] = kz; R[4] = 1.0;
  R[5] = um - kx * cm; R[6] = kx * um; R[7] = ky * um - kz * cm; R[8] = kz * um + ky * cm; R[9] = um + kx * cm;
  R[10] = vm - ky * cm; R[11] = kx * vm + kz * cm; R[12] = ky * vm; R[13] = kz * vm - kx * cm; R[14] = vm + ky * cm;
  R[15] = wm - kz * cm; R[16] = kx * wm - ky * cm; R[17] = ky * wm + kx * cm; R[18] = kz * wm; R[19] = wm + kz * cm;
  R[20] = hm - Uk * cm;
  R[21] = kx * alpha / gm1 + (kz * vm - ky * wm) * cm;
  R[22] = ky * alpha / gm1 + (kx * wm - kz * um) * cm;
  R[23] = kz * alpha / gm1 + (ky * um - kx * vm) * cm;
  R[24] = hm + Uk * cm;
  double ql[5], qr[5];
  for (int m = 0; m < 5; ++m) {
    ql[m] = 0;
    qr[m] = 0;
    for (int n = 0; n < 5; ++n) {
      ql[m] += R[m * 5 + n] * vmi[n];
      qr[m] += R[m * 5 + n] * vpl[n];
    }
  }
  pl[0] = ql[0];
  pl[1] = ql[1] / ql[0];
  pl[2] = ql[2] / ql[0];
  pl[3] = ql[3] / ql[0];
  pl[4] = gm1 * (ql[4] - 0.5 * (pl[1] * pl[1] + pl[2] * pl[2] + pl[3] * pl[3]) * ql[0]);
  pl[5] = ql[4];
  pr[0] = qr[0];
  pr[1] = qr[1] / qr[0];
  pr[2] = qr[2] / qr[0];
  pr[3] = qr[3] / qr[0];
  pr[4] = gm1 * (qr[4] - 0.5 * (pr[1] * pr[1] + pr[2] * pr[2] + pr[3] * pr[3]) * qr[0]);
  pr[5] = qr[4];
}

/* riemannSolver_ausmPlus<Air> (RiemannSolver.cuh:9-96). pl/pr: rho,u,v,w,p,rhoE. */
static void ausm_plus(const double pl[6], const double pr[6], const double mt[2][3], const double jc[2],
                      double fc[5]) {
  const double k1 = 0.5 * (jc[0] * mt[0][0] + jc[1] * mt[1][0]);
  const double k2 = 0.5 * (jc[0] * mt[0][1] + jc[1] * mt[1][1]);
  const double k3 = 0.5 * (jc[0] * mt[0][2] + jc[1] * mt[1][2]);
  const double gkj = sqrt(k1 * k1 + k2 * k2 + k3 * k3);
  const double ul = (k1 * pl[1] + k2 * pl[2] + k3 * pl[3]) / gkj;
  const double ur = (k1 * pr[1] + k2 * pr[2] + k3 * pr[3]) / gkj;
  const double p_l = pl[4], p_r = pr[4], rho_l = pl[0], rho_r = pr[0];
  const double c = 0.5 * (sqrt(GAMMA_AIR * p_l / rho_l) + sqrt(GAMMA_AIR * p_r / rho_r));
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
  fc[4] = coeff * (q[5] + q[4]) / q[0];
}

/* riemannSolver_hllc<Air> (RiemannSolver.cuh:98-230). */
static void hllc(const double pl[6], const double pr[6], const double mt[2][3], const double jc[2], double fc[5]) {
  const double rl_c = sqrt(pl[0]) / (sqrt(pl[0]) + sqrt(pr[0]));
  const double rr_c = sqrt(pr[0]) / (sqrt(pl[0]) + sqrt(pr[0]));
  const double ut = pl[1] * rl_c + pr[1] * rr_c;
  const double vt = pl[2] * rl_c + pr[2] * rr_c;
  const double wt = pl[3] * rl_c + pr[3] * rr_c;
  const double hl = (pl[5] + pl[4]) / pl[0];
  const double hr = (pr[5] + pr[4]) / pr[0];
  const double ht = hl * rl_c + hr * rr_c;
  const double ekt = 0.5 * (ut * ut + vt * vt + wt * wt);
  const double ct = sqrt((GAMMA_AIR - 1) * (ht - ekt));
  const double kx = 0.5 * (mt[0][0] + mt[1][0]);
  const double ky = 0.5 * (mt[0][1] + mt[1][1]);
  const double kz = 0.5 * (mt[0][2] + mt[1][2]);
  const double gradK = sqrt(kx * kx + ky * ky + kz * kz);
  const double Ubar = (kx * ut + ky * vt + kz * wt) / gradK;
  const double jac = 0.5 * (jc[0] + jc[1]);
  const double Ul = kx * pl[1] + ky * pl[2] + kz * pl[3];
  const double cl = sqrt(GAMMA_AIR * pl[4] / pl[0]);
  const double sl = fmin(Ul / gradK - cl, Ubar - ct);
  if (sl >= 0) {
    const double rU = pl[0] * Ul;
    fc[0] = jac * rU;
    fc[1] = jac * (rU * pl[1] + pl[4] * kx);
    fc[2] = jac * (rU * pl[2] + pl[4] * ky);
    fc[3] = jac * (rU * pl[3] + pl[4] * kz);
    fc[4] = jac * ((pl[5] + pl[4]) * Ul);
    return;
  }
  const double Ur = kx * pr[1] + ky * pr[2] + kz * pr[3];
  const double cr = sqrt(GAMMA_AIR * pr[4] / pr[0]);
  const double sr = fmax(Ur / gradK + cr, Ubar + ct);
  if (sr < 0) {
    const double rU = pr[0] * Ur;
    fc[0] = jac * rU;
    fc[1] = jac * (rU * pr[1] + pr[4] * kx);
    fc[2] = jac * (rU * pr[2] + pr[4] * ky);
    fc[3] = jac * (rU * pr[3] + pr[4] * kz);
    fc[4] = jac * ((pr[5] + pr[4]) * Ur);
    return;
  }
  const double sm = ((pr[0] * Ur * (sr - Ur / gradK) - pl[0] * Ul * (sl - Ul / gradK)) / gradK + pl[4] - pr[4]) /
                    (pr[0] * (sr - Ur / gradK) - pl[0] * (sl - Ul / gradK));
  const double pm = pl[0] * (sl - Ul / gradK) * (sm - Ul / gradK) + pl[4];
  if (sm >= 0) {
    const double pc = 1.0 / (sl - sm);
    const double Q = jac * pc * sm * (sl * gradK - Ul) * pl[0];
    fc[0] = Q;
    const double dP = (sl * pm - sm * pl[4]) * pc * jac;
    fc[1] = Q * pl[1] + dP * kx;
    fc[2] = Q * pl[2] + dP * ky;
    fc[3] = Q * pl[3] + dP * kz;
    fc[4] = Q * pl[5] / pl[0] + pc * jac * (sl * pm * sm * gradK - sm * pl[4] * Ul);
  } else {
    const double pc = 1.0 / (sr - sm);
    const double Q = jac * pc * sm * (sr * gradK - Ur) * pr[0];
    fc[0] = Q;
    const double dP = (sr * pm - sm * pr[4]) * pc * jac;
    fc[1] = Q * pr[1] + dP * kx;
    fc[2] = Q * pr[2] + dP * ky;
    fc[3] = Q * pr[3] + dP * kz;
    fc[4] = Q * pr[5] / pr[0] + pc * jac * (sr * pm * sm * gradK - sm * pr[4] * Ur);
  }
}

/* riemannSolver_laxFriedrich<Air> (RiemannSolver.cuh:420-460). */
static void lax_friedrichs(const double pl[6], const double pr[6], const double mt[2][3], const double jc[2],
                           double fc[5]) {
  const double kx = 0.5 * (mt[0][0] + mt[1][0]);
  const double ky = 0.5 * (mt[0][1] + mt[1][1]);
  const double kz = 0.5 * (mt[0][2] + mt[1][2]);
  const double gradK = sqrt(kx * kx + ky * ky + kz * kz);
  const double Ukl = pl[1] * kx + pl[2] * ky + pl[3] * kz;
  const double Ukr = pr[1] * kx + pr[2] * ky + pr[3] * kz;
  const double cl = sqrt(GAMMA_AIR * pl[4] / pl[0]);
  const double cr = sqrt(GAMMA_AIR * pr[4] / pr[0]);
  const double sr = fmax(fabs(Ukl) + cl * gradK, fabs(Ukr) + cr * gradK);
  const double hj = 0.5 * 0.5 * (jc[0] + jc[1]);
  const double rUl = pl[0] * Ukl, rUr = pr[0] * Ukr;
  fc[0] = (rUl + rUr - sr * (pr[0] - pl[0])) * hj;
  fc[1] = (rUl * pl[1] + rUr * pr[1] + kx * (pl[4] + pr[4]) - sr * (pr[1] * pr[0] - pl[1] * pl[0])) * hj;
  fc[2] = (rUl * pl[2] + rUr * pr[2] + ky * (pl[4] + pr[4]) - sr * (pr[2] * pr[0] - pl[2] * pl[0])) * hj;
  fc[3] = (rUl * pl[3] + rUr * pr[3] + kz * (pl[4] + pr[4]) - sr * (pr[3] * pr[0] - pl[3] * pl[0])) * hj;
  fc[4] = ((pl[5] + pl[4]) * Ukl + (pr[5] + pr[4]) * Ukr - sr * (pr[5] - pl[5])) * hj;
}

/* compute_entropy_fix_delta<Air> (InviscidScheme.cu:417-456) at padded index p. */
static double entropy_fix_delta(const orc_ctx *o, long p) {
  const long P = o->P;
  const double u = o->bv[P + p], v = o->bv[2 * P + p], w = o->bv[3 * P + p];
  const double U = fabs(u * M(o, 1, 1, p) + v * M(o, 1, 2, p) + w * M(o, 1, 3, p));
  const double V = fabs(u * M(o, 2, 1, p) + v * M(o, 2, 2, p) + w * M(o, 2, 3, p));
  const double W = fabs(u * M(o, 3, 1, p) + v * M(o, 3, 2, p) + w * M(o, 3, 3, p));
  const double kx = sqrt(M(o, 1, 1, p) * M(o, 1, 1, p) + M(o, 1, 2, p) * M(o, 1, 2, p) + M(o, 1, 3, p) * M(o, 1, 3, p));
  const double ky = sqrt(M(o, 2, 1, p) * M(o, 2, 1, p) + M(o, 2, 2, p) * M(o, 2, 2, p) + M(o, 2, 3, p) * M(o, 2, 3, p));
  const double kz = sqrt(M(o, 3, 1, p) * M(o, 3, 1, p) + M(o, 3, 2, p) * M(o, 3, 2, p) + M(o, 3, 3, p) * M(o, 3, 3, p));
  const double c = o->ns ? o->acs[p] : sqrt(GAMMA_AIR * o->bv[4 * P + p] / o->bv[p]);
  if (o->dim == 2) return o->c.entropy_fix_factor * (U + V + c * 0.5 * (kx + ky));
  return o->c.entropy_fix_factor * (U + V + W + c * (kx + ky + kz) / 3.0);
}

/* riemannSolver_Roe<Air> (RiemannSolver.cuh:279-417) with compute_half_sum_left_right_flux
 * (:232-277): central part from each side's own metric and Jacobian, Roe dissipation with Harten's
 * entropy fix.  dl/dr: entropy-fix thresholds of the two face nodes. */
static void roe(const double pl[6], const double pr[6], const double mt[2][3], const double jc[2], double d0,
                double d1, double fc[5]) {
  double jx = jc[0] * mt[0][0], jy = jc[0] * mt[0][1], jz = jc[0] * mt[0][2];
  double Uk = pl[1] * jx + pl[2] * jy + pl[3] * jz;
  double co = Uk * pl[0];
  fc[0] = 0.5 * co;
  fc[1] = 0.5 * (co * pl[1] + pl[4] * jx);
  fc[2] = 0.5 * (co * pl[2] + pl[4] * jy);
  fc[3] = 0.5 * (co * pl[3] + pl[4] * jz);
  fc[4] = 0.5 * Uk * (pl[4] + pl[5]);
  jx = jc[1] * mt[1][0], jy = jc[1] * mt[1][1], jz = jc[1] * mt[1][2];
  Uk = pr[1] * jx + pr[2] * jy + pr[3] * jz;
  co = Uk * pr[0];
  fc[0] += 0.5 * co;
  fc[1] += 0.5 * (co * pr[1] + pr[4] * jx);
  fc[2] += 0.5 * (co * pr[2] + pr[4] * jy);
  fc[3] += 0.5 * (co * pr[3] + pr[4] * jz);
  fc[4] += 0.5 * Uk * (pr[4] + pr[5]);

  const double dl = sqrt(pl[0]), dr = sqrt(pr[0]);
  const double inv = 1.0 / (dl + dr);
  const double u = (dl * pl[1] + dr * pr[1]) * inv;
  const double v = (dl * pl[2] + dr * pr[2]) * inv;
  const double w = (dl * pl[3] + dr * pr[3]) * inv;
  const double ek = 0.5 * (u * u + v * v + w * w);
  const double hl = (pl[5] + pl[4]) / pl[0];
  const double hr = (pr[5] + pr[4]) / pr[0];
  const double h = (dl * hl + dr * hr) * inv;
  const double gamma = GAMMA_AIR;
  const double c = sqrt((gamma - 1) * (h - ek));
  double kx = 0.5 * (mt[0][0] + mt[1][0]);
  double ky = 0.5 * (mt[0][1] + mt[1][1]);
  double kz = 0.5 * (mt[0][2] + mt[1][2]);
  const double gradK = sqrt(kx * kx + ky * ky + kz * kz);
  Uk = kx * u + ky * v + kz * w;
  double ch[3] = {Uk - gradK * c, Uk, Uk + gradK * c};
  const double da = 0.5 * (d0 + d1);
  for (int n = 0; n < 3; ++n) {
    ch[n] = fabs(ch[n]);
    if (ch[n] < da) ch[n] = 0.5 * (ch[n] * ch[n] / da + da);
  }
  kx /= gradK;
  ky /= gradK;
  kz /= gradK;
  Uk /= gradK;
  const double ja = 0.5 * (jc[0] + jc[1]);
  double dq[5];
  dq[0] = ja * (pr[0] - pl[0]);
  for (int l = 1; l < 5; ++l) dq[l] = ja * (pr[0] * pr[l] - pl[0] * pl[l]);
  dq[4] = ja * (pr[5] - pl[5]);
  double c1 = (gamma - 1) * (ek * dq[0] - u * dq[1] - v * dq[2] - w * dq[3] + dq[4]) / (c * c);
  double c2 = (kx * dq[1] + ky * dq[2] + kz * dq[3] - Uk * dq[0]) / c;
  double c3 = dq[0] - c1;
  double L[5];
  L[0] = 0.5 * (c1 - c2);
  L[1] = kx * c3 - ((kz * v - ky * w) * dq[0] - kz * dq[2] + ky * dq[3]) / c;
  L[2] = ky * c3 - ((kx * w - kz * u) * dq[0] - kx * dq[3] + kz * dq[1]) / c;
  L[3] = kz * c3 - ((ky * u - kx * v) * dq[0] - ky * dq[1] + kx * dq[2]) / c;
  L[4] = 0.5 * (c1 + c2);
  double b[5];
  b[0] = -ch[0] * L[0];
  for (int l = 1; l < 5; ++l) b[l] = -ch[1] * L[l];
  b[4] = -ch[2] * L[4];
  const double c0 = kx * b[1] + ky * b[2] + kz * b[3];
  c1 = c0 + b[0] + b[4];
  c2 = c * (b[4] - b[0]);
  c3 = 0;
  fc[0] += 0.5 * c1;
  fc[1] += 0.5 * (u * c1 + kx * c2 - c * (kz * b[2] - ky * b[3]));
  fc[2] += 0.5 * (v * c1 + ky * c2 - c * (kx * b[3] - kz * b[1]));
  fc[3] += 0.5 * (w * c1 + kz * c2 - c * (ky * b[1] - kx * b[2]));
  fc[4] += 0.5 * (h * c1 + Uk * c2 - c * c * c0 / (gamma - 1) +
                  c * ((kz * v - ky * w) * b[1] + (kx * w - kz * u) * b[2] + (ky * u - kx * v) * b[3]) + c3);
}

/* minmod limiter, sgn(0) = +1 (Limiter.cuh:13-16, gxl_lib/Math.hpp:13-15). */
static double minmod(double a, double b) {
  const int sa = a < 0 ? -1 : 1, sb = b < 0 ? -1 : 1;
  return 0.5 * (sa + sb) * fmin(fabs(a), fabs(b));
}

/* reconstruction<Air> (InviscidScheme.cu:163-215) with first_order_reconstruct, MUSCL_reconstruct and
 * NND2_reconstruct (Reconstruction.cu:5-45).  st[m][l]: primitive l of nodes i-1, i, i+1, i+2. */
static void pv_reconstruct(const double st[4][5], int recon, double pl[6], double pr[6]) {
  const double kappa = 1.0 / 3.0;
  for (int l = 0; l < 5; ++l) {
    const double di = st[1][l] - st[0][l], di1 = st[2][l] - st[1][l], di2 = st[3][l] - st[2][l];
    if (recon == 2) {
      const double dnl = minmod(di, di1), dpl = minmod(di1, di);
      const double dnr = minmod(di1, di2), dpr = minmod(di2, di1);
      pl[l] = st[1][l] + 0.25 * ((1 - kappa) * dnl + (1 + kappa) * dpl);
      pr[l] = st[2][l] - 0.25 * ((1 - kappa) * dpr + (1 + kappa) * dnr);
    } else if (recon == 3) {
      pl[l] = st[1][l] + 0.5 * minmod(di, di1);
      pr[l] = st[2][l] - 0.5 * minmod(di1, di2);
    } else {
      pl[l] = st[1][l];
      pr[l] = st[2][l];
    }
  }
  const double el = 0.5 * (pl[1] * pl[1] + pl[2] * pl[2] + pl[3] * pl[3]);
  const double er = 0.5 * (pr[1] * pr[1] + pr[2] * pr[2] + pr[3] * pr[3]);
  pl[5] = el * pl[0] + pl[4] / (GAMMA_AIR - 1);
  pr[5] = er * pr[0] + pr[4] / (GAMMA_AIR - 1);
}

/* compute_convective_term_pv_1D (InviscidScheme.cu:52-161) and Roe_compute_inviscid_flux_1D
 * (:459-548) for one direction: faces at idx+1/2, idx = -1 .. n-1, then dq -= fc(i+1/2) - fc(i-1/2). */
/* ---- mixtures: the primitive-reconstruction path with the mixture branches of reconstruction()
 * (InviscidScheme.cu:163-215) and of the Riemann solvers (RiemannSolver.cuh:9-417).  A reconstructed
 * state holds rho, u, v, w, p, Y_1..Y_ns at [0, nv), then rho E at [nv] and gamma at [nv + 1]. */
#define PVM_MAX (FVS_MAXV + 2)

static void pv_reconstruct_mix(const orc_ctx *o, double st[4][FVS_MAXV], int recon, double *pl, double *pr) {
  const orc_chem *ch = o->c.chem;
  const int nv = o->nv, ns = o->ns;
  const double kappa = 1.0 / 3.0;
  for (int l = 0; l < nv; ++l) {
    const double di = st[1][l] - st[0][l], di1 = st[2][l] - st[1][l], di2 = st[3][l] - st[2][l];
    if (recon == 2) {
      const double dnl = minmod(di, di1), dpl = minmod(di1, di);
      const double dnr = minmod(di1, di2), dpr = minmod(di2, di1);
      pl[l] = st[1][l] + 0.25 * ((1 - kappa) * dnl + (1 + kappa) * dpl);
      pr[l] = st[2][l] - 0.25 * ((1 - kappa) * dpr + (1 + kappa) * dnr);
    } else if (recon == 3) {
      pl[l] = st[1][l] + 0.5 * minmod(di, di1);
      pr[l] = st[2][l] - 0.5 * minmod(di1, di2);
    } else {
      pl[l] = st[1][l];
      pr[l] = st[2][l];
    }
  }
  double el = 0.5 * (pl[1] * pl[1] + pl[2] * pl[2] + pl[3] * pl[3]);
  double er = 0.5 * (pr[1] * pr[1] + pr[2] * pr[2] + pr[3] * pr[3]);
  double mw_inv_l = 0, mw_inv_r = 0;
  for (int l = 0; l < ns; ++l) {
    mw_inv_l += pl[5 + l] / ch->mw[l];
    mw_inv_r += pr[5 + l] / ch->mw[l];
  }
  const double t_l = pl[4] / (pl[0] * R_U * mw_inv_l);
  const double t_r = pr[4] / (pr[0] * R_U * mw_inv_r);
  double hl[ORC_MAX_SPEC], hr[ORC_MAX_SPEC], cpl_i[ORC_MAX_SPEC], cpr_i[ORC_MAX_SPEC];
  mix_h_cp(ch, t_l, hl, cpl_i);
  mix_h_cp(ch, t_r, hr, cpr_i);
  double cpl = 0, cpr = 0, cvl = 0, cvr = 0;
  for (int l = 0; l < ns; ++l) {
    cpl += cpl_i[l] * pl[l + 5];
    cpr += cpr_i[l] * pr[l + 5];
    cvl += pl[l + 5] * (cpl_i[l] - R_U / ch->mw[l]);
    cvr += pr[l + 5] * (cpr_i[l] - R_U / ch->mw[l]);
    el += hl[l] * pl[l + 5];
    er += hr[l] * pr[l + 5];
  }
  pl[nv] = pl[0] * el - pl[4];
  pr[nv] = pr[0] * er - pr[4];
  pl[nv + 1] = cpl / cvl;
  pr[nv + 1] = cpr / cvr;
}

/* riemannSolver_ausmPlus<mixture> (RiemannSolver.cuh:9-96) */
static void ausm_mix(const orc_ctx *o, const double *pl, const double *pr, const double mt[2][3],
                     const double jc[2], double *fc) {
  const int nv = o->nv;
  const double k1 = 0.5 * (jc[0] * mt[0][0] + jc[1] * mt[1][0]);
  const double k2 = 0.5 * (jc[0] * mt[0][1] + jc[1] * mt[1][1]);
  const double k3 = 0.5 * (jc[0] * mt[0][2] + jc[1] * mt[1][2]);
  const double gkj = sqrt(k1 * k1 + k2 * k2 + k3 * k3);
  const double ul = (k1 * pl[1] + k2 * pl[2] + k3 * pl[3]) / gkj;
  const double ur = (k1 * pr[1] + k2 * pr[2] + k3 * pr[3]) / gkj;
  const double p_l = pl[4], p_r = pr[4], rho_l = pl[0], rho_r = pr[0];
  const double gam_l = pl[nv + 1], gam_r = pr[nv + 1];
  const double c = 0.5 * (sqrt(gam_l * p_l / rho_l) + sqrt(gam_r * p_r / rho_r));
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

/* gamma, speed of sound, mixture molecular weight and species enthalpies at the Roe-averaged state
 * (the mixture branches of riemannSolver_hllc / riemannSolver_Roe, RiemannSolver.cuh:118-137, 316-336) */
static void roe_mixture_sound(const orc_ctx *o, const double *svm, double tl, double tr, double wl, double wr,
                              double wsum_inv, int hllc_form, double *gamma, double *c, double *mw, double *h_i) {
  const orc_chem *ch = o->c.chem;
  double mw_inv = 0;
  for (int l = 0; l < o->ns; ++l) mw_inv += svm[l] / ch->mw[l];
  const double t = hllc_form ? (wl * tl + wr * tr) / (R_U * mw_inv) : (wl * tl + wr * tr) * wsum_inv / (R_U * mw_inv);
  double cp_i[ORC_MAX_SPEC];
  mix_h_cp(ch, t, h_i, cp_i);
  double cv = 0, cp = 0;
  for (int l = 0; l < o->ns; ++l) {
    cp += cp_i[l] * svm[l];
    cv += svm[l] * (cp_i[l] - R_U / ch->mw[l]);
  }
  *gamma = cp / cv;
  *c = sqrt(*gamma * R_U * mw_inv * t);
  *mw = 1.0 / mw_inv;
}

/* riemannSolver_hllc<mixture> (RiemannSolver.cuh:98-230) */
static void hllc_mix(const orc_ctx *o, const double *pl, const double *pr, const double mt[2][3], const double jc[2],
                     double *fc) {
  const int nv = o->nv;
  const double rl_c = sqrt(pl[0]) / (sqrt(pl[0]) + sqrt(pr[0])), rr_c = sqrt(pr[0]) / (sqrt(pl[0]) + sqrt(pr[0]));
  const double u_t = pl[1] * rl_c + pr[1] * rr_c, v_t = pl[2] * rl_c + pr[2] * rr_c, w_t = pl[3] * rl_c + pr[3] * rr_c;
  double svm[FVS_MAXV];
  for (int l = 0; l < nv - 5; ++l) svm[l] = rl_c * pl[l + 5] + rr_c * pr[l + 5];
  double gamma, c_t, mw, h_i[ORC_MAX_SPEC];
  roe_mixture_sound(o, svm, pl[4] / pl[0], pr[4] / pr[0], rl_c, rr_c, 0, 1, &gamma, &c_t, &mw, h_i);
  const double kx = 0.5 * (mt[0][0] + mt[1][0]), ky = 0.5 * (mt[0][1] + mt[1][1]), kz = 0.5 * (mt[0][2] + mt[1][2]);
  const double gradK = sqrt(kx * kx + ky * ky + kz * kz);
  const double U_t = (kx * u_t + ky * v_t + kz * w_t) / gradK;
  const double jac_ave = 0.5 * (jc[0] + jc[1]);
  const double gamma_l = pl[nv + 1], gamma_r = pr[nv + 1];
  const double Ul = kx * pl[1] + ky * pl[2] + kz * pl[3];
  const double cl = sqrt(gamma_l * pl[4] / pl[0]);
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
  const double cr = sqrt(gamma_r * pr[4] / pr[0]);
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

/* compute_half_sum_left_right_flux + riemannSolver_Roe<mixture> (RiemannSolver.cuh:232-417) */
static void roe_mix(const orc_ctx *o, const double *pl, const double *pr, const double mt[2][3], const double jc[2],
                    double d0, double d1, double *fc) {
  const orc_chem *ch = o->c.chem;
  const int nv = o->nv, ns = o->ns;
  double JacKx = jc[0] * mt[0][0], JacKy = jc[0] * mt[0][1], JacKz = jc[0] * mt[0][2];
  double Uk = pl[1] * JacKx + pl[2] * JacKy + pl[3] * JacKz;
  double coeff = Uk * pl[0];
  fc[0] = 0.5 * coeff;
  fc[1] = 0.5 * (coeff * pl[1] + pl[4] * JacKx);
  fc[2] = 0.5 * (coeff * pl[2] + pl[4] * JacKy);
  fc[3] = 0.5 * (coeff * pl[3] + pl[4] * JacKz);
  fc[4] = 0.5 * Uk * (pl[4] + pl[nv]);
  for (int l = 5; l < nv; ++l) fc[l] = 0.5 * coeff * pl[l];
  JacKx = jc[1] * mt[1][0];
  JacKy = jc[1] * mt[1][1];
  JacKz = jc[1] * mt[1][2];
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
  double svm[FVS_MAXV];
  for (int l = 0; l < nv - 5; ++l) svm[l] = (dl * pl[l + 5] + dr * pr[l + 5]) * inv_den;
  double gamma, c, mw, h_i[ORC_MAX_SPEC];
  roe_mixture_sound(o, svm, pl[4] / pl[0], pr[4] / pr[0], dl, dr, inv_den, 0, &gamma, &c, &mw, h_i);
  double kx = 0.5 * (mt[0][0] + mt[1][0]), ky = 0.5 * (mt[0][1] + mt[1][1]), kz = 0.5 * (mt[0][2] + mt[1][2]);
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
  const double jac_ave = 0.5 * (jc[0] + jc[1]);
  double dq[FVS_MAXV];
  dq[0] = jac_ave * (pr[0] - pl[0]);
  for (int l = 1; l < nv; ++l) dq[l] = jac_ave * (pr[0] * pr[l] - pl[0] * pl[l]);
  dq[4] = jac_ave * (pr[nv] - pl[nv]);
  double c1 = (gamma - 1) * (ek * dq[0] - u * dq[1] - v * dq[2] - w * dq[3] + dq[4]) / (c * c);
  double c2 = (kx * dq[1] + ky * dq[2] + kz * dq[3] - Ukk * dq[0]) / c;
  for (int l = 0; l < ns; ++l) c1 += (mw / ch->mw[l] - h_i[l] * (gamma - 1) / (c * c)) * dq[l + 5];
  double c3 = dq[0] - c1;
  double LDq[FVS_MAXV];
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
  for (int l = 0; l < ns; ++l) c3 += (h_i[l] - mw / ch->mw[l] * c * c / (gamma - 1)) * b[l + 5];
  fc[0] += 0.5 * c1;
  fc[1] += 0.5 * (u * c1 + kx * c2 - c * (kz * b[2] - ky * b[3]));
  fc[2] += 0.5 * (v * c1 + ky * c2 - c * (kx * b[3] - kz * b[1]));
  fc[3] += 0.5 * (w * c1 + kz * c2 - c * (ky * b[1] - kx * b[2]));
  fc[4] += 0.5 * (h * c1 + Ukk * c2 - c * c * c0 / (gamma - 1) +
                  c * ((kz * v - ky * w) * b[1] + (kx * w - kz * u) * b[2] + (ky * u - kx * v) * b[3]) + c3);
  for (int l = 0; l < nv - 5; ++l) fc[5 + l] += 0.5 * (b[l + 5] + svm[l] * c1);
}

static void pv_direction(orc_ctx *o, int dir) {
  const int ext[3] = {o->mx, o->my, o->mz};
  const long P = o->P, N = (long)o->mx * o->my * o->mz;
  int e[3] = {0, 0, 0};
  e[dir] = 1;
  const int n = ext[dir];
  int hi[3] = {o->mx, o->my, o->mz};
  hi[dir] = 1;
  const int nv = o->nv;
  double *fc = (double *)malloc(sizeof(double) * nv * (n + 1));
  for (int a = 0; a < hi[0]; ++a)
    for (int b = 0; b < hi[1]; ++b)
      for (int cc = 0; cc < hi[2]; ++cc) {
        for (int idx = -1; idx < n; ++idx) {
          double st[4][FVS_MAXV], mt[2][3], jc[2], ed[2] = {0, 0};
          for (int m = 0; m < 4; ++m) {
            const long p = ID(o, a + (idx - 1 + m) * e[0], b + (idx - 1 + m) * e[1], cc + (idx - 1 + m) * e[2]);
            for (int l = 0; l < 5; ++l) st[m][l] = o->bv[l * P + p];
            for (int l = 0; l < o->ns; ++l) st[m][5 + l] = o->sv[l * P + p];
          }
          for (int s = 0; s < 2; ++s) {
            const long p = ID(o, a + (idx + s) * e[0], b + (idx + s) * e[1], cc + (idx + s) * e[2]);
            for (int q = 0; q < 3; ++q) mt[s][q] = o->met[(long)(dir * 3 + q) * P + p];
            jc[s] = o->jac[p];
            if (o->c.riemann == 2) ed[s] = entropy_fix_delta(o, p);
          }
          double *f = &fc[nv * (idx + 1)];
          if (o->ns) {
            double pl[PVM_MAX], pr[PVM_MAX];
            pv_reconstruct_mix(o, st, o->c.reconstruction, pl, pr);
            switch (o->c.riemann) {
              case 2: roe_mix(o, pl, pr, mt, jc, ed[0], ed[1], f); break;
              case 4: hllc_mix(o, pl, pr, mt, jc, f); break;
              default: ausm_mix(o, pl, pr, mt, jc, f); break;
            }
            continue;
          }
          double st5[4][5];
          for (int m = 0; m < 4; ++m)
            for (int l = 0; l < 5; ++l) st5[m][l] = st[m][l];
          double pl[6], pr[6];
          pv_reconstruct(st5, o->c.reconstruction, pl, pr);
          switch (o->c.riemann) {
            case 1: lax_friedrichs(pl, pr, mt, jc, f); break;
            case 2: roe(pl, pr, mt, jc, ed[0], ed[1], f); break;
            case 4: hllc(pl, pr, mt, jc, f); break;
            default: ausm_plus(pl, pr, mt, jc, f); break;
          }
        }
        for (int idx = 0; idx < n; ++idx) {
          const long q = IQ(o, a + idx * e[0], b + idx * e[1], cc + idx * e[2]);
          for (int l = 0; l < nv; ++l) o->dq[l * N + q] -= fc[nv * (idx + 1) + l] - fc[nv * idx + l];
        }
      }
  free(fc);
}

/* Physical flux of one node for the central-difference correction (AWENO.cu:307-321). */
static void node_flux(const orc_ctx *o, long p, int dir, double f[5]) {
  const long P = o->P;
  const double kx = o->met[(long)(dir * 3 + 0) * P + p], ky = o->met[(long)(dir * 3 + 1) * P + p],
               kz = o->met[(long)(dir * 3 + 2) * P + p];
  const double u = o->bv[P + p], v = o->bv[2 * P + p], w = o->bv[3 * P + p];
  const double Uk = kx * u + ky * v + kz * w;
  const double rhoUk = o->bv[p] * Uk;
  const double pp = o->bv[4 * P + p], jac = o->jac[p];
  f[0] = rhoUk * jac;
  f[1] = jac * (rhoUk * u + kx * pp);
  f[2] = jac * (rhoUk * v + ky * pp);
  f[3] = jac * (rhoUk * w + kz * pp);
  f[4] = jac * Uk * (o->cv[4 * P + p] + pp);
}

/* compute_convective_term_aweno for one direction (InviscidScheme.cu:217-367) followed by
 * CDSPart1D<Air> (AWENO.cu:287-351).  The central correction is applied only on nodes
 * [0, extent - 2*ngg): CDSPart1D returns early for idx >= max_extent - ngg before building the flux
 * table (AWENO.cu:302) and skips idx >= max_extent - 2*ngg (AWENO.cu:325); that range is kept. */
static void aweno_direction(orc_ctx *o, int dir) {
  const int ngg = o->g, ext[3] = {o->mx, o->my, o->mz};
  const long P = o->P;
  int e[3] = {0, 0, 0};
  e[dir] = 1;
  const int n = ext[dir];
  int lo[3] = {0, 0, 0}, hi[3] = {o->mx, o->my, o->mz};
  hi[dir] = 1;
  double *fc = (double *)malloc(sizeof(double) * 5 * (n + 1));
  double *fp = (double *)malloc(sizeof(double) * 5 * (n + 2 * ngg));
  for (int a = lo[0]; a < hi[0]; ++a)
    for (int b = lo[1]; b < hi[1]; ++b)
      for (int cc = lo[2]; cc < hi[2]; ++cc) {
        /* face fluxes at idx+1/2, idx = -1 .. n-1 */
        for (int idx = -1; idx < n; ++idx) {
          double st[8][7], mt[2][3], jc[2];
          for (int s = -ngg + 1; s <= ngg; ++s) {
            const int ii = a + (idx + s) * e[0], jj = b + (idx + s) * e[1], kk = cc + (idx + s) * e[2];
            const long p = ID(o, ii, jj, kk);
            for (int l = 0; l < 5; ++l) st[s + ngg - 1][l] = o->cv[l * P + p];
            st[s + ngg - 1][5] = o->bv[4 * P + p];
            st[s + ngg - 1][6] = o->bv[5 * P + p];
          }
          for (int s = 0; s < 2; ++s) {
            const long p = ID(o, a + (idx + s) * e[0], b + (idx + s) * e[1], cc + (idx + s) * e[2]);
            for (int q = 0; q < 3; ++q) mt[s][q] = o->met[(long)(dir * 3 + q) * P + p];
            jc[s] = o->jac[p];
          }
          double pl[6], pr[6];
          aweno_interp(st, ngg, o->c.reconstruction, mt, pl, pr);
          double *f = &fc[5 * (idx + 1)];
          if (o->c.riemann == 4) hllc(pl, pr, mt, jc, f);
          else if (o->c.riemann == 1) lax_friedrichs(pl, pr, mt, jc, f);
          else ausm_plus(pl, pr, mt, jc, f);
        }
        for (int idx = 0; idx < n; ++idx) {
          const long q = IQ(o, a + idx * e[0], b + idx * e[1], cc + idx * e[2]);
          for (int l = 0; l < 5; ++l) o->dq[l * o->mx * (long)o->my * o->mz + q] -= fc[5 * (idx + 1) + l] - fc[5 * idx + l];
        }
        /* central correction */
        for (int idx = -ngg; idx < n - ngg; ++idx) {
          const long p = ID(o, a + idx * e[0], b + idx * e[1], cc + idx * e[2]);
          node_flux(o, p, dir, &fp[5 * (idx + ngg)]);
        }
        const long N = (long)o->mx * o->my * o->mz;
        for (int idx = 0; idx < n - 2 * ngg; ++idx) {
          const long q = IQ(o, a + idx * e[0], b + idx * e[1], cc + idx * e[2]);
#define F(m, l) fp[5 * (idx + (m) + ngg) + (l)]
          for (int l = 0; l < 5; ++l) {
            if (o->c.reconstruction == 4) {
              const double c1 = -19.0 / 3840, c2 = 13.0 / 320, c3 = -17.0 / 256;
              o->dq[l * N + q] += c1 * (F(3, l) - F(-3, l)) + c2 * (F(2, l) - F(-2, l)) + c3 * (F(1, l) - F(-1, l));
            } else {
              const double c4 = -81.0 / 71680, c3 = 1261.0 / 107520, c2 = -289.0 / 5120, c1 = 421.0 / 5120;
              o->dq[l * N + q] += c4 * (F(4, l) - F(-4, l)) + c3 * (F(3, l) - F(-3, l)) +
                                  c2 * (F(2, l) - F(-2, l)) + c1 * (F(1, l) - F(-1, l));
            }
          }
#undef F
        }
      }
  free(fc);
  free(fp);
}

/* ---------------------------------------------------------------- mixtures: thermodynamics */

/* compute_enthalpy_and_cp / compute_enthalpy / compute_cp (Thermo.cu:136-192, two-range NASA-7 with
 * linear extrapolation of h below t_low).  Either output may be NULL. */
static void mix_h_cp(const orc_chem *ch, double t, double *h, double *cp) {
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t, t5 = t4 * t;
  for (int i = 0; i < ch->n_spec; ++i) {
    double hh, cc;
    if (t < ch->t_low[i]) {
      const double tt = ch->t_low[i], tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt, tt5 = tt4 * tt;
      const double *a = &ch->low[i * 7];
      hh = a[0] * tt + 0.5 * a[1] * tt2 + a[2] * tt3 / 3 + 0.25 * a[3] * tt4 + 0.2 * a[4] * tt5 + a[5];
      cc = a[0] + a[1] * tt + a[2] * tt2 + a[3] * tt3 + a[4] * tt4;
      hh += cc * (t - tt);
    } else {
      const double *a = t < ch->t_mid[i] ? &ch->low[i * 7] : &ch->high[i * 7];
      hh = a[0] * t + 0.5 * a[1] * t2 + a[2] * t3 / 3 + 0.25 * a[3] * t4 + 0.2 * a[4] * t5 + a[5];
      cc = a[0] + a[1] * t + a[2] * t2 + a[3] * t3 + a[4] * t4;
    }
    if (h) h[i] = hh * (R_U / ch->mw[i]);
    if (cp) cp[i] = cc * (R_U / ch->mw[i]);
  }
}

/* compute_gibbs_div_rt (Thermo.cu:194-210): g_k / (R_u T) */
static void mix_gibbs_rt(const orc_chem *ch, double t, double *g) {
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t, ti = 1 / t, lt = log(t);
  for (int i = 0; i < ch->n_spec; ++i) {
    if (t < ch->t_low[i]) {
      const double tt = ch->t_low[i], tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt, tti = 1 / tt, ltt = log(tt);
      const double *a = &ch->low[i * 7];
      g[i] = a[0] * (1.0 - ltt) - 0.5 * a[1] * tt - a[2] * tt2 / 6.0 - a[3] * tt3 / 12.0 - a[4] * tt4 * 0.05 +
             a[5] * tti - a[6];
    } else {
      const double *a = t < ch->t_mid[i] ? &ch->low[i * 7] : &ch->high[i * 7];
      g[i] = a[0] * (1.0 - lt) - 0.5 * a[1] * t - a[2] * t2 / 6.0 - a[3] * t3 / 12.0 - a[4] * t4 * 0.05 + a[5] * ti -
             a[6];
    }
  }
}

/* compute_Omega_D (Transport.cu:168-170) */
static double omega_d(double tr) { return 1.0 / pow(tr, 0.145) + 1.0 / ((tr + 0.5) * (tr + 0.5)); }

/* update_physical_properties<mixture> (FieldOperation.cuh:116-134) with compute_transport_property
 * (Transport.cu:43-136): cp, gamma, c, Wilke viscosity, Eucken-type conductivity, mixture-averaged
 * rho*D_k. */
static void mix_properties_node(orc_ctx *o, long p) {
  const orc_chem *ch = o->c.chem;
  const int ns = o->ns;
  const long P = o->P;
  const double t = o->bv[5 * P + p];
  double cp[ORC_MAX_SPEC];
  mix_h_cp(ch, t, NULL, cp);
  double mw = 0, cpt = 0, cvt = 0;
  for (int l = 0; l < ns; ++l) {
    const double y = o->sv[l * P + p];
    mw += y / ch->mw[l];
    cpt += y * cp[l];
    cvt += y * (cp[l] - R_U / ch->mw[l]);
  }
  mw = 1 / mw;
  o->cpm[p] = cpt;
  o->gam[p] = cpt / cvt;
  o->acs[p] = sqrt(o->gam[p] * R_U * t / mw);
  double X[ORC_MAX_SPEC], vis[ORC_MAX_SPEC], dij[ORC_MAX_SPEC * ORC_MAX_SPEC];
  for (int l = 0; l < ns; ++l) {
    X[l] = o->sv[l * P + p] * mw / ch->mw[l];
    const double tdl = t * ch->lj_potent_inv[l];
    const double ci = 1.147 * pow(tdl, -0.145) + pow(tdl + 0.5, -2);
    vis[l] = ch->vis_coeff[l] * sqrt(t) / ci;
  }
  const double t32p = t * sqrt(t) / o->bv[4 * P + p];
  for (int m = 0; m < ns; ++m)
    for (int n = m; n < ns; ++n) {
      const double tr = t * ch->kb_over_eps_jk[m * ns + n];
      dij[m * ns + n] = ch->binary_diff[m * ns + n] * t32p / omega_d(tr);
      if (m != n) dij[n * ns + m] = dij[m * ns + n];
    }
  double visc = 0, cond = 0;
  for (int m = 0; m < ns; ++m) {
    double vt = 0;
    for (int n = 0; n < ns; ++n) {
      double pf = 1.0;
      if (m != n) {
        const double num = 1 + sqrt(vis[m] / vis[n]) * ch->wj_div_wi_1_4[m * ns + n];
        pf = num * num * ch->sqrt_wiwj_8[m * ns + n];
      }
      vt += pf * X[n];
    }
    const double ct = 1.065 * vt - 0.065 * X[m];
    visc += vis[m] * X[m] / vt;
    const double lam = vis[m] * (cp[m] + 1.25 * R_U / ch->mw[m]);
    cond += lam * X[m] / ct;
  }
  o->mul[p] = visc;
  o->cond[p] = cond;
  const double eps = 1e-12;
  for (int l = 0; l < ns; ++l) {
    double num = 0, den = 0;
    for (int n = 0; n < ns; ++n)
      if (l != n) {
        num += (X[n] + eps) * ch->mw[n];
        den += (X[n] + eps) / dij[l * ns + n];
      }
    o->rhod[l * P + p] = o->bv[p] * num / (den * mw);
  }
}

/* compute_temperature_and_pressure (FieldOperation.cu:3-40): Newton on e(T) from the current T,
 * relative tolerance 1e-3, at most 1000 iterations; p = rho R T. */
static void mix_t_and_p(orc_ctx *o, long p, double total_energy) {
  const orc_chem *ch = o->c.chem;
  const long P = o->P;
  double mw = 0;
  for (int l = 0; l < o->ns; ++l) mw += o->sv[l * P + p] / ch->mw[l];
  mw = 1 / mw;
  const double gc = R_U / mw;
  const double u = o->bv[P + p], v = o->bv[2 * P + p], w = o->bv[3 * P + p];
  const double e = total_energy / o->bv[p] - 0.5 * (u * u + v * v + w * w);
  double err = 1, t = o->bv[5 * P + p];
  int iter = 0;
  double h[ORC_MAX_SPEC], cp[ORC_MAX_SPEC];
  while (err > 1e-3 && iter++ < 1000) {
    mix_h_cp(ch, t, h, cp);
    double cpt = 0, hm = 0;
    for (int l = 0; l < o->ns; ++l) {
      cpt += cp[l] * o->sv[l * P + p];
      hm += h[l] * o->sv[l * P + p];
    }
    const double et = hm - gc * t;
    const double cv = cpt - gc;
    const double t1 = t - (et - e) / cv;
    err = fabs(1 - t1 / t);
    t = t1;
  }
  o->bv[5 * P + p] = t;
  o->bv[4 * P + p] = o->bv[p] * t * gc;
}

/* ---------------------------------------------------------------- mixtures: chemistry */

static double arrhenius(double t, double A, double b, double Ea) { return A * pow(t, b) * exp(-Ea / t); }

/* finite_rate_chemistry (FiniteRateChem.cu:7-58) with forward_reaction_rate (:60-102),
 * backward_reaction_rate (:108-150), rate_of_progress (:152-177), chemical_source (:179-195):
 * dq[5+l] += jac * omega_l at interior node (i,j,k). */
static void chemistry_node_jac(orc_ctx *o, int i, int j, int k, int implicit);
static void chemistry_node(orc_ctx *o, int i, int j, int k) { chemistry_node_jac(o, i, j, k, 0); }

/* solve_chem_system (FiniteRateChem.cu:302-357): column-pivoted LU in place, then substitution. */
static void lu_solve(double *lhs, double *b, int dim) {
  int ipiv[ORC_MAX_SPEC] = {0};
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

/* implicit = 1: also compute_chem_src_jacobian (FiniteRateChem.cu:197-217) and replace the species dq
 * by the EPI solution (FiniteRateChem.cu:233-254) with dt_cur.  implicit = 2: store that Jacobian in
 * o->cj (chemSrcMethod 1 of the steady driver); implicit = 3: store the diagonal approximation
 * -omega_d / (rho Y) (compute_chem_src_jacobian_diagonal, FiniteRateChem.cu:219-231; chemSrcMethod 2). */
static void chemistry_node_jac(orc_ctx *o, int i, int j, int k, int implicit) {
  const orc_chem *ch = o->c.chem;
  const int ns = ch->n_spec, nr = ch->n_reac;
  const long P = o->P, N = (long)o->mx * o->my * o->mz;
  const long p = ID(o, i, j, k), q = IQ(o, i, j, k);
  double c[ORC_MAX_SPEC];
  const double rho = o->bv[p];
  for (int l = 0; l < ns; ++l) c[l] = rho * o->sv[l * P + p] / ch->mw[l] * 1e-3;
  const double t = o->bv[5 * P + p];
  double kf[ORC_MAX_REAC], kb[ORC_MAX_REAC];
  for (int r = 0; r < nr; ++r) {
    kb[r] = 0;
    kf[r] = arrhenius(t, ch->A[r], ch->b[r], ch->Ea[r]);
    const int ty = ch->label[r];
    if (ty == 3) {
      kf[r] += arrhenius(t, ch->A2[r], ch->b2[r], ch->Ea2[r]);
    } else if (ty > 3) {
      double cc = 0;
      for (int l = 0; l < ns; ++l) cc += c[l] * ch->third_body[r * ns + l];
      if (ty == 4) {
        kf[r] *= cc;
      } else {
        const double klow = arrhenius(t, ch->A2[r], ch->b2[r], ch->Ea2[r]);
        const double khigh = kf[r];
        const double pr = klow * cc / khigh;
        double F = 1.0;
        if (ty > 5) {
          double fc = (1 - ch->troe_alpha[r]) * exp(-t / ch->troe_t3[r]) + ch->troe_alpha[r] * exp(-t / ch->troe_t1[r]);
          if (ty == 7) fc += exp(-ch->troe_t2[r] / t);
          const double lfc = log10(fc);
          const double cq = -0.4 - 0.67 * lfc;
          const double nq = 0.75 - 1.27 * lfc;
          const double lpr = log10(pr);
          const double tmp = (lpr + cq) / (nq - 0.14 * (lpr + cq));
          const double pw = lfc / (1.0 + tmp * tmp);
          F = pow(10, pw);
        }
        kf[r] = khigh * pr / (1.0 + pr) * F;
      }
    }
  }
  int n_gibbs = nr;
  for (int r = 0; r < nr; ++r) {
    if (ch->label[r] == 0) {
      kb[r] = 0;
      --n_gibbs;
    } else if (ch->rev_type[r] == 1) {
      kb[r] = arrhenius(t, ch->A2[r], ch->b2[r], ch->Ea2[r]);
      if (ch->label[r] == 4) {
        double cc = 0;
        for (int l = 0; l < ns; ++l) cc += c[l] * ch->third_body[r * ns + l];
        kb[r] *= cc;
      }
      --n_gibbs;
    }
  }
  if (n_gibbs >= 1) {
    double g[ORC_MAX_SPEC];
    mix_gibbs_rt(ch, t, g);
    const double temp_p = 101325.0 / R_U * 1e-3;
    const double temp_t = temp_p / t;
    for (int r = 0; r < nr; ++r) {
      if (ch->label[r] != 2 && ch->label[r] != 0) {
        double dg = 0;
        for (int l = 0; l < ns; ++l) dg += g[l] * (ch->stoi_b[r * ns + l] - ch->stoi_f[r * ns + l]);
        const double kc = pow(temp_t, ch->order[r]) * exp(-dg);
        kb[r] = kf[r] / kc;
      }
    }
  }
  double q1[ORC_MAX_REAC], q2[ORC_MAX_REAC];
  for (int r = 0; r < nr; ++r) {
    q1[r] = 1.0;
    q2[r] = ch->label[r] != 0 ? 1.0 : 0.0;
    for (int l = 0; l < ns; ++l) q1[r] *= pow(c[l], ch->stoi_f[r * ns + l]);
    if (ch->label[r] != 0)
      for (int l = 0; l < ns; ++l) q2[r] *= pow(c[l], ch->stoi_b[r * ns + l]);
    q1[r] *= kf[r];
    if (ch->label[r] != 0) q2[r] *= kb[r];
  }
  const double jac = o->jac[p];
  for (int l = 0; l < ns; ++l) {
    double cre = 0, des = 0;
    for (int r = 0; r < nr; ++r) {
      cre += q2[r] * ch->stoi_f[r * ns + l] + q1[r] * ch->stoi_b[r * ns + l];
      des += q1[r] * ch->stoi_f[r * ns + l] + q2[r] * ch->stoi_b[r * ns + l];
    }
    cre *= ch->mw[l] * 1e+3;
    des *= ch->mw[l] * 1e+3;
    o->dq[(5 + l) * N + q] += jac * (cre - des);
    if (implicit == 3) {
      const double yl = o->sv[l * P + p];
      o->cj[q * ns + l] = 0;
      if (yl > 1e-25) o->cj[q * ns + l] = -des / (yl * rho);
    }
  }
  if (!implicit || implicit == 3) return;
  if (implicit == 2) {
    for (int m = 0; m < ns; ++m)
      for (int n = 0; n < ns; ++n) {
        double zz = 0;
        const double yn = o->sv[n * P + p];
        if (yn > 1e-25) {
          for (int r = 0; r < nr; ++r)
            zz += (ch->stoi_b[r * ns + m] - ch->stoi_f[r * ns + m]) *
                  (ch->stoi_f[r * ns + n] * q1[r] - ch->stoi_b[r * ns + n] * q2[r]);
          zz /= rho * yn;
        }
        o->cj[(q * ns + m) * ns + n] = ch->mw[m] * zz * 1e+3;
      }
    return;
  }
  double lhs[ORC_MAX_SPEC * ORC_MAX_SPEC], b[ORC_MAX_SPEC];
  for (int m = 0; m < ns; ++m)
    for (int n = 0; n < ns; ++n) {
      double zz = 0;
      const double yn = o->sv[n * P + p];
      if (yn > 1e-25) {
        for (int r = 0; r < nr; ++r)
          zz += (ch->stoi_b[r * ns + m] - ch->stoi_f[r * ns + m]) *
                (ch->stoi_f[r * ns + n] * q1[r] - ch->stoi_b[r * ns + n] * q2[r]);
        zz /= rho * yn;
      }
      const double jm = ch->mw[m] * zz * 1e+3;
      lhs[m * ns + n] = (m == n ? 1.0 : 0.0) - o->dt_cur * jm;
    }
  for (int l = 0; l < ns; ++l) b[l] = o->dq[(5 + l) * N + q];
  lu_solve(lhs, b, ns);
  for (int l = 0; l < ns; ++l) o->dq[(5 + l) * N + q] = b[l];
}

/* ---------------------------------------------------------------- flux-split WENO (51/52/71/72) */

/* WENO7 of the flux-split path (WENO.cu:1619-1693): Z-type weights with tau = |b0 - b3|, linear
 * weights 1/35, 12/35, 18/35, 4/35; returns f+ + f-. */
static double fvs_beta7(double s1, double s2, double s3) {
  return s1 * s1 + 13.0 / 12.0 * s2 * s2 + 1043.0 / 960 * s3 * s3 + 1.0 / 12 * s1 * s3;
}

static double fvs_weno7(const double *vp, const double *vm, double eps) {
  const double one6th = 1.0 / 6, one12th = 1.0 / 12;
  const double c0 = 1.0 / 35, c1 = 12.0 / 35, c2 = 18.0 / 35, c3 = 4.0 / 35;
  double s1 = one6th * (-2 * vp[0] + 9 * vp[1] - 18 * vp[2] + 11 * vp[3]);
  double s2 = -vp[0] + 4 * vp[1] - 5 * vp[2] + 2 * vp[3];
  double s3 = -vp[0] + 3 * vp[1] - 3 * vp[2] + vp[3];
  double b0 = fvs_beta7(s1, s2, s3);
  s1 = one6th * (vp[1] - 6 * vp[2] + 3 * vp[3] + 2 * vp[4]);
  s2 = vp[2] - 2 * vp[3] + vp[4];
  s3 = -vp[1] + 3 * vp[2] - 3 * vp[3] + vp[4];
  double b1 = fvs_beta7(s1, s2, s3);
  s1 = one6th * (-2 * vp[2] - 3 * vp[3] + 6 * vp[4] - vp[5]);
  s3 = -vp[2] + 3 * vp[3] - 3 * vp[4] + vp[5];
  double b2 = fvs_beta7(s1, s2, s3);
  s1 = one6th * (-11 * vp[3] + 18 * vp[4] - 9 * vp[5] + 2 * vp[6]);
  s2 = 2 * vp[3] - 5 * vp[4] + 4 * vp[5] - vp[6];
  s3 = -vp[3] + 3 * vp[4] - 3 * vp[5] + vp[6];
  double b3 = fvs_beta7(s1, s2, s3);
  double tau = (b0 - b3) * (b0 - b3);
  double a0 = c0 + c0 * tau / ((eps + b0) * (eps + b0));
  double a1 = c1 + c1 * tau / ((eps + b1) * (eps + b1));
  double a2 = c2 + c2 * tau / ((eps + b2) * (eps + b2));
  double a3 = c3 + c3 * tau / ((eps + b3) * (eps + b3));
  double v0 = one12th * (-3 * vp[0] + 13 * vp[1] - 23 * vp[2] + 25 * vp[3]);
  double v1 = one12th * (vp[1] - 5 * vp[2] + 13 * vp[3] + 3 * vp[4]);
  double v2 = one12th * (-vp[2] + 7 * vp[3] + 7 * vp[4] - vp[5]);
  double v3 = one12th * (3 * vp[3] + 13 * vp[4] - 5 * vp[5] + vp[6]);
  const double fp = (a0 * v0 + a1 * v1 + a2 * v2 + a3 * v3) / (a0 + a1 + a2 + a3);
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
  a0 = c0 + c0 * tau / ((eps + b0) * (eps + b0));
  a1 = c1 + c1 * tau / ((eps + b1) * (eps + b1));
  a2 = c2 + c2 * tau / ((eps + b2) * (eps + b2));
  a3 = c3 + c3 * tau / ((eps + b3) * (eps + b3));
  v0 = one12th * (-3 * vm[6] + 13 * vm[5] - 23 * vm[4] + 25 * vm[3]);
  v1 = one12th * (vm[5] - 5 * vm[4] + 13 * vm[3] + 3 * vm[2]);
  v2 = one12th * (-vm[4] + 7 * vm[3] + 7 * vm[2] - vm[1]);
  v3 = one12th * (3 * vm[3] + 13 * vm[2] - 5 * vm[1] + vm[0]);
  const double fm = (a0 * v0 + a1 * v1 + a2 * v2 + a3 * v3) / (a0 + a1 + a2 + a3);
  return fp + fm;
}

/* compute_flux (WENO.cu:697-720): Lax-Friedrichs split F+- of one node with lambda0 = |U_k| + c|grad k|.
 * Q: cv[nv], then p, then c. */
static void fvs_node_flux(const double *Q, int nv, const double *k, double jac, double *Fp, double *Fm) {
  const double Uk = (Q[1] * k[0] + Q[2] * k[1] + Q[3] * k[2]) / Q[0];
  const double pk = Q[nv];
  const double cg = Q[nv + 1] * sqrt(k[0] * k[0] + k[1] * k[1] + k[2] * k[2]);
  const double l0 = fabs(Uk) + cg;
  Fp[0] = 0.5 * jac * (Uk * Q[0] + l0 * Q[0]);
  Fp[1] = 0.5 * jac * (Uk * Q[1] + pk * k[0] + l0 * Q[1]);
  Fp[2] = 0.5 * jac * (Uk * Q[2] + pk * k[1] + l0 * Q[2]);
  Fp[3] = 0.5 * jac * (Uk * Q[3] + pk * k[2] + l0 * Q[3]);
  Fp[4] = 0.5 * jac * (Uk * (Q[4] + pk) + l0 * Q[4]);
  Fm[0] = 0.5 * jac * (Uk * Q[0] - l0 * Q[0]);
  Fm[1] = 0.5 * jac * (Uk * Q[1] + pk * k[0] - l0 * Q[1]);
  Fm[2] = 0.5 * jac * (Uk * Q[2] + pk * k[1] - l0 * Q[2]);
  Fm[3] = 0.5 * jac * (Uk * Q[3] + pk * k[2] - l0 * Q[3]);
  Fm[4] = 0.5 * jac * (Uk * (Q[4] + pk) - l0 * Q[4]);
  for (int l = 5; l < nv; ++l) {
    Fp[l] = 0.5 * jac * (Uk * Q[l] + l0 * Q[l]);
    Fm[l] = 0.5 * jac * (Uk * Q[l] - l0 * Q[l]);
  }
}


/* compute_weno_flux_ch<mixture> for inviscid_scheme 72 (WENO.cu:722-758, 899-965, 1119-1142):
 * Roe-averaged mixture eigensystem at the face, characteristic projection of the split fluxes of
 * 7 nodes each side, WENO7-Z per field, back-projection.  Q[s]: node idx-3+s (s = 0..7), each
 * cv[nv], p, c; mt/jc: metric row and Jacobian of the same nodes. */
static void fvs_char_face(const orc_ctx *o, double Q[8][FVS_MAXV + 2], double mt[8][3], const double jc[8],
                          double *fc) {
  const orc_chem *ch = o->c.chem;
  const int nv = o->nv, ns = o->ns;
  double Fp[8][FVS_MAXV], Fm[8][FVS_MAXV];
  for (int s = 0; s < 8; ++s) fvs_node_flux(Q[s], nv, mt[s], jc[s], Fp[s], Fm[s]);
  const double *cvl = Q[3], *cvr = Q[4];
  const double *m_l = mt[3], *m_r = mt[4];
  const double rli = 1.0 / cvl[0], rri = 1.0 / cvr[0];
  const double rlc = sqrt(cvl[0]) / (sqrt(cvl[0]) + sqrt(cvr[0]));
  const double rrc = sqrt(cvr[0]) / (sqrt(cvl[0]) + sqrt(cvr[0]));
  const double um = rlc * cvl[1] * rli + rrc * cvr[1] * rri;
  const double vm = rlc * cvl[2] * rli + rrc * cvr[2] * rri;
  const double wm = rlc * cvl[3] * rli + rrc * cvr[3] * rri;
  const double ekm = 0.5 * (um * um + vm * vm + wm * wm);
  const double hl = (cvl[4] + cvl[nv]) * rli;
  const double hr = (cvr[4] + cvr[nv]) * rri;
  const double hm = rlc * hl + rrc * hr;
  double svm[ORC_MAX_SPEC];
  for (int l = 0; l < ns; ++l) svm[l] = rlc * cvl[l + 5] * rli + rrc * cvr[l + 5] * rri;
  double mw_inv = 0;
  for (int l = 0; l < ns; ++l) mw_inv += svm[l] / ch->mw[l];
  const double tl = cvl[nv] * rli, tr = cvr[nv] * rri;
  const double tm = (rlc * tl + rrc * tr) / (R_U * mw_inv);
  double cpi[ORC_MAX_SPEC], hi[ORC_MAX_SPEC];
  mix_h_cp(ch, tm, hi, cpi);
  double cp = 0, cvt = 0;
  for (int l = 0; l < ns; ++l) {
    cp += svm[l] * cpi[l];
    cvt += svm[l] * (cpi[l] - R_U / ch->mw[l]);
  }
  const double gamma = cp / cvt;
  const double cm = sqrt(gamma * R_U * mw_inv * tm);
  const double gm1 = gamma - 1;
  const double jl = jc[3], jr = jc[4];
  const double kxJ = m_l[0] * jl + m_r[0] * jr, kyJ = m_l[1] * jl + m_r[1] * jr, kzJ = m_l[2] * jl + m_r[2] * jr;
  double kx = kxJ / (jl + jr), ky = kyJ / (jl + jr), kz = kzJ / (jl + jr);
  const double gradK = sqrt(kx * kx + ky * ky + kz * kz);
  kx /= gradK;
  ky /= gradK;
  kz /= gradK;
  const double Ukb = kx * um + ky * vm + kz * wm;
  const double alpha = gm1 * ekm;
  const double c2i = 1.0 / (cm * cm);
  const double eps = 1e-40 * o->c.weno_eps_scale * 0.25 * (kxJ * kxJ + kyJ * kyJ + kzJ * kzJ);
  double al[ORC_MAX_SPEC];
  for (int l = 0; l < ns; ++l) {
    al[l] = gamma * R_U / ch->mw[l] * tm - (gamma - 1) * hi[l];
    al[l] *= c2i;
  }
  double fch[FVS_MAXV];
  for (int l = 0; l < 5; ++l) {
    double cs = 0.5, L[5];
    switch (l) {
      case 0:
        L[0] = (alpha + Ukb * cm) * c2i * 0.5;
        L[1] = -(gm1 * um + kx * cm) * c2i * 0.5;
        L[2] = -(gm1 * vm + ky * cm) * c2i * 0.5;
        L[3] = -(gm1 * wm + kz * cm) * c2i * 0.5;
        L[4] = gm1 * c2i * 0.5;
        break;
      case 1:
        cs = -kx;
        L[0] = kx * (1 - alpha * c2i) - (kz * vm - ky * wm) / cm;
        L[1] = kx * gm1 * um * c2i;
        L[2] = (kx * gm1 * vm + kz * cm) * c2i;
        L[3] = (kx * gm1 * wm - ky * cm) * c2i;
        L[4] = -kx * gm1 * c2i;
        break;
      case 2:
        cs = -ky;
        L[0] = ky * (1 - alpha * c2i) - (kx * wm - kz * um) / cm;
        L[1] = (ky * gm1 * um - kz * cm) * c2i;
        L[2] = ky * gm1 * vm * c2i;
        L[3] = (ky * gm1 * wm + kx * cm) * c2i;
        L[4] = -ky * gm1 * c2i;
        break;
      case 3:
        cs = -kz;
        L[0] = kz * (1 - alpha * c2i) - (ky * um - kx * vm) / cm;
        L[1] = (kz * gm1 * um + ky * cm) * c2i;
        L[2] = (kz * gm1 * vm - kx * cm) * c2i;
        L[3] = kz * gm1 * wm * c2i;
        L[4] = -kz * gm1 * c2i;
        break;
      default:
        L[0] = (alpha - Ukb * cm) * c2i * 0.5;
        L[1] = -(gm1 * um - kx * cm) * c2i * 0.5;
        L[2] = -(gm1 * vm - ky * cm) * c2i * 0.5;
        L[3] = -(gm1 * wm - kz * cm) * c2i * 0.5;
        L[4] = gm1 * c2i * 0.5;
        break;
    }
    double vp[7] = {0}, vmn[7] = {0};
    for (int m = 0; m < 7; ++m) {
      for (int n = 0; n < 5; ++n) {
        vp[m] += L[n] * Fp[m][n];
        vmn[m] += L[n] * Fm[m + 1][n];
      }
      for (int n = 0; n < ns; ++n) {
        vp[m] += cs * al[n] * Fp[m][5 + n];
        vmn[m] += cs * al[n] * Fm[m + 1][5 + n];
      }
    }
    fch[l] = fvs_weno7(vp, vmn, eps);
  }
  for (int l = 0; l < ns; ++l) {
    double vp[7], vmn[7];
    for (int m = 0; m < 7; ++m) {
      vp[m] = -svm[l] * Fp[m][0] + Fp[m][5 + l];
      vmn[m] = -svm[l] * Fm[m + 1][0] + Fm[m + 1][5 + l];
    }
    fch[5 + l] = fvs_weno7(vp, vmn, eps);
  }
  fc[0] = fch[0] + kx * fch[1] + ky * fch[2] + kz * fch[3] + fch[4];
  fc[1] = (um - kx * cm) * fch[0] + kx * um * fch[1] + (ky * um - kz * cm) * fch[2] + (kz * um + ky * cm) * fch[3] +
          (um + kx * cm) * fch[4];
  fc[2] = (vm - ky * cm) * fch[0] + (kx * vm + kz * cm) * fch[1] + ky * vm * fch[2] + (kz * vm - kx * cm) * fch[3] +
          (vm + ky * cm) * fch[4];
  fc[3] = (wm - kz * cm) * fch[0] + (kx * wm - ky * cm) * fch[1] + (ky * wm + kx * cm) * fch[2] + kz * wm * fch[3] +
          (wm + kz * cm) * fch[4];
  fc[4] = (hm - Ukb * cm) * fch[0] + (kx * (hm - cm * cm / gm1) + (kz * vm - ky * wm) * cm) * fch[1] +
          (ky * (hm - cm * cm / gm1) + (kx * wm - kz * um) * cm) * fch[2] +
          (kz * (hm - cm * cm / gm1) + (ky * um - kx * vm) * cm) * fch[3] + (hm + Ukb * cm) * fch[4];
  double add = 0;
  const double ca = fch[0] + kx * fch[1] + ky * fch[2] + kz * fch[3] + fch[4];
  for (int l = 0; l < ns; ++l) {
    fc[5 + l] = svm[l] * ca + fch[l + 5];
    add += al[l] * fch[l + 5];
  }
  fc[4] -= add * cm * cm / gm1;
}

/* compute_weno_flux_cp for inviscid_scheme 71 (WENO.cu:1455-1536): component-wise WENO7-Z of F+-
 * with eps scaled by the face metric and the reference velocity per equation group. */
static void fvs_cp_face(const orc_ctx *o, double Q[8][FVS_MAXV + 2], double mt[8][3], const double jc[8],
                        double *fc) {
  const int nv = o->nv;
  double Fp[8][FVS_MAXV], Fm[8][FVS_MAXV];
  for (int s = 0; s < 8; ++s) fvs_node_flux(Q[s], nv, mt[s], jc[s], Fp[s], Fm[s]);
  const double j1 = jc[3], j2 = jc[4];
  const double a0 = mt[3][0] * j1 + mt[4][0] * j2, a1 = mt[3][1] * j1 + mt[4][1] * j2, a2 = mt[3][2] * j1 + mt[4][2] * j2;
  const double eps_ref = 1e-20 * o->c.weno_eps_scale * 0.25 * (a0 * a0 + a1 * a1 + a2 * a2);
  double es[3];
  es[0] = eps_ref;
  es[1] = eps_ref * o->c.v_ref * o->c.v_ref;
  es[2] = es[1] * o->c.v_ref * o->c.v_ref;
  for (int l = 0; l < nv; ++l) {
    const double e = (l >= 1 && l <= 3) ? es[1] : (l == 4 ? es[2] : es[0]);
    double vp[7], vmn[7];
    for (int m = 0; m < 7; ++m) {
      vp[m] = Fp[m][l];
      vmn[m] = Fm[m + 1][l];
    }
    fc[l] = fvs_weno7(vp, vmn, e);
  }
}

/* compute_convective_term_weno_x/_y/_z (WENO.cu:8-461) for scheme 71 or 72 in direction dir: faces
 * idx+1/2 for idx = -1..n-1, dq -= fc(i+1/2) - fc(i-1/2). */
static void fvs_direction(orc_ctx *o, int dir) {
  const int ext[3] = {o->mx, o->my, o->mz};
  const int nv = o->nv;
  const long P = o->P, N = (long)o->mx * o->my * o->mz;
  int e[3] = {0, 0, 0};
  e[dir] = 1;
  const int n = ext[dir];
  int hi[3] = {o->mx, o->my, o->mz};
  hi[dir] = 1;
  double *fc = (double *)malloc(sizeof(double) * nv * (n + 1));
  for (int a = 0; a < hi[0]; ++a)
    for (int b = 0; b < hi[1]; ++b)
      for (int cc = 0; cc < hi[2]; ++cc) {
        for (int idx = -1; idx < n; ++idx) {
          double Q[8][FVS_MAXV + 2], mt[8][3], jc[8];
          for (int s = 0; s < 8; ++s) {
            const int off = idx - 3 + s;
            const long p = ID(o, a + off * e[0], b + off * e[1], cc + off * e[2]);
            for (int l = 0; l < nv; ++l) Q[s][l] = o->cv[l * P + p];
            Q[s][nv] = o->bv[4 * P + p];
            Q[s][nv + 1] = o->ns ? o->acs[p] : sqrt(GAMMA_AIR * (R_U / MW_AIR) * o->bv[5 * P + p]);
            for (int q = 0; q < 3; ++q) mt[s][q] = o->met[(long)(dir * 3 + q) * P + p];
            jc[s] = o->jac[p];
          }
          if (o->c.inviscid_scheme == 72) fvs_char_face(o, Q, mt, jc, &fc[nv * (idx + 1)]);
          else fvs_cp_face(o, Q, mt, jc, &fc[nv * (idx + 1)]);
        }
        for (int idx = 0; idx < n; ++idx) {
          const long q = IQ(o, a + idx * e[0], b + idx * e[1], cc + idx * e[2]);
          for (int l = 0; l < nv; ++l) o->dq[l * N + q] -= fc[nv * (idx + 1) + l] - fc[nv * idx + l];
        }
      }
  free(fc);
}

/* ---------------------------------------------------------------- viscous flux */

/* compute_fv/gv/hv_2nd_order<Air, Laminar> (ViscousScheme.cuh:24-318, 321-616, 619-911): face flux
 * between node (i,j,k) and its neighbour in direction d. */
/* Gradient (x, y, z) at the face between (i,j,k) and its d-neighbour of the padded plane B: 2-point
 * normal difference, 4-point averages across, chain rule with the face-averaged metric m. */
static void face_grad(const orc_ctx *o, const double *B, int i, int j, int k, int d, const double m[9], double out[3]) {
  int e[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  const long p0 = ID(o, i, j, k), p1 = ID(o, i + e[d][0], j + e[d][1], k + e[d][2]);
  double g[3];
  for (int c = 0; c < 3; ++c) {
    if (c == d) {
      g[c] = B[p1] - B[p0];
    } else {
      const int a0 = e[c][0], a1 = e[c][1], a2 = e[c][2];
      g[c] = 0.25 * (B[ID(o, i + a0, j + a1, k + a2)] - B[ID(o, i - a0, j - a1, k - a2)] +
                     B[ID(o, i + e[d][0] + a0, j + e[d][1] + a1, k + e[d][2] + a2)] -
                     B[ID(o, i + e[d][0] - a0, j + e[d][1] - a1, k + e[d][2] - a2)]);
    }
  }
  out[0] = g[0] * m[0] + g[1] * m[3] + g[2] * m[6];
  out[1] = g[0] * m[1] + g[1] * m[4] + g[2] * m[7];
  out[2] = g[0] * m[2] + g[1] * m[5] + g[2] * m[8];
}

static void viscous_face(const orc_ctx *o, int i, int j, int k, int d, double *fv) {
  const long P = o->P;
  int e[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  const long p0 = ID(o, i, j, k), p1 = ID(o, i + e[d][0], j + e[d][1], k + e[d][2]);
  double m[9];
  for (int r = 0; r < 9; ++r) m[r] = 0.5 * (o->met[r * P + p0] + o->met[r * P + p1]);
  const double *bv = o->bv;
  /* derivatives of u,v,w,T (bv 1,2,3,5) in computational coordinates */
  double g[4][3];
  const int var[4] = {1, 2, 3, 5};
  for (int q = 0; q < 4; ++q) {
    const double *B = bv + var[q] * P;
    for (int c = 0; c < 3; ++c) {
      if (c == d) {
        g[q][c] = B[p1] - B[p0];
      } else {
        const int a0 = e[c][0], a1 = e[c][1], a2 = e[c][2];
        g[q][c] = 0.25 * (B[ID(o, i + a0, j + a1, k + a2)] - B[ID(o, i - a0, j - a1, k - a2)] +
                          B[ID(o, i + e[d][0] + a0, j + e[d][1] + a1, k + e[d][2] + a2)] -
                          B[ID(o, i + e[d][0] - a0, j + e[d][1] - a1, k + e[d][2] - a2)]);
      }
    }
  }
  /* chain rule; m index (r-1)*3+(c-1): xi_x=m[0], xi_y=m[1], xi_z=m[2], eta_x=m[3] ... */
  double dx[4], dy[4], dz[4];
  for (int q = 0; q < 4; ++q) {
    dx[q] = g[q][0] * m[0] + g[q][1] * m[3] + g[q][2] * m[6];
    dy[q] = g[q][0] * m[1] + g[q][1] * m[4] + g[q][2] * m[7];
    dz[q] = g[q][0] * m[2] + g[q][1] * m[5] + g[q][2] * m[8];
  }
  const double u_x = dx[0], u_y = dy[0], u_z = dz[0];
  const double v_x = dx[1], v_y = dy[1], v_z = dz[1];
  const double w_x = dx[2], w_y = dy[2], w_z = dz[2];
  const double mul = 0.5 * (o->mul[p0] + o->mul[p1]);
  const double vis = mul;
  const double txx = vis * (4 * u_x - 2 * v_y - 2 * w_z) / 3.0;
  const double tyy = vis * (4 * v_y - 2 * u_x - 2 * w_z) / 3.0;
  const double tzz = vis * (4 * w_z - 2 * u_x - 2 * v_y) / 3.0;
  const double txy = vis * (u_y + v_x);
  const double txz = vis * (u_z + w_x);
  const double tyz = vis * (v_z + w_y);
  const double nx = 0.5 * (o->met[(d * 3 + 0) * P + p0] * o->jac[p0] + o->met[(d * 3 + 0) * P + p1] * o->jac[p1]);
  const double ny = 0.5 * (o->met[(d * 3 + 1) * P + p0] * o->jac[p0] + o->met[(d * 3 + 1) * P + p1] * o->jac[p1]);
  const double nz = 0.5 * (o->met[(d * 3 + 2) * P + p0] * o->jac[p0] + o->met[(d * 3 + 2) * P + p1] * o->jac[p1]);
  fv[0] = 0;
  fv[1] = nx * txx + ny * txy + nz * txz;
  fv[2] = nx * txy + ny * tyy + nz * tyz;
  fv[3] = nx * txz + ny * tyz + nz * tzz;
  const double um = 0.5 * (bv[P + p0] + bv[P + p1]);
  const double vm = 0.5 * (bv[2 * P + p0] + bv[2 * P + p1]);
  const double wm = 0.5 * (bv[3 * P + p0] + bv[3 * P + p1]);
  double cond;
  if (o->ns) {
    cond = 0.5 * (o->cond[p0] + o->cond[p1]);
  } else {
    const double cp = GAMMA_AIR * R_U / MW_AIR / (GAMMA_AIR - 1);
    cond = (mul / o->c.prandtl + 0.0 / 0.9) * cp;
  }
  fv[4] = um * fv[1] + vm * fv[2] + wm * fv[3] + cond * (nx * dx[3] + ny * dy[3] + nz * dz[3]);
  if (o->ns) {
    /* species diffusion, mixture-averaged with the correction velocity (ViscousScheme.cuh:126-206,
     * gradPInDiffusionFlux off) */
    const orc_chem *ch = o->c.chem;
    const int ns = o->ns;
    double dif[ORC_MAX_SPEC], yk[ORC_MAX_SPEC], ddf[ORC_MAX_SPEC];
    double sgw = 0, srdy = 0, corr = 0, mwt = 0;
    for (int l = 0; l < ns; ++l) {
      const double *Y = o->sv + (long)l * P;
      yk[l] = 0.5 * (Y[p0] + Y[p1]);
      dif[l] = 0.5 * (o->rhod[l * P + p0] + o->rhod[l * P + p1]) + 0.0;
      double gy[3];
      face_grad(o, Y, i, j, k, d, m, gy);
      const double gdy = nx * gy[0] + ny * gy[1] + nz * gy[2];
      ddf[l] = gdy;
      corr += dif[l] * gdy;
      sgw += gdy / ch->mw[l];
      mwt += yk[l] / ch->mw[l];
      srdy += dif[l] * yk[l];
    }
    mwt = 1.0 / mwt;
    corr -= mwt * srdy * sgw;
    double h[ORC_MAX_SPEC];
    mix_h_cp(ch, 0.5 * (bv[5 * P + p0] + bv[5 * P + p1]), h, NULL);
    for (int l = 0; l < ns; ++l) {
      const double flux = dif[l] * (ddf[l] - mwt * yk[l] * sgw) - yk[l] * corr;
      fv[5 + l] = flux;
      fv[4] += h[l] * flux;
    }
  }
}

/* viscous_flux_fv/gv/hv (SchemeSelector.cuh:69-154) */
static void viscous(orc_ctx *o) {
  const int ext[3] = {o->mx, o->my, o->mz};
  const long N = (long)o->mx * o->my * o->mz;
  for (int d = 0; d < o->dim; ++d) {
    for (int k = 0; k < o->mz; ++k)
      for (int j = 0; j < o->my; ++j)
        for (int i = 0; i < o->mx; ++i) {
          const int c[3] = {i, j, k};
          double fl[FVS_MAXV], fr[FVS_MAXV];
          viscous_face(o, i - (d == 0), j - (d == 1), k - (d == 2), d, fl);
          viscous_face(o, i, j, k, d, fr);
          (void)c;
          (void)ext;
          const long q = IQ(o, i, j, k);
          for (int l = 0; l < o->nv; ++l) o->dq[l * N + q] += fr[l] - fl[l];
        }
  }
}

/* ---------------------------------------------------------------- boundary conditions */

static void copy_node(orc_ctx *o, long dst, long src) {
  for (int l = 0; l < 6; ++l) o->bv[l * o->P + dst] = o->bv[l * o->P + src];
  for (int l = 0; l < o->ns; ++l) o->sv[l * o->P + dst] = o->sv[l * o->P + src];
}

/* apply_symmetry (BoundCond.cuh:137-203) */
static void bc_symmetry(orc_ctx *o, const face_t *f) {
  const long P = o->P;
  int dir[3] = {0, 0, 0};
  dir[f->face] = f->direction;
  for (int i = f->rs[0]; i <= f->re[0]; ++i)
    for (int j = f->rs[1]; j <= f->re[1]; ++j)
      for (int k = f->rs[2]; k <= f->re[2]; ++k) {
        const long pb = ID(o, i, j, k), pin = ID(o, i - dir[0], j - dir[1], k - dir[2]);
        double kx = o->met[(f->face * 3 + 0) * P + pb], ky = o->met[(f->face * 3 + 1) * P + pb],
               kz = o->met[(f->face * 3 + 2) * P + pb];
        const double km = sqrt(kx * kx + ky * ky + kz * kz);
        kx /= km;
        ky /= km;
        kz /= km;
        const double u1 = o->bv[P + pin], v1 = o->bv[2 * P + pin], w1 = o->bv[3 * P + pin];
        double uk = kx * u1 + ky * v1 + kz * w1;
        o->bv[P + pb] = u1 - kx * uk;
        o->bv[2 * P + pb] = v1 - ky * uk;
        o->bv[3 * P + pb] = w1 - kz * uk;
        o->bv[pb] = o->bv[pin];
        o->bv[4 * P + pb] = o->bv[4 * P + pin];
        o->bv[5 * P + pb] = o->bv[5 * P + pin];
        for (int l = 0; l < o->ns; ++l) o->sv[l * P + pb] = o->sv[l * P + pin];
        for (int g = 1; g <= o->g; ++g) {
          const long pg = ID(o, i + g * dir[0], j + g * dir[1], k + g * dir[2]);
          const long pi = ID(o, i - g * dir[0], j - g * dir[1], k - g * dir[2]);
          o->bv[pg] = o->bv[pi];
          const double u = o->bv[P + pi], v = o->bv[2 * P + pi], w = o->bv[3 * P + pi];
          uk = kx * u + ky * v + kz * w;
          o->bv[P + pg] = u - 2 * uk * kx;
          o->bv[2 * P + pg] = v - 2 * uk * ky;
          o->bv[3 * P + pg] = w - 2 * uk * kz;
          o->bv[4 * P + pg] = o->bv[4 * P + pi];
          o->bv[5 * P + pg] = o->bv[5 * P + pi];
          for (int l = 0; l < o->ns; ++l) o->sv[l * P + pg] = o->sv[l * P + pi];
          cv_from_bv(o, pg);
        }
      }
}

/* apply_outflow (BoundCond.cuh:205-233) */
static void bc_outflow(orc_ctx *o, const face_t *f) {
  int dir[3] = {0, 0, 0};
  dir[f->face] = f->direction;
  for (int i = f->rs[0]; i <= f->re[0]; ++i)
    for (int j = f->rs[1]; j <= f->re[1]; ++j)
      for (int k = f->rs[2]; k <= f->re[2]; ++k)
        for (int g = 1; g <= o->g; ++g) {
          const long pg = ID(o, i + g * dir[0], j + g * dir[1], k + g * dir[2]);
          copy_node(o, pg, ID(o, i, j, k));
          cv_from_bv(o, pg);
        }
}

/* apply_inflow with a constant state (BoundCond.cuh:483-613): the face node and its ghost layers
 * take the inflow state and mass fractions. */
/* apply_inflow (BoundCond.cuh:235-613) without fluctuation: the face node and its ghost layers take
 * the constant state, or (inflow_type 2) the upper / lower stream by the sign of the face node's y with
 * u = (u1 + u2) / 2 + (u1 - u2) / 2 tanh(2 y / delta_omega) (BoundCond.cuh:384-400). */
static void bc_inflow(orc_ctx *o, const face_t *f) {
  const long P = o->P;
  int dir[3] = {0, 0, 0};
  dir[f->face] = f->direction;
  for (int i = f->rs[0]; i <= f->re[0]; ++i)
    for (int j = f->rs[1]; j <= f->re[1]; ++j)
      for (int k = f->rs[2]; k <= f->re[2]; ++k) {
        double st[6] = {f->density, f->u, f->v, f->w, f->pressure, f->temperature};
        const double *ys = f->y;
        if (f->inflow_type == 2) {
          const double yc = o->y[IC(o, i, j, k)];
          if (yc < 0) {
            for (int l = 0; l < 6; ++l) st[l] = f->lower[l];
            ys = f->y_lower;
          }
          st[1] = 0.5 * (f->u + f->lower[1]) + 0.5 * (f->u - f->lower[1]) * tanh(2 * yc / f->delta_omega);
        }
        for (int g = 0; g <= o->g; ++g) {
          const long pg = ID(o, i + g * dir[0], j + g * dir[1], k + g * dir[2]);
          for (int l = 0; l < 6; ++l) o->bv[l * P + pg] = st[l];
          for (int l = 0; l < o->ns; ++l) o->sv[l * P + pg] = ys[l];
          cv_from_bv(o, pg);
        }
      }
}

/* apply_back_pressure / apply_subsonic_inflow (BoundCond.cuh:1272-1441), air: the face node keeps its
 * values; back pressure: subsonic normal flow takes p_b and the first interior node's characteristic
 * state at the face, ghosts extrapolate through it (2 q_b - q_in), supersonic copies the face node;
 * subsonic inflow: speed of sound from the quadratic that keeps the face node's negative Riemann
 * invariant and total enthalpy, then p and T from the total state, the same in every ghost layer. */
static void bc_characteristic(orc_ctx *o, const face_t *f) {
  const long P = o->P;
  const double g = GAMMA_AIR;
  int dir[3] = {0, 0, 0};
  dir[f->face] = f->direction;
  for (int i = f->rs[0]; i <= f->re[0]; ++i)
    for (int j = f->rs[1]; j <= f->re[1]; ++j)
      for (int k = f->rs[2]; k <= f->re[2]; ++k) {
        const long pb = ID(o, i, j, k);
        double nx = o->met[(f->face * 3 + 0) * P + pb], ny = o->met[(f->face * 3 + 1) * P + pb],
               nz = o->met[(f->face * 3 + 2) * P + pb];
        const double gni = f->direction / sqrt(nx * nx + ny * ny + nz * nz);
        nx *= gni;
        ny *= gni;
        nz *= gni;
        const double rb = o->bv[pb], ub = o->bv[P + pb], vb = o->bv[2 * P + pb], wb = o->bv[3 * P + pb];
        const double pbv = o->bv[4 * P + pb];
        const double u_face = nx * ub + ny * vb + nz * wb;
        const double ab = sqrt(g * pbv / rb);
        if (f->type == ORC_BACK_PRESSURE) {
          double rho_b = rb, u_b = ub, v_b = vb, w_b = wb, p_b = pbv;
          const int sub = fabs(u_face / ab) < 1;
          if (sub) {
            p_b = f->pressure;
            const long p1 = ID(o, i - dir[0], j - dir[1], k - dir[2]);
            const double d1 = o->bv[p1], u1 = o->bv[P + p1], v1 = o->bv[2 * P + p1], w1 = o->bv[3 * P + p1];
            const double pr1 = o->bv[4 * P + p1];
            const double c1 = sqrt(g * pr1 / d1);
            rho_b = d1 + (p_b - pr1) / (c1 * c1);
            u_b = u1 + nx * (pr1 - p_b) / (d1 * c1);
            v_b = v1 + ny * (pr1 - p_b) / (d1 * c1);
            w_b = w1 + nz * (pr1 - p_b) / (d1 * c1);
          }
          for (int q = 1; q <= o->g; ++q) {
            const long pg = ID(o, i + q * dir[0], j + q * dir[1], k + q * dir[2]);
            const long pi = ID(o, i - q * dir[0], j - q * dir[1], k - q * dir[2]);
            double r = rho_b, u = u_b, v = v_b, w = w_b, pr = p_b;
            if (sub) {
              pr = 2 * p_b - o->bv[4 * P + pi];
              r = 2 * rho_b - o->bv[pi];
              u = 2 * u_b - o->bv[P + pi];
              v = 2 * v_b - o->bv[2 * P + pi];
              w = 2 * w_b - o->bv[3 * P + pi];
            }
            o->bv[pg] = r;
            o->bv[P + pg] = u;
            o->bv[2 * P + pg] = v;
            o->bv[3 * P + pg] = w;
            o->bv[4 * P + pg] = pr;
            o->bv[5 * P + pg] = pr / (r * R_U / MW_AIR);
            cv_from_bv(o, pg);
          }
        } else {
          const double rn = fabs(u_face) - 2 * ab / (g - 1);
          const double hti = pbv / rb * g / (g - 1) + 0.5 * (ub * ub + vb * vb + wb * wb);
          const double qa = 1 + 2.0 / (g - 1), qb = 2 * rn, qc = (g - 1) * (0.5 * rn * rn - hti);
          const double delta = qb * qb - 4 * qa * qc;
          double a_new = ab;
          if (delta >= 0) {
            const double ap = (-qb + sqrt(delta)) / (2 * qa), am = (-qb - sqrt(delta)) / (2 * qa);
            a_new = ap > am ? ap : am;
          }
          const double u_new = rn + 2 * a_new / (g - 1);
          const double mach = u_new / a_new;
          const double pr = f->pressure * pow(1 + 0.5 * (g - 1) * mach * mach, -g / (g - 1));
          const double tt = f->temperature * pow(pr / f->pressure, (g - 1) / g);
          const double r = pr * MW_AIR / (tt * R_U);
          for (int q = 1; q <= o->g; ++q) {
            const long pg = ID(o, i + q * dir[0], j + q * dir[1], k + q * dir[2]);
            o->bv[pg] = r;
            o->bv[P + pg] = u_new * f->u;
            o->bv[2 * P + pg] = u_new * f->v;
            o->bv[3 * P + pg] = u_new * f->w;
            o->bv[4 * P + pg] = pr;
            o->bv[5 * P + pg] = tt;
            cv_from_bv(o, pg);
          }
        }
      }
}

/* mixture molecular weight of node p from its mass fractions */
static double node_mw(const orc_ctx *o, long p) {
  if (!o->ns) return MW_AIR;
  double s = 0;
  for (int l = 0; l < o->ns; ++l) s += o->sv[l * o->P + p] / o->c.chem->mw[l];
  return 1 / s;
}

/* apply_wall (BoundCond.cuh:1024-1270) without blowing or fluctuations: the wall node gets the first
 * interior node's p (and Y), T_w (isothermal) or that node's T (adiabatic), zero velocity; ghost g
 * mirrors interior node g: p and Y copied, velocity reversed, T_g = 2 T_w - T_in (isothermal; T_w
 * when that is <= 0.1 T_w) or T_in (adiabatic), rho from the equation of state. */
static void bc_wall(orc_ctx *o, const face_t *f) {
  const long P = o->P;
  int dir[3] = {0, 0, 0};
  dir[f->face] = f->direction;
  for (int i = f->rs[0]; i <= f->re[0]; ++i)
    for (int j = f->rs[1]; j <= f->re[1]; ++j)
      for (int k = f->rs[2]; k <= f->re[2]; ++k) {
        const long pb = ID(o, i, j, k), pin = ID(o, i - dir[0], j - dir[1], k - dir[2]);
        const double tw = f->wall_adiabatic ? o->bv[5 * P + pin] : f->temperature;
        const double pw = o->bv[4 * P + pin];
        for (int l = 0; l < o->ns; ++l) o->sv[l * P + pb] = o->sv[l * P + pin];
        o->bv[pb] = pw * node_mw(o, pb) / (tw * R_U);
        o->bv[P + pb] = 0;
        o->bv[2 * P + pb] = 0;
        o->bv[3 * P + pb] = 0;
        o->bv[4 * P + pb] = pw;
        o->bv[5 * P + pb] = tw;
        cv_from_bv(o, pb);
        for (int g = 1; g <= o->g; ++g) {
          const long pi = ID(o, i - g * dir[0], j - g * dir[1], k - g * dir[2]);
          const long pg = ID(o, i + g * dir[0], j + g * dir[1], k + g * dir[2]);
          const double p_i = o->bv[4 * P + pi], t_i = o->bv[5 * P + pi];
          double t_g = t_i;
          if (!f->wall_adiabatic) {
            t_g = 2 * tw - t_i;
            if (t_g <= 0.1 * tw) t_g = tw;
          }
          for (int l = 0; l < o->ns; ++l) o->sv[l * P + pg] = o->sv[l * P + pi];
          o->bv[pg] = p_i * node_mw(o, pg) / (t_g * R_U);
          o->bv[P + pg] = -o->bv[P + pi];
          o->bv[2 * P + pg] = -o->bv[2 * P + pi];
          o->bv[3 * P + pg] = -o->bv[3 * P + pi];
          o->bv[4 * P + pg] = p_i;
          o->bv[5 * P + pg] = t_g;
          cv_from_bv(o, pg);
        }
      }
}

/* apply_periodic (BoundCond.cuh:1443-1486): node-coincident, ghost mx-1+g <- interior g. */
static void bc_periodic(orc_ctx *o, const face_t *f) {
  int dir[3] = {0, 0, 0};
  dir[f->face] = f->direction;
  const int ext[3] = {o->mx, o->my, o->mz};
  for (int i = f->rs[0]; i <= f->re[0]; ++i)
    for (int j = f->rs[1]; j <= f->re[1]; ++j)
      for (int k = f->rs[2]; k <= f->re[2]; ++k) {
        int other[3] = {i, j, k};
        other[f->face] = f->direction < 0 ? ext[f->face] - 1 : 0;
        for (int g = 1; g <= o->g; ++g) {
          const long pg = ID(o, i + g * dir[0], j + g * dir[1], k + g * dir[2]);
          const long ps = ID(o, other[0] + g * dir[0], other[1] + g * dir[1], other[2] + g * dir[2]);
          copy_node(o, pg, ps);
          cv_from_bv(o, pg);
        }
      }
}

/* apply_farfield<Air> (BoundCond.cuh:755-1022) */
/* apply_farfield<mixture> (BoundCond.cuh:755-1022) at face node (i, j, k): gamma of the node, mixture
 * molecular weight from its mass fractions; supersonic inflow / outflow as for air; subsonic: Riemann
 * invariants, far-field (u_n < 0) or node velocity and composition, and a gamma iterated with cp of
 * the face temperature until its relative change is below 1e-4 (entropy of the inflow branch for
 * u_n <= 0, as the reference writes it). */
static void farfield_mixture_node(orc_ctx *o, const face_t *f, int i, int j, int k, const int dir[3]) {
  const long P = o->P;
  const orc_chem *ch = o->c.chem;
  const int ns = o->ns;
  const long pb = ID(o, i, j, k);
  double nx = o->met[(f->face * 3 + 0) * P + pb], ny = o->met[(f->face * 3 + 1) * P + pb],
         nz = o->met[(f->face * 3 + 2) * P + pb];
  const double gni = f->direction / sqrt(nx * nx + ny * ny + nz * nz);
  nx *= gni;
  ny *= gni;
  nz *= gni;
  const double ub = o->bv[P + pb], vb = o->bv[2 * P + pb], wb = o->bv[3 * P + pb];
  const double uf = nx * ub + ny * vb + nz * wb;
  double svb[ORC_MAX_SPEC];
  for (int l = 0; l < ns; ++l) svb[l] = o->sv[l * P + pb];
  const double gb = o->gam[pb];
  double mw_inv = 0;
  for (int l = 0; l < ns; ++l) mw_inv += svb[l] / ch->mw[l];
  double mw = 1.0 / mw_inv;
  const double pbv = o->bv[4 * P + pb], rb = o->bv[pb];
  const double ab = sqrt(gb * pbv / rb);
  const double mb = uf / ab;
  double vals[6];
  if (mb <= -1) {
    vals[0] = f->density; vals[1] = f->u; vals[2] = f->v; vals[3] = f->w; vals[4] = f->pressure;
    vals[5] = f->temperature;
    for (int l = 0; l < ns; ++l) svb[l] = f->y[l];
  } else if (mb >= 1) {
    for (int g = 1; g <= o->g; ++g) {
      const long pg = ID(o, i + g * dir[0], j + g * dir[1], k + g * dir[2]);
      copy_node(o, pg, pb);
      cv_from_bv(o, pg);
    }
    return;
  } else {
    const double rpos = uf + 2 * ab / (gb - 1);
    const double uinf = f->u * nx + f->v * ny + f->w * nz;
    const double rneg = uinf - 2 * f->acoustic_speed / (f->gamma - 1);
    const double Un = 0.5 * (rpos + rneg);
    if (mb < 0) {
      vals[1] = f->u + (Un - uinf) * nx;
      vals[2] = f->v + (Un - uinf) * ny;
      vals[3] = f->w + (Un - uinf) * nz;
      for (int l = 0; l < ns; ++l) svb[l] = f->y[l];
      mw = f->mw;
    } else {
      vals[1] = ub + (Un - uf) * nx;
      vals[2] = vb + (Un - uf) * ny;
      vals[3] = wb + (Un - uf) * nz;
    }
    double gamma = GAMMA_AIR, err = 1, rho = 0, pr = 0, t = 0;
    for (int it = 0; err > 1e-4 && it < 100; ++it) {
      const double glast = gamma;
      const double cb = 0.25 * (gamma - 1) * (rpos - rneg);
      const double sb = mb <= 0 ? f->entropy : pbv / pow(rb, gamma);
      rho = pow(cb * cb / (gamma * sb), 1 / (gamma - 1));
      pr = rho * cb * cb / gamma;
      t = pr * mw / (rho * R_U);
      double h[ORC_MAX_SPEC], cp[ORC_MAX_SPEC];
      mix_h_cp(ch, t, h, cp);
      double cpt = 0;
      for (int l = 0; l < ns; ++l) cpt += cp[l] * svb[l];
      gamma = cpt / (cpt - R_U / mw);
      err = fabs(1 - gamma / glast);
    }
    vals[0] = rho;
    vals[4] = pr;
    vals[5] = t;
  }
  for (int g = 0; g <= o->g; ++g) {
    const long pg = ID(o, i + g * dir[0], j + g * dir[1], k + g * dir[2]);
    for (int l = 0; l < 6; ++l) o->bv[l * P + pg] = vals[l];
    for (int l = 0; l < ns; ++l) o->sv[l * P + pg] = svb[l];
    cv_from_bv(o, pg);
  }
}

static void bc_farfield(orc_ctx *o, const face_t *f) {
  const long P = o->P;
  int dir[3] = {0, 0, 0};
  dir[f->face] = f->direction;
  if (o->ns) {
    for (int i = f->rs[0]; i <= f->re[0]; ++i)
      for (int j = f->rs[1]; j <= f->re[1]; ++j)
        for (int k = f->rs[2]; k <= f->re[2]; ++k) farfield_mixture_node(o, f, i, j, k, dir);
    return;
  }
  for (int i = f->rs[0]; i <= f->re[0]; ++i)
    for (int j = f->rs[1]; j <= f->re[1]; ++j)
      for (int k = f->rs[2]; k <= f->re[2]; ++k) {
        const long pb = ID(o, i, j, k);
        double nx = o->met[(f->face * 3 + 0) * P + pb], ny = o->met[(f->face * 3 + 1) * P + pb],
               nz = o->met[(f->face * 3 + 2) * P + pb];
        const double gni = f->direction / sqrt(nx * nx + ny * ny + nz * nz);
        nx *= gni;
        ny *= gni;
        nz *= gni;
        const double ub = o->bv[P + pb], vb = o->bv[2 * P + pb], wb = o->bv[3 * P + pb];
        const double uf = nx * ub + ny * vb + nz * wb;
        const double gam = GAMMA_AIR;
        const double pbv = o->bv[4 * P + pb], rb = o->bv[pb];
        const double ab = sqrt(gam * pbv / rb);
        const double mb = uf / ab;
        double rho, u, v, w, p, t;
        if (mb <= -1) {
          rho = f->density; u = f->u; v = f->v; w = f->w; p = f->pressure; t = f->temperature;
        } else if (mb >= 1) {
          for (int g = 1; g <= o->g; ++g) {
            const long pg = ID(o, i + g * dir[0], j + g * dir[1], k + g * dir[2]);
            copy_node(o, pg, pb);
            cv_from_bv(o, pg);
          }
          continue;
        } else {
          const double rpos = uf + 2 * ab / (gam - 1);
          const double uinf = f->u * nx + f->v * ny + f->w * nz;
          const double rneg = uinf - 2 * f->acoustic_speed / (f->gamma - 1);
          const double Un = 0.5 * (rpos + rneg);
          const double cb = 0.25 * (GAMMA_AIR - 1) * (rpos - rneg);
          double sb;
          if (mb <= 0) {
            sb = f->entropy;
            u = f->u + (Un - uinf) * nx;
            v = f->v + (Un - uinf) * ny;
            w = f->w + (Un - uinf) * nz;
          } else {
            sb = pbv / pow(rb, GAMMA_AIR);
            u = ub + (Un - uf) * nx;
            v = vb + (Un - uf) * ny;
            w = wb + (Un - uf) * nz;
          }
          rho = pow(cb * cb / (GAMMA_AIR * sb), 1 / (GAMMA_AIR - 1));
          p = rho * cb * cb / GAMMA_AIR;
          t = p * MW_AIR / (rho * R_U);
        }
        const double vals[6] = {rho, u, v, w, p, t};
        for (int l = 0; l < 6; ++l) o->bv[l * P + pb] = vals[l];
        cv_from_bv(o, pb);
        for (int g = 1; g <= o->g; ++g) {
          const long pg = ID(o, i + g * dir[0], j + g * dir[1], k + g * dir[2]);
          for (int l = 0; l < 6; ++l) o->bv[l * P + pg] = vals[l];
          cv_from_bv(o, pg);
        }
      }
}

/* DBoundCond::apply_boundary_conditions priority order (BoundCond.cuh:1488-1679):
 * farfield, outflow, symmetry, periodic (other types are not on this path). */
static void apply_bcs(orc_ctx *o) {
  /* priority order of DBoundCond::apply_boundary_conditions (BoundCond.cuh:1488-1679) */
  const int order[8] = {ORC_FARFIELD, ORC_OUTFLOW, ORC_BACK_PRESSURE, ORC_INFLOW, ORC_SUBSONIC_INFLOW,
                        ORC_SYMMETRY, ORC_WALL, ORC_PERIODIC};
  for (int t = 0; t < 8; ++t)
    for (int n = 0; n < o->nf; ++n) {
      const face_t *f = &o->f[n];
      if (f->type != order[t]) continue;
      switch (f->type) {
        case ORC_FARFIELD: bc_farfield(o, f); break;
        case ORC_OUTFLOW: bc_outflow(o, f); break;
        case ORC_SYMMETRY: bc_symmetry(o, f); break;
        case ORC_PERIODIC: bc_periodic(o, f); break;
        case ORC_WALL: bc_wall(o, f); break;
        case ORC_INFLOW: bc_inflow(o, f); break;
        case ORC_BACK_PRESSURE:
        case ORC_SUBSONIC_INFLOW: bc_characteristic(o, f); break;
      }
    }
}

/* eliminate_k_gradient (FieldOperation.cu:42-67) */
static void eliminate_k(orc_ctx *o) {
  const long P = o->P;
  for (int j = -o->g; j < o->my + o->g; ++j)
    for (int i = -o->g; i < o->mx + o->g; ++i)
      for (int k = 1; k <= o->g; ++k) {
        const long p0 = ID(o, i, j, 0), pp = ID(o, i, j, k), pm = ID(o, i, j, -k);
        for (int l = 0; l < 6; ++l) {
          o->bv[l * P + pp] = o->bv[l * P + p0];
          o->bv[l * P + pm] = o->bv[l * P + p0];
        }
        for (int l = 0; l < o->ns; ++l) {
          o->sv[l * P + pp] = o->sv[l * P + p0];
          o->sv[l * P + pm] = o->sv[l * P + p0];
        }
        for (int l = 0; l < o->nv; ++l) {
          o->cv[l * P + pp] = o->cv[l * P + p0];
          o->cv[l * P + pm] = o->cv[l * P + p0];
        }
      }
}

/* update_physical_properties<Air> (FieldOperation.cuh:107-140): mu over the padded block */
static void mix_properties_node(orc_ctx *o, long p);
static void properties(orc_ctx *o) {
  if (o->ns) {
    for (long p = 0; p < o->P; ++p) mix_properties_node(o, p);
    return;
  }
  for (long p = 0; p < o->P; ++p) o->mul[p] = sutherland(o->bv[5 * o->P + p]);
}

/* local_time_step<Air, Laminar> (TimeAdvanceFunc.cuh:28-83) and the min of global_time_step
 * (TimeAdvanceFunc.cu:39-64, initial value 1e6). */
double orc_dt(orc_ctx *o) {
  const long P = o->P;
  double dt = 1e6;
  for (int k = 0; k < o->mz; ++k)
    for (int j = 0; j < o->my; ++j)
      for (int i = 0; i < o->mx; ++i) {
        const long p = ID(o, i, j, k);
        double m[9];
        for (int r = 0; r < 9; ++r) m[r] = o->met[r * P + p];
        const double gx = sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
        const double ge = sqrt(m[3] * m[3] + m[4] * m[4] + m[5] * m[5]);
        const double gz = sqrt(m[6] * m[6] + m[7] * m[7] + m[8] * m[8]);
        const double u = o->bv[P + p], v = o->bv[2 * P + p], w = o->bv[3 * P + p];
        const double U = u * m[0] + v * m[1] + w * m[2];
        const double V = u * m[3] + v * m[4] + w * m[5];
        const double W = u * m[6] + v * m[7] + w * m[8];
        const double a = o->ns ? o->acs[p] : sqrt(GAMMA_AIR * R_U * o->bv[5 * P + p] / MW_AIR);
        const double s0 = fabs(U) + a * gx, s1 = fabs(V) + a * ge;
        const double s2 = o->dim == 3 ? fabs(W) + a * gz : 0;
        const double sinv = s0 + s1 + s2;
        const double c1 = fmax(o->ns ? o->gam[p] : GAMMA_AIR, 4.0 / 3.0) / o->bv[p];
        const double c2 = o->mul[p] / o->c.prandtl;
        double sv = gx * gx + ge * ge;
        if (o->dim == 3) sv += gz * gz;
        sv *= c1 * c2;
        const double d = o->c.cfl / (sinv + sv);
        o->dtl[IQ(o, i, j, k)] = d;
        if (o->srad) {
          o->srad[3 * IQ(o, i, j, k)] = s0;
          o->srad[3 * IQ(o, i, j, k) + 1] = s1;
          o->srad[3 * IQ(o, i, j, k) + 2] = s2;
        }
        if (d < dt) dt = d;
      }
  return dt;
}

/* update_cv_and_bv_rk<Air> (RK.cuh:230-284) */
static void rk_update(orc_ctx *o, double dt, int rk) {
  static const double A[3] = {1.0, 0.75, 1.0 / 3.0}, B[3] = {0.0, 0.25, 2.0 / 3.0}, C[3] = {1.0, 0.25, 2.0 / 3.0};
  const long P = o->P, N = (long)o->mx * o->my * o->mz;
  for (int k = 0; k < o->mz; ++k)
    for (int j = 0; j < o->my; ++j)
      for (int i = 0; i < o->mx; ++i) {
        const long p = ID(o, i, j, k), q = IQ(o, i, j, k);
        const double dtj = dt / o->jac[p];
        for (int l = 0; l < o->nv; ++l)
          o->cv[l * P + p] = A[rk] * o->qn[l * P + p] + B[rk] * o->cv[l * P + p] + C[rk] * dtj * o->dq[l * N + q];
        if (o->mz == 1) o->cv[3 * P + p] = 0;
        o->bv[p] = o->cv[p];
        const double di = 1.0 / o->cv[p];
        o->bv[P + p] = o->cv[P + p] * di;
        o->bv[2 * P + p] = o->cv[2 * P + p] * di;
        o->bv[3 * P + p] = o->cv[3 * P + p] * di;
        const double V2 = o->bv[P + p] * o->bv[P + p] + o->bv[2 * P + p] * o->bv[2 * P + p] +
                          o->bv[3 * P + p] * o->bv[3 * P + p];
        if (o->ns) {
          for (int l = 0; l < o->ns; ++l) o->sv[l * P + p] = o->cv[(5 + l) * P + p] * di;
          mix_t_and_p(o, p, o->cv[4 * P + p]);
        } else {
          o->bv[4 * P + p] = (GAMMA_AIR - 1) * (o->cv[4 * P + p] - 0.5 * o->bv[p] * V2);
          o->bv[5 * P + p] = o->bv[4 * P + p] * MW_AIR * di / R_U;
        }
      }
}

static void fill_ghosts(orc_ctx *o) {
  apply_bcs(o);
  if (o->dim == 2) eliminate_k(o);
  properties(o);
}

/* ---------------------------------------------------------------- public entry points */

static orc_ctx *create_block(const orc_case *c, const double *x, const double *y, const double *z, int finish);

orc_ctx *orc_create(const orc_case *c, const double *x, const double *y, const double *z) {
  return create_block(c, x, y, z, 1);
}

/* finish = 0 leaves the edge / corner ghost coordinates and the metric to the caller, which first
 * copies the interface ghost layers from the neighbours (multi-block). */
static orc_ctx *create_block(const orc_case *c, const double *x, const double *y, const double *z, int finish) {
  orc_ctx *o = (orc_ctx *)calloc(1, sizeof(orc_ctx));
  o->c = *c;
  o->mx = c->mx;
  o->my = c->my;
  o->mz = c->mz;
  o->dim = c->mz == 1 ? 2 : 3;
  o->g = c->reconstruction == 5 ? 4 : c->reconstruction == 4 ? 3 : 2; /* Parameter.cpp:194-248 */
  if (c->inviscid_scheme == 71 || c->inviscid_scheme == 72) o->g = 4;
  o->ns = c->n_spec;
  o->nv = 5 + c->n_spec;
  o->sx = o->mx + 2 * o->g;
  o->sy = o->my + 2 * o->g;
  o->sz = o->mz + 2 * o->g;
  o->P = (long)o->sx * o->sy * o->sz;
  o->cx = o->mx + 2 * o->g + 2;
  o->cy = o->my + 2 * o->g + 2;
  o->cz = o->mz + 2 * o->g + 2;
  o->PC = (long)o->cx * o->cy * o->cz;
  o->x = (double *)calloc(o->PC, sizeof(double));
  o->y = (double *)calloc(o->PC, sizeof(double));
  o->z = (double *)calloc(o->PC, sizeof(double));
  for (int k = 0; k < o->mz; ++k)
    for (int j = 0; j < o->my; ++j)
      for (int i = 0; i < o->mx; ++i) {
        const long s = ((long)k * o->my + j) * o->mx + i;
        o->x[IC(o, i, j, k)] = x[s];
        o->y[IC(o, i, j, k)] = y[s];
        o->z[IC(o, i, j, k)] = z[s];
      }
  o->jac = (double *)calloc(o->P, sizeof(double));
  o->met = (double *)calloc(9 * o->P, sizeof(double));
  ghost_grid(o);
  if (finish) {
    ghost_grid_edges(o);
    compute_metric(o);
  }
  const long N = (long)o->mx * o->my * o->mz;
  o->cv = (double *)calloc(o->nv * o->P, sizeof(double));
  o->qn = (double *)calloc(o->nv * o->P, sizeof(double));
  o->bv = (double *)calloc(6 * o->P, sizeof(double));
  o->mul = (double *)calloc(o->P, sizeof(double));
  o->dq = (double *)calloc(o->nv * N, sizeof(double));
  o->sv = (double *)calloc(o->ns * o->P + 1, sizeof(double));
  o->rhod = (double *)calloc(o->ns * o->P + 1, sizeof(double));
  o->cond = (double *)calloc(o->P, sizeof(double));
  o->cpm = (double *)calloc(o->P, sizeof(double));
  o->gam = (double *)calloc(o->P, sizeof(double));
  o->acs = (double *)calloc(o->P, sizeof(double));
  o->dtl = (double *)calloc(N, sizeof(double));
  o->nf = c->n_face;
  for (int n = 0; n < c->n_face; ++n) register_face(o, &c->face[n], &o->f[n]);
  return o;
}

void orc_destroy(orc_ctx *o) {
  if (!o) return;
  free(o->x); free(o->y); free(o->z); free(o->jac); free(o->met);
  free(o->cv); free(o->qn); free(o->bv); free(o->mul); free(o->dq); free(o->dtl);
  free(o->sv); free(o->rhod); free(o->cond); free(o->cpm); free(o->gam); free(o->acs);
  free(o->srad); free(o->cj); free(o->dq0); free(o->dqk); free(o->qn1); free(o->qstar); free(o->inlast);
  free(o);
}

int orc_ngg(const orc_ctx *o) { return o->g; }

double orc_time(const orc_ctx *o) { return o->t; }

/* Initialisation: Driver::initialize_computation (Driver.cu:115-199) then compute_cv_from_bv over
 * the padded block at the start of RK3 (RK.cuh:37-45). */
void orc_set_state(orc_ctx *o, const double *bv) { orc_set_state_sv(o, bv, NULL); }

static void load_state(orc_ctx *o, const double *bv, const double *sv);

void orc_set_state_sv(orc_ctx *o, const double *bv, const double *sv) {
  load_state(o, bv, sv);
  if (o->dim == 2) eliminate_k(o);
  apply_bcs(o);
  properties(o);
  for (long p = 0; p < o->P; ++p) cv_from_bv(o, p);
  o->t = 0;
}

static void load_state(orc_ctx *o, const double *bv, const double *sv) {
  const long P = o->P, N = (long)o->mx * o->my * o->mz;
  memset(o->bv, 0, sizeof(double) * 6 * P);
  memset(o->cv, 0, sizeof(double) * o->nv * P);
  if (o->ns) memset(o->sv, 0, sizeof(double) * o->ns * P);
  if (o->c.problem_type == 1) {
    /* initialize_mixing_layer_with_info (Initialize.cu:259-326): the stream of each node's y */
    const int gz = o->dim == 3 ? o->g : o->g;
    for (int k = -gz; k < o->mz + gz; ++k)
      for (int j = -o->g; j < o->my + o->g; ++j)
        for (int i = -o->g; i < o->mx + o->g; ++i) {
          const long p = ID(o, i, j, k);
          const double yc = o->y[IC(o, i, j, k)];
          const double *st = yc >= 0 ? o->c.ml_upper : o->c.ml_lower;
          const double *ys = yc >= 0 ? o->c.ml_y_upper : o->c.ml_y_lower;
          for (int l = 0; l < 6; ++l) o->bv[l * P + p] = st[l];
          o->bv[P + p] = 0.5 * (o->c.ml_upper[1] + o->c.ml_lower[1]) +
                         0.5 * (o->c.ml_upper[1] - o->c.ml_lower[1]) * tanh(2 * yc / o->c.ml_delta_omega);
          for (int l = 0; l < o->ns; ++l) o->sv[l * P + p] = ys[l];
        }
  } else if (o->c.has_init) {
    for (int l = 0; l < 6; ++l)
      for (long p = 0; p < P; ++p) o->bv[l * P + p] = o->c.init_bv[l];
    for (int l = 0; l < o->ns; ++l)
      for (long p = 0; p < P; ++p) o->sv[l * P + p] = o->c.init_sv[l];
  }
  for (int l = 0; l < 6; ++l)
    for (int k = 0; k < o->mz; ++k)
      for (int j = 0; j < o->my; ++j)
        for (int i = 0; i < o->mx; ++i) o->bv[l * P + ID(o, i, j, k)] = bv[l * N + IQ(o, i, j, k)];
  for (int l = 0; l < o->ns && sv; ++l)
    for (int k = 0; k < o->mz; ++k)
      for (int j = 0; j < o->my; ++j)
        for (int i = 0; i < o->mx; ++i) o->sv[l * P + ID(o, i, j, k)] = sv[l * N + IQ(o, i, j, k)];
}

void orc_get_state(const orc_ctx *o, double *cv, double *bv, double *mul) {
  const long P = o->P, N = (long)o->mx * o->my * o->mz;
  for (int k = 0; k < o->mz; ++k)
    for (int j = 0; j < o->my; ++j)
      for (int i = 0; i < o->mx; ++i) {
        const long p = ID(o, i, j, k), q = IQ(o, i, j, k);
        if (cv) for (int l = 0; l < o->nv; ++l) cv[l * N + q] = o->cv[l * P + p];
        if (bv) for (int l = 0; l < 6; ++l) bv[l * N + q] = o->bv[l * P + p];
        if (mul) mul[q] = o->mul[p];
      }
}

void orc_get_metric(const orc_ctx *o, double *metric9, double *jac) {
  const long P = o->P, N = (long)o->mx * o->my * o->mz;
  for (int k = 0; k < o->mz; ++k)
    for (int j = 0; j < o->my; ++j)
      for (int i = 0; i < o->mx; ++i) {
        const long p = ID(o, i, j, k), q = IQ(o, i, j, k);
        if (metric9) for (int r = 0; r < 9; ++r) metric9[r * N + q] = o->met[r * P + p];
        if (jac) jac[q] = o->jac[p];
      }
}

void orc_get_mixture(const orc_ctx *o, double *sv, double *cond, double *rho_d, double *acoustic, double *gamma) {
  const long P = o->P, N = (long)o->mx * o->my * o->mz;
  for (int k = 0; k < o->mz; ++k)
    for (int j = 0; j < o->my; ++j)
      for (int i = 0; i < o->mx; ++i) {
        const long p = ID(o, i, j, k), q = IQ(o, i, j, k);
        for (int l = 0; l < o->ns; ++l) {
          if (sv) sv[l * N + q] = o->sv[l * P + p];
          if (rho_d) rho_d[l * N + q] = o->rhod[l * P + p];
        }
        if (cond) cond[q] = o->cond[p];
        if (acoustic) acoustic[q] = o->acs[p];
        if (gamma) gamma[q] = o->gam[p];
      }
}

void orc_rhs(orc_ctx *o, unsigned mask, double *dq) {
  const long N = (long)o->mx * o->my * o->mz;
  memset(o->dq, 0, sizeof(double) * o->nv * N);
  if ((mask & 4u) && o->ns && o->c.finite_rate && !o->c.chem_mode)
    for (int k = 0; k < o->mz; ++k)
      for (int j = 0; j < o->my; ++j)
        for (int i = 0; i < o->mx; ++i) chemistry_node(o, i, j, k);
  if (mask & 1u)
    for (int d = 0; d < o->dim; ++d) {
      const int is = o->c.inviscid_scheme;
      if (is == 71 || is == 72) fvs_direction(o, d);
      else if (o->c.reconstruction == 4 || o->c.reconstruction == 5) aweno_direction(o, d);
      else pv_direction(o, d);
    }
  if ((mask & 2u) && o->c.viscous_order != 0) viscous(o);
  if ((mask & 4u) && o->ns && o->c.finite_rate && o->c.chem_mode)
    for (int k = 0; k < o->mz; ++k)
      for (int j = 0; j < o->my; ++j)
        for (int i = 0; i < o->mx; ++i) chemistry_node_jac(o, i, j, k, 1);
  if (dq) memcpy(dq, o->dq, sizeof(double) * o->nv * N);
}

/* RK3<mixture model, Laminar> time loop body (RK.cuh:85-185) */
double orc_step(orc_ctx *o, int n) {
  double dt = o->c.fixed_time_step ? o->c.dt : 1e6;
  for (int s = 0; s < n; ++s) {
    memcpy(o->qn, o->cv, sizeof(double) * o->nv * o->P);
    for (int rk = 0; rk < 3; ++rk) {
      if (!o->c.fixed_time_step && rk == 0) dt = orc_dt(o);
      o->dt_cur = dt;
      orc_rhs(o, 7u, NULL);
      rk_update(o, dt, rk);
      fill_ghosts(o);
    }
    o->t += dt;
  }
  return dt;
}

/* ---------------------------------------------------------------- steady driver (SteadySim.cuh) */

/* compute_jacobian_times_dq (DPLUR.cuh:96-154): the split convective Jacobian of direction dir at
 * interior node (i, j, k), with eigenvalue shift lam, times that node's dq. */
static void jac_times_dq(const orc_ctx *o, const double *dqv, int i, int j, int k, int dir, double lam,
                         double *out) {
  const long P = o->P, N = (long)o->mx * o->my * o->mz;
  const long p = ID(o, i, j, k), q = IQ(o, i, j, k);
  const double xi_x = M(o, dir + 1, 1, p), xi_y = M(o, dir + 1, 2, p), xi_z = M(o, dir + 1, 3, p);
  const double u = o->bv[P + p], v = o->bv[2 * P + p], w = o->bv[3 * P + p];
  const double U = xi_x * u + xi_y * v + xi_z * w;
  const double lmd1 = U + lam;
  const double e = 0.5 * (u * u + v * v + w * w);
  double gamma = GAMMA_AIR, b3 = 0, b4 = 0, h = 0;
  double d[FVS_MAXV];
  for (int l = 0; l < o->nv; ++l) d[l] = dqv[l * N + q];
  if (!o->ns) {
    h = gamma / (gamma - 1) * o->bv[4 * P + p] / o->bv[p] + e;
  } else {
    const orc_chem *ch = o->c.chem;
    double hs[ORC_MAX_SPEC], cps[ORC_MAX_SPEC];
    const double t = o->bv[5 * P + p];
    mix_h_cp(ch, t, hs, cps);
    gamma = o->gam[p];
    for (int l = 0; l < o->ns; ++l) {
      b3 += R_U * t / ch->mw[l] * d[5 + l];
      b4 += hs[l] * d[5 + l];
      h += o->sv[l * P + p] * hs[l];
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
  for (int l = 0; l < o->ns; ++l) out[5 + l] = lmd1 * d[5 + l] + o->sv[l * P + p] * b1;
}

/* (diag I - dt J) x = b for the species of node q (EPI_for_dq0 / EPI_for_dqk / EPI, FiniteRateChem.cu:
 * 233-300), b solved in place */
static void epi_solve(const orc_ctx *o, long q, double diag, double dt, double *b) {
  const int ns = o->ns;
  double lhs[ORC_MAX_SPEC * ORC_MAX_SPEC];
  for (int m = 0; m < ns; ++m)
    for (int n = 0; n < ns; ++n) {
      const double jm = o->cj[(q * ns + m) * ns + n];
      lhs[m * ns + n] = m == n ? diag - dt * jm : -dt * jm;
    }
  lu_solve(lhs, b, ns);
}

/* DPLUR (DPLUR.cuh:282-322, DPLUR.cu:5-40) on o->dq of one block: compute_DQ_0, DPLUR_inner_step
 * inner iterations (walls' dq zeroed first, set_wall_dq_to_0), convert_dq_back_to_dqDt.  The viscous
 * spectral radius the reference adds to the diagonal is never computed there (its array keeps the
 * zeros of its allocation, Field.cu:553-565), so those terms are zero. */
static void dplur(orc_ctx *o, double diag_factor) {
  const long N = (long)o->mx * o->my * o->mz;
  const int nv = o->nv, ns = o->ns;
  const int fr = ns && o->c.finite_rate, csm = o->c.chem_src_method;
  for (int k = 0; k < o->mz; ++k)
    for (int j = 0; j < o->my; ++j)
      for (int i = 0; i < o->mx; ++i) {
        const long q = IQ(o, i, j, k);
        const double dt = o->dtl[q];
        for (int l = 0; l < nv; ++l) o->dq[l * N + q] *= dt;
        const double diag = 1 + diag_factor * dt + dt * (o->srad[3 * q] + o->srad[3 * q + 1] + o->srad[3 * q + 2]);
        if (!fr) {
          for (int l = 0; l < nv; ++l) o->dq[l * N + q] /= diag;
          continue;
        }
        for (int l = 0; l < 5; ++l) o->dq[l * N + q] /= diag;
        if (csm == 1) {
          double b[ORC_MAX_SPEC];
          for (int l = 0; l < ns; ++l) b[l] = o->dq[(5 + l) * N + q];
          epi_solve(o, q, diag, dt, b);
          for (int l = 0; l < ns; ++l) o->dq[(5 + l) * N + q] = b[l];
        } else if (csm == 2) {
          for (int l = 0; l < ns; ++l) o->dq[(5 + l) * N + q] /= diag - dt * o->cj[q * ns + l];
        } else {
          for (int l = 0; l < ns; ++l) o->dq[(5 + l) * N + q] /= diag;
        }
      }
  memcpy(o->dq0, o->dq, sizeof(double) * nv * N);
  for (int it = 0; it < o->c.dplur_inner; ++it) {
    for (int n = 0; n < o->nf; ++n) {
      const face_t *f = &o->f[n];
      if (f->type != ORC_WALL) continue;
      int lo[3] = {0, 0, 0}, hi[3] = {o->mx - 1, o->my - 1, o->mz - 1};
      const int fi = f->face, at = f->direction < 0 ? 0 : (fi == 0 ? o->mx - 1 : fi == 1 ? o->my - 1 : o->mz - 1);
      lo[fi] = hi[fi] = at;
      for (int k = lo[2]; k <= hi[2]; ++k)
        for (int j = lo[1]; j <= hi[1]; ++j)
          for (int i = lo[0]; i <= hi[0]; ++i)
            for (int l = 0; l < nv; ++l) o->dq[l * N + IQ(o, i, j, k)] = 0;
    }
    for (int k = 0; k < o->mz; ++k)
      for (int j = 0; j < o->my; ++j)
        for (int i = 0; i < o->mx; ++i) {
          const long q = IQ(o, i, j, k);
          double conv[FVS_MAXV], tot[FVS_MAXV];
          for (int l = 0; l < nv; ++l) tot[l] = 0;
          const int nb[3][3] = {{i - 1, j, k}, {i, j - 1, k}, {i, j, k - 1}};
          const int pb[3][3] = {{i + 1, j, k}, {i, j + 1, k}, {i, j, k + 1}};
          const int ext[3] = {o->mx, o->my, o->mz}, at[3] = {i, j, k};
          for (int d = 0; d < 3; ++d) {
            if (at[d] > 0) {
              const long qn = IQ(o, nb[d][0], nb[d][1], nb[d][2]);
              jac_times_dq(o, o->dq, nb[d][0], nb[d][1], nb[d][2], d, o->srad[3 * qn + d], conv);
              for (int l = 0; l < nv; ++l) tot[l] += 0.5 * conv[l];
            }
          }
          for (int d = 0; d < 3; ++d) {
            if (at[d] != ext[d] - 1) {
              const long qn = IQ(o, pb[d][0], pb[d][1], pb[d][2]);
              jac_times_dq(o, o->dq, pb[d][0], pb[d][1], pb[d][2], d, -o->srad[3 * qn + d], conv);
              for (int l = 0; l < nv; ++l) tot[l] -= 0.5 * conv[l];
            }
          }
          const double dt = o->dtl[q];
          const double diag = 1 + diag_factor * dt + dt * (o->srad[3 * q] + o->srad[3 * q + 1] + o->srad[3 * q + 2]);
          const int nflow = fr ? 5 : nv;
          for (int l = 0; l < nflow; ++l) o->dqk[l * N + q] = o->dq0[l * N + q] + dt * tot[l] / diag;
          if (!fr) continue;
          if (csm == 1) {
            double b[ORC_MAX_SPEC];
            for (int l = 0; l < ns; ++l) b[l] = tot[5 + l] * dt;
            epi_solve(o, q, diag, dt, b);
            for (int l = 0; l < ns; ++l) o->dqk[(5 + l) * N + q] = o->dq0[(5 + l) * N + q] + b[l];
          } else if (csm == 2) {
            for (int l = 0; l < ns; ++l)
              o->dqk[(5 + l) * N + q] = o->dq0[(5 + l) * N + q] + dt * tot[5 + l] / (diag - dt * o->cj[q * ns + l]);
          } else {
            for (int l = 0; l < ns; ++l) o->dqk[(5 + l) * N + q] = o->dq0[(5 + l) * N + q] + dt * tot[5 + l] / diag;
          }
        }
    memcpy(o->dq, o->dqk, sizeof(double) * nv * N);
  }
  for (long q = 0; q < N; ++q)
    for (int l = 0; l < nv; ++l) o->dq[l * N + q] /= o->dtl[q];
}

/* update_cv_and_bv (FieldOperation.cuh:189-232): cv += dt_local / jac * dq, then the primitive state */
static void steady_update(orc_ctx *o) {
  const long P = o->P, N = (long)o->mx * o->my * o->mz;
  for (int k = 0; k < o->mz; ++k)
    for (int j = 0; j < o->my; ++j)
      for (int i = 0; i < o->mx; ++i) {
        const long p = ID(o, i, j, k), q = IQ(o, i, j, k);
        const double dtj = o->dtl[q] / o->jac[p];
        for (int l = 0; l < o->nv; ++l) o->cv[l * P + p] += dtj * o->dq[l * N + q];
        if (o->mz == 1) o->cv[3 * P + p] = 0;
        o->bv[p] = o->cv[p];
        const double di = 1.0 / o->cv[p];
        o->bv[P + p] = o->cv[P + p] * di;
        o->bv[2 * P + p] = o->cv[2 * P + p] * di;
        o->bv[3 * P + p] = o->cv[3 * P + p] * di;
        if (o->ns) {
          for (int l = 0; l < o->ns; ++l) o->sv[l * P + p] = o->cv[(5 + l) * P + p] * di;
          mix_t_and_p(o, p, o->cv[4 * P + p]);
        } else {
          const double V2 = o->bv[P + p] * o->bv[P + p] + o->bv[2 * P + p] * o->bv[2 * P + p] +
                            o->bv[3 * P + p] * o->bv[3 * P + p];
          o->bv[4 * P + p] = (GAMMA_AIR - 1) * (o->cv[4 * P + p] - 0.5 * o->bv[p] * V2);
          o->bv[5 * P + p] = o->bv[4 * P + p] * MW_AIR * di / R_U;
        }
      }
}

/* dq of the steady and dual-time drivers: from zero, the chemical source first (with its Jacobian for
 * chemSrcMethod 1 / 2), then the inviscid and viscous fluxes (SteadySim.cuh:78-88) */
static void steady_rhs(orc_ctx *o) {
  const long N = (long)o->mx * o->my * o->mz;
  const int fr = o->ns && o->c.finite_rate, csm = o->c.chem_src_method;
  memset(o->dq, 0, sizeof(double) * o->nv * N);
  if (fr)
    for (int k = 0; k < o->mz; ++k)
      for (int j = 0; j < o->my; ++j)
        for (int i = 0; i < o->mx; ++i) chemistry_node_jac(o, i, j, k, csm == 1 ? 2 : csm == 2 ? 3 : 0);
  for (int d = 0; d < o->dim; ++d) {
    const int is = o->c.inviscid_scheme;
    if (is == 71 || is == 72) fvs_direction(o, d);
    else if (o->c.reconstruction == 4 || o->c.reconstruction == 5) aweno_direction(o, d);
    else pv_direction(o, d);
  }
  if (o->c.viscous_order != 0) viscous(o);
}

static void steady_buffers(orc_ctx *o, int dplur_needed) {
  const long N = (long)o->mx * o->my * o->mz;
  const int ns = o->ns, fr = ns && o->c.finite_rate, csm = o->c.chem_src_method;
  if (!o->srad) o->srad = (double *)calloc(3 * N, sizeof(double));
  if (fr && csm && !o->cj) o->cj = (double *)calloc(N * (csm == 1 ? ns * ns : ns), sizeof(double));
  if (dplur_needed && !o->dq0) {
    o->dq0 = (double *)calloc(o->nv * N, sizeof(double));
    o->dqk = (double *)calloc(o->nv * N, sizeof(double));
  }
}

/* steady_simulation<mixture model, Laminar> iteration body for one block (SteadySim.cuh:65-140): dq
 * from zero; the chemical source first (with its Jacobian for chemSrcMethod 1 / 2), the inviscid and
 * viscous fluxes; local_time_step; implicit_treatment (ImplicitTreatmentHPP.cuh:7-54: EPI or DA when
 * explicit, else DPLUR); update_cv_and_bv; boundary faces, 2-D k copy, properties.  The physical time
 * does not advance. */
void orc_steady(orc_ctx *o, int n) {
  const long N = (long)o->mx * o->my * o->mz;
  const int ns = o->ns, fr = ns && o->c.finite_rate, csm = o->c.chem_src_method;
  steady_buffers(o, o->c.implicit_method == 1);
  for (int s = 0; s < n; ++s) {
    steady_rhs(o);
    orc_dt(o);
    if (o->c.implicit_method == 1) {
      dplur(o, 0.0);
    } else if (fr && csm) {
      for (long q = 0; q < N; ++q) {
        const double dt = o->dtl[q];
        if (csm == 1) {
          double b[ORC_MAX_SPEC];
          for (int l = 0; l < ns; ++l) b[l] = o->dq[(5 + l) * N + q];
          epi_solve(o, q, 1.0, dt, b);
          for (int l = 0; l < ns; ++l) o->dq[(5 + l) * N + q] = b[l];
        } else {
          for (int l = 0; l < ns; ++l) o->dq[(5 + l) * N + q] /= 1 - dt * o->cj[q * ns + l];
        }
      }
    }
    steady_update(o);
    fill_ghosts(o);
  }
}

/* (rho, |V|, p, T) of every interior node (store_last_iter, DualTimeStepping.cu:154-167) */
static void store_last_iter(orc_ctx *o) {
  const long P = o->P;
  for (int k = 0; k < o->mz; ++k)
    for (int j = 0; j < o->my; ++j)
      for (int i = 0; i < o->mx; ++i) {
        const long p = ID(o, i, j, k), q = IQ(o, i, j, k);
        o->inlast[4 * q] = o->bv[p];
        o->inlast[4 * q + 1] = sqrt(o->bv[P + p] * o->bv[P + p] + o->bv[2 * P + p] * o->bv[2 * P + p] +
                                    o->bv[3 * P + p] * o->bv[3 * P + p]);
        o->inlast[4 * q + 2] = o->bv[4 * P + p];
        o->inlast[4 * q + 3] = o->bv[5 * P + p];
      }
}

/* inner_converged (DualTimeStepping.cu:32-135): RMS change since store_last_iter, scaled by that of the
 * first inner iteration; adapts the inner-iteration count; returns 1 when the inner loop stops */
static int inner_converged(orc_ctx *o, int iter) {
  const long P = o->P, N = (long)o->mx * o->my * o->mz;
  double res[4] = {0, 0, 0, 0};
  for (int k = 0; k < o->mz; ++k)
    for (int j = 0; j < o->my; ++j)
      for (int i = 0; i < o->mx; ++i) {
        const long p = ID(o, i, j, k), q = IQ(o, i, j, k);
        const double vel = sqrt(o->bv[P + p] * o->bv[P + p] + o->bv[2 * P + p] * o->bv[2 * P + p] +
                                o->bv[3 * P + p] * o->bv[3 * P + p]);
        const double d[4] = {o->bv[p] - o->inlast[4 * q], vel - o->inlast[4 * q + 1],
                             o->bv[4 * P + p] - o->inlast[4 * q + 2], o->bv[5 * P + p] - o->inlast[4 * q + 3]};
        for (int l = 0; l < 4; ++l) res[l] += d[l] * d[l];
      }
  for (int l = 0; l < 4; ++l) res[l] = sqrt(res[l] / N);
  if (iter == 1)
    for (int l = 0; l < 4; ++l) o->res_scale_inner[l] = res[l] < 1e-20 ? 1e-20 : res[l];
  double err = res[0] / o->res_scale_inner[0];
  for (int l = 1; l < 4; ++l)
    if (res[l] / o->res_scale_inner[l] > err) err = res[l] / o->res_scale_inner[l];
  if (iter == o->inner && err > 1e-3 && o->inner < o->c.max_inner_iteration) {
    o->inner += 5;
    if (o->inner > o->c.max_inner_iteration) o->inner = o->c.max_inner_iteration;
  }
  if (err < 1e-3) {
    if (o->inner - iter > 0) o->inner = iter;
    return 1;
  }
  return 0;
}

/* dual_time_stepping<mixture model, Laminar> (DualTimeStepping.cuh:32-252) for one block: per physical
 * step q* = jac / (2 dt) (4 cv - cv_prev) (compute_qn_star, DualTimeStepping.cu:3-14), then up to
 * `inner` pseudo-time iterations: dq, local time steps, dq += q* - 1.5 jac / dt cv (compute_modified_rhs,
 * :16-30), DPLUR with diag_factor 1.5 / dt, update_cv_and_bv, boundary faces, k copy, properties; every
 * iteration_adjust_step-th step the inner loop is monitored and its count adapted. */
int orc_dual(orc_ctx *o, int n) {
  const long P = o->P, N = (long)o->mx * o->my * o->mz;
  const int nv = o->nv;
  const double dt = o->c.dt, diag_factor = 1.5 / dt;
  steady_buffers(o, 1);
  if (!o->qn1) {
    o->qn1 = (double *)calloc((size_t)nv * P, sizeof(double));
    o->qstar = (double *)calloc((size_t)nv * N, sizeof(double));
    o->inlast = (double *)calloc(4 * N, sizeof(double));
  }
  if (!o->dual_init) {
    memcpy(o->qn1, o->cv, sizeof(double) * nv * P);
    o->inner = o->c.inner_iteration;
    o->dual_init = 1;
  }
  for (int s = 0; s < n; ++s) {
    const int step = ++o->dual_step;
    for (int k = 0; k < o->mz; ++k)
      for (int j = 0; j < o->my; ++j)
        for (int i = 0; i < o->mx; ++i) {
          const long p = ID(o, i, j, k), q = IQ(o, i, j, k);
          const double factor = 0.5 * o->jac[p] / dt;
          for (int l = 0; l < nv; ++l) o->qstar[l * N + q] = factor * (4 * o->cv[l * P + p] - o->qn1[l * P + p]);
        }
    memcpy(o->qn1, o->cv, sizeof(double) * nv * P);
    const int monitor = step % o->c.iteration_adjust_step == 0;
    for (int iter = 1; iter <= o->inner; ++iter) {
      if (monitor) store_last_iter(o);
      steady_rhs(o);
      orc_dt(o);
      for (int k = 0; k < o->mz; ++k)
        for (int j = 0; j < o->my; ++j)
          for (int i = 0; i < o->mx; ++i) {
            const long p = ID(o, i, j, k), q = IQ(o, i, j, k);
            const double factor = 1.5 * o->jac[p] / dt;
            for (int l = 0; l < nv; ++l) o->dq[l * N + q] += o->qstar[l * N + q] - factor * o->cv[l * P + p];
          }
      dplur(o, diag_factor);
      steady_update(o);
      fill_ghosts(o);
      if (monitor && inner_converged(o, iter)) break;
    }
    o->t += dt;
  }
  return o->inner;
}

/* ---------------------------------------------------------------- single-point statistics */

/* collect_single_point_basic_statistics (SinglePointStat.cu:641-706): one collection added to acc,
 * laid out as four groups [n_var][mz+2][my+2][mx+2] back to back (Reynolds 1st: rho, p, extras by
 * primitive index; Favre 1st: rho u, rho v, rho w, rho T, rho Y_k; Reynolds 2nd: rho rho, p p
 * [, rho p]; Favre 2nd: rho u u, rho v v, rho w w, rho u v, rho u w, rho v w, rho T T, rho Y_k Y_k).
 * Nodes i = -1..mx, j = -1..my, k = -1..mz, read from the ghost layers as they stand after the
 * step (2-D blocks: the k layers eliminate_k copied from k = 0). */
void orc_stat_collect(const orc_ctx *o, int n_rey, const int *rey_idx, int rho_p, double *acc) {
  const long P = o->P;
  const int nx = o->mx + 2, ny = o->my + 2, nz = o->mz + 2;
  const long np = (long)nx * ny * nz;
  double *rey1 = acc, *fav1 = rey1 + (2 + n_rey) * np, *rey2 = fav1 + (4 + o->ns) * np;
  double *fav2 = rey2 + (2 + rho_p) * np;
  for (int k = -1; k <= o->mz; ++k)
    for (int j = -1; j <= o->my; ++j)
      for (int i = -1; i <= o->mx; ++i) {
        const long n = (((long)(k + 1) * ny) + (j + 1)) * nx + (i + 1);
        const long p = ID(o, i, j, k);
        const double rho = o->bv[p], u = o->bv[P + p], v = o->bv[2 * P + p], w = o->bv[3 * P + p];
        const double pr = o->bv[4 * P + p], T = o->bv[5 * P + p];
        rey1[n] += rho;
        rey1[np + n] += pr;
        for (int l = 0; l < n_rey; ++l) rey1[(2 + l) * np + n] += o->bv[rey_idx[l] * P + p];
        fav1[n] += rho * u;
        fav1[np + n] += rho * v;
        fav1[2 * np + n] += rho * w;
        fav1[3 * np + n] += rho * T;
        for (int l = 0; l < o->ns; ++l) fav1[(4 + l) * np + n] += rho * o->sv[l * P + p];
        rey2[n] += rho * rho;
        rey2[np + n] += pr * pr;
        if (rho_p) rey2[2 * np + n] += rho * pr;
        fav2[n] += rho * u * u;
        fav2[np + n] += rho * v * v;
        fav2[2 * np + n] += rho * w * w;
        fav2[3 * np + n] += rho * u * v;
        fav2[4 * np + n] += rho * u * w;
        fav2[5 * np + n] += rho * v * w;
        fav2[6 * np + n] += rho * T * T;
        for (int l = 0; l < o->ns; ++l) fav2[(7 + l) * np + n] += rho * o->sv[l * P + p] * o->sv[l * P + p];
      }
}

/* collect_single_point_additional_statistics (SinglePointStat.cu:707-722) on the interior nodes:
 * collect_tke_budget (TkeBudget.cu:123-170) into tke[7][N] when tke != 0, and for the species
 * ss_idx[0..nss) collect_species_velocity_correlation into svc[3 nss][N] and
 * collect_species_dissipation_rate into sdr[5 nss][N] (SpeciesStat.cu:5-85); null arrays are skipped.
 * Gradients as the reference forms them: half the central differences in computational space times
 * the metric (in 2-D the k ghost layers are copies of k = 0, so their difference is zero). */
static double stat_grad(const orc_ctx *o, const double *f, int i, int j, int k, int c) {
  const long p = ID(o, i, j, k);
  const double di = f[ID(o, i + 1, j, k)] - f[ID(o, i - 1, j, k)];
  const double dj = f[ID(o, i, j + 1, k)] - f[ID(o, i, j - 1, k)];
  if (o->dim == 2) return 0.5 * (M(o, 1, c, p) * di + M(o, 2, c, p) * dj);
  const double dk = f[ID(o, i, j, k + 1)] - f[ID(o, i, j, k - 1)];
  return 0.5 * (M(o, 1, c, p) * di + M(o, 2, c, p) * dj + M(o, 3, c, p) * dk);
}

void orc_stat_extra(const orc_ctx *o, double *tke, int nss, const int *ss_idx, double *svc, double *sdr) {
  const long P = o->P, N = (long)o->mx * o->my * o->mz;
  for (int k = 0; k < o->mz; ++k)
    for (int j = 0; j < o->my; ++j)
      for (int i = 0; i < o->mx; ++i) {
        const long n = IQ(o, i, j, k), p = ID(o, i, j, k);
        if (tke) {
          double gu[3], gv[3], gw[3];
          for (int c = 0; c < 3; ++c) {
            gu[c] = stat_grad(o, o->bv + P, i, j, k, c + 1);
            gv[c] = stat_grad(o, o->bv + 2 * P, i, j, k, c + 1);
            gw[c] = stat_grad(o, o->bv + 3 * P, i, j, k, c + 1);
          }
          const double mu = o->mul[p];
          const double t11 = mu * (4.0 * gu[0] - 2 * gv[1] - 2 * gw[2]) / 3.0;
          const double t12 = mu * (gu[1] + gv[0]);
          const double t13 = mu * (gu[2] + gw[0]);
          const double t22 = mu * (4.0 * gv[1] - 2 * gu[0] - 2 * gw[2]) / 3.0;
          const double t23 = mu * (gv[2] + gw[1]);
          const double t33 = mu * (4.0 * gw[2] - 2 * gu[0] - 2 * gv[1]) / 3.0;
          tke[n] += t11;
          tke[N + n] += t12;
          tke[2 * N + n] += t13;
          tke[3 * N + n] += t22;
          tke[4 * N + n] += t23;
          tke[5 * N + n] += t33;
          tke[6 * N + n] += t11 * gu[0] + t12 * gu[1] + t13 * gu[2] + t12 * gv[0] + t22 * gv[1] + t23 * gv[2] +
                            t13 * gw[0] + t23 * gw[1] + t33 * gw[2];
        }
        for (int q = 0; q < nss; ++q) {
          const int is = ss_idx[q];
          if (svc) {
            const double rho = o->bv[p], u = o->bv[P + p], v = o->bv[2 * P + p], w = o->bv[3 * P + p];
            const double z = o->sv[is * P + p];
            svc[(3 * q) * N + n] += rho * u * z;
            svc[(3 * q + 1) * N + n] += rho * v * z;
            svc[(3 * q + 2) * N + n] += rho * w * z;
          }
          if (sdr) {
            const double zx = stat_grad(o, o->sv + is * P, i, j, k, 1), zy = stat_grad(o, o->sv + is * P, i, j, k, 2),
                         zz = stat_grad(o, o->sv + is * P, i, j, k, 3);
            const double rd = o->rhod[is * P + p];
            sdr[(5 * q) * N + n] += rd * (zx * zx + zy * zy + zz * zz);
            sdr[(5 * q + 1) * N + n] += rd * zx;
            sdr[(5 * q + 2) * N + n] += rd * zy;
            sdr[(5 * q + 3) * N + n] += rd * zz;
            sdr[(5 * q + 4) * N + n] += rd;
          }
        }
      }
}

/* ---------------------------------------------------------------- multi-block (interfaces) */

typedef struct {
  int rs[3], re[3], ts[3], te[3];
  int face, direction, target_face, target_direction;
  int src_tar[3], loop_dir[3], target_loop_dir[3], n_point[3];
  int target;
} inner_t;

struct orc_multi {
  int nb;
  orc_ctx **b;
  int *nf;
  inner_t **f;
};

static int isgn(int a) { return a < 0 ? -1 : 1; } /* gxl::sgn, sgn(0) = +1 (gxl_lib/Math.hpp:13-15) */

/* InnerFace::register_boundary (Mesh.cpp:38-141) */
static void register_inner(inner_t *f, int ngg, int dim) {
  f->direction = f->target_direction = 1;
  f->face = f->target_face = 0;
  for (int i = 0; i < 3; ++i) f->src_tar[i] = 0;
  for (int i = 0; i < dim; ++i)
    if (f->rs[i] == f->re[i]) {
      f->face = i;
      if (f->rs[i] == 1) f->direction = -1;
      f->rs[i] -= 1;
      f->re[i] -= 1;
      break;
    }
  for (int i = 0; i < dim; ++i)
    if (f->ts[i] == f->te[i]) {
      f->target_face = i;
      if (f->ts[i] == 1) f->target_direction = -1;
      f->ts[i] -= 1;
      f->te[i] -= 1;
      break;
    }
  f->src_tar[f->target_face] = -(f->direction * f->target_direction) * (f->face + 1);
  if (dim == 2) {
    const int nf = 1 - f->face, tnf = 1 - f->target_face;
    f->rs[nf] = abs(f->rs[nf]) - 1;
    f->re[nf] = abs(f->re[nf]) - 1;
    f->ts[tnf] = abs(f->ts[tnf]) - 1;
    f->te[tnf] = abs(f->te[tnf]) - 1;
    f->src_tar[tnf] = isgn((f->te[tnf] - f->ts[tnf]) * (f->re[nf] - f->rs[nf])) * (nf + 1);
    f->src_tar[2] = 3;
    f->rs[2] = f->re[2] = f->ts[2] = f->te[2] = 0;
  } else {
    int nf = 0, tnf = 0;
    for (int i = 0; i < dim; ++i)
      if (f->rs[i] < 0) {
        nf = i;
        f->rs[i] = -f->rs[i] - 1;
        f->re[i] = -f->re[i] - 1;
        break;
      }
    for (int i = 0; i < dim; ++i)
      if (f->ts[i] < 0) {
        tnf = i;
        f->ts[i] = -f->ts[i] - 1;
        f->te[i] = -f->te[i] - 1;
        break;
      }
    f->src_tar[tnf] = isgn((f->te[tnf] - f->ts[tnf]) * (f->re[nf] - f->rs[nf])) * (nf + 1);
    nf = 3 - f->face - nf;
    tnf = 3 - f->target_face - tnf;
    f->rs[nf] -= 1;
    f->re[nf] -= 1;
    f->ts[tnf] -= 1;
    f->te[tnf] -= 1;
    f->src_tar[tnf] = isgn((f->te[tnf] - f->ts[tnf]) * (f->re[nf] - f->rs[nf])) * (nf + 1);
  }
  f->rs[f->face] = f->direction < 0 ? -ngg : f->re[f->face];
  f->re[f->face] = f->direction < 0 ? 0 : f->re[f->face] + ngg;
  const int st = isgn(f->src_tar[f->target_face]);
  if (f->target_direction > 0) f->ts[f->target_face] = st > 0 ? f->te[f->target_face] - ngg : f->te[f->target_face];
  else f->ts[f->target_face] = st > 0 ? 0 : ngg;
  for (int i = 0; i < 3; ++i) {
    f->loop_dir[i] = f->rs[i] <= f->re[i] ? 1 : -1;
    f->target_loop_dir[i] = isgn(f->src_tar[i]);
    f->src_tar[i] = abs(f->src_tar[i]) - 1;
    f->n_point[i] = abs(f->rs[i] - f->re[i]) + 1;
  }
}

/* Mesh::init_inner_ghost_grid (Mesh.cpp:1049-1097) */
static void inner_ghost_grid(orc_multi *m) {
  for (int bb = 0; bb < m->nb; ++bb) {
    orc_ctx *B = m->b[bb];
    for (int n = 0; n < m->nf[bb]; ++n) {
      const inner_t *fc = &m->f[bb][n];
      orc_ctx *T = m->b[fc->target];
      int mn[3] = {fc->rs[0], fc->rs[1], fc->rs[2]}, mx[3] = {fc->re[0], fc->re[1], fc->re[2]};
      int mt[3] = {fc->ts[0], fc->ts[1], fc->ts[2]};
      const int sh = fc->direction < 0 ? -1 : 1;
      mn[fc->face] += sh;
      mx[fc->face] += sh;
      mt[fc->target_face] += fc->target_direction > 0 ? -1 : 1;
      int di[3];
      for (int i1 = mn[0]; fc->loop_dir[0] * (i1 - mx[0]) != 1; i1 += fc->loop_dir[0]) {
        di[0] = i1 - mn[0];
        for (int j1 = mn[1]; fc->loop_dir[1] * (j1 - mx[1]) != 1; j1 += fc->loop_dir[1]) {
          di[1] = j1 - mn[1];
          for (int k1 = mn[2]; fc->loop_dir[2] * (k1 - mx[2]) != 1; k1 += fc->loop_dir[2]) {
            di[2] = k1 - mn[2];
            const int i2 = mt[0] + fc->target_loop_dir[0] * di[fc->src_tar[0]];
            const int j2 = mt[1] + fc->target_loop_dir[1] * di[fc->src_tar[1]];
            const int k2 = mt[2] + fc->target_loop_dir[2] * di[fc->src_tar[2]];
            B->x[IC(B, i1, j1, k1)] = T->x[IC(T, i2, j2, k2)];
            B->y[IC(B, i1, j1, k1)] = T->y[IC(T, i2, j2, k2)];
            B->z[IC(B, i1, j1, k1)] = T->z[IC(T, i2, j2, k2)];
          }
        }
      }
    }
  }
}

/* data_communication / inner_communication (DataCommunication.cuh:29-105) */
static void exchange(orc_multi *m) {
  for (int bb = 0; bb < m->nb; ++bb) {
    orc_ctx *o = m->b[bb];
    for (int n = 0; n < m->nf[bb]; ++n) {
      const inner_t *f = &m->f[bb][n];
      orc_ctx *t = m->b[f->target];
      const int face_dir = f->direction > 0 ? f->rs[f->face] : f->re[f->face];
      for (int n2 = 0; n2 < f->n_point[2]; ++n2)
        for (int n1 = 0; n1 < f->n_point[1]; ++n1)
          for (int n0 = 0; n0 < f->n_point[0]; ++n0) {
            const int d[3] = {f->loop_dir[0] * n0, f->loop_dir[1] * n1, f->loop_dir[2] * n2};
            const int idx[3] = {f->rs[0] + d[0], f->rs[1] + d[1], f->rs[2] + d[2]};
            int it[3];
            for (int q = 0; q < 3; ++q) it[q] = f->ts[q] + f->target_loop_dir[q] * d[f->src_tar[q]];
            const long p = ID(o, idx[0], idx[1], idx[2]), pt = ID(t, it[0], it[1], it[2]);
            if (idx[f->face] == face_dir) {
              for (int l = 0; l < 6; ++l) {
                const double ave = 0.5 * (t->bv[l * t->P + pt] + o->bv[l * o->P + p]);
                o->bv[l * o->P + p] = ave;
                t->bv[l * t->P + pt] = ave;
              }
              for (int l = 0; l < o->ns; ++l) {
                const double ave = 0.5 * (t->sv[l * t->P + pt] + o->sv[l * o->P + p]);
                o->sv[l * o->P + p] = ave;
                t->sv[l * t->P + pt] = ave;
              }
            } else {
              for (int l = 0; l < 6; ++l) o->bv[l * o->P + p] = t->bv[l * t->P + pt];
              for (int l = 0; l < o->ns; ++l) o->sv[l * o->P + p] = t->sv[l * t->P + pt];
            }
            cv_from_bv(o, p);
          }
    }
  }
}

orc_multi *orc_multi_create(int nb, const orc_case *cases, const double *const *x, const double *const *y,
                            const double *const *z, const int *n_inner, const orc_inner_in *inner) {
  orc_multi *m = (orc_multi *)calloc(1, sizeof(orc_multi));
  m->nb = nb;
  m->b = (orc_ctx **)calloc(nb, sizeof(orc_ctx *));
  m->nf = (int *)calloc(nb, sizeof(int));
  m->f = (inner_t **)calloc(nb, sizeof(inner_t *));
  for (int b = 0; b < nb; ++b) m->b[b] = create_block(&cases[b], x[b], y[b], z[b], 0);
  int off = 0;
  for (int b = 0; b < nb; ++b) {
    m->nf[b] = n_inner[b];
    m->f[b] = (inner_t *)calloc(n_inner[b] + 1, sizeof(inner_t));
    for (int n = 0; n < n_inner[b]; ++n) {
      const orc_inner_in *in = &inner[off++];
      inner_t *f = &m->f[b][n];
      for (int q = 0; q < 3; ++q) {
        f->rs[q] = in->raw[2 * q];
        f->re[q] = in->raw[2 * q + 1];
        f->ts[q] = in->traw[2 * q];
        f->te[q] = in->traw[2 * q + 1];
      }
      f->target = in->traw[6] - 1;
      register_inner(f, m->b[b]->g, m->b[b]->dim);
    }
  }
  inner_ghost_grid(m);
  for (int b = 0; b < nb; ++b) {
    ghost_grid_edges(m->b[b]);
    compute_metric(m->b[b]);
  }
  return m;
}

void orc_multi_destroy(orc_multi *m) {
  if (!m) return;
  for (int b = 0; b < m->nb; ++b) {
    orc_destroy(m->b[b]);
    free(m->f[b]);
  }
  free(m->b);
  free(m->f);
  free(m->nf);
  free(m);
}

orc_ctx *orc_multi_block(orc_multi *m, int b) { return m->b[b]; }

/* Driver::initialize_computation (Driver.cu:115-199) over all blocks, then cv <- bv (RK.cuh:37-45) */
void orc_multi_set_state(orc_multi *m, const double *const *bv, const double *const *sv) {
  for (int b = 0; b < m->nb; ++b) {
    load_state(m->b[b], bv[b], sv ? sv[b] : NULL);
    if (m->b[b]->dim == 2) eliminate_k(m->b[b]);
  }
  for (int b = 0; b < m->nb; ++b) apply_bcs(m->b[b]);
  exchange(m);
  for (int b = 0; b < m->nb; ++b) {
    properties(m->b[b]);
    for (long p = 0; p < m->b[b]->P; ++p) cv_from_bv(m->b[b], p);
    m->b[b]->t = 0;
  }
}

/* RK3 over all blocks (RK.cuh:85-185): one dt (minimum over the blocks), per stage every block's RHS,
 * update and boundary faces, then the interfaces, then the k copies (2-D) and the properties. */
double orc_multi_step(orc_multi *m, int n) {
  double dt = m->b[0]->c.fixed_time_step ? m->b[0]->c.dt : 1e6;
  for (int s = 0; s < n; ++s) {
    for (int b = 0; b < m->nb; ++b) memcpy(m->b[b]->qn, m->b[b]->cv, sizeof(double) * m->b[b]->nv * m->b[b]->P);
    for (int rk = 0; rk < 3; ++rk) {
      if (!m->b[0]->c.fixed_time_step && rk == 0) {
        dt = 1e6;
        for (int b = 0; b < m->nb; ++b) {
          const double d = orc_dt(m->b[b]);
          if (d < dt) dt = d;
        }
      }
      for (int b = 0; b < m->nb; ++b) {
        m->b[b]->dt_cur = dt;
        orc_rhs(m->b[b], 7u, NULL);
        rk_update(m->b[b], dt, rk);
        apply_bcs(m->b[b]);
      }
      exchange(m);
      for (int b = 0; b < m->nb; ++b) {
        if (m->b[b]->dim == 2) eliminate_k(m->b[b]);
        properties(m->b[b]);
      }
    }
    for (int b = 0; b < m->nb; ++b) m->b[b]->t += dt;
  }
  return dt;
}
