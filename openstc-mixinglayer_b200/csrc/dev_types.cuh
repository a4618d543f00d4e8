// dev_types.cuh -- device-side views of a block (DevBlock: extents, padded layout, metric), of a
// state slot (DevState), of a boundary face (DevFace), of an interface (DevInner) and the fill
// values of the initial state.
// Part of the ostc_b200.cu translation unit (included in order; not a standalone header).
#pragma once

namespace ostc {

// Bounds-checked build (-DOSTC_BOUNDS_CHECK, libostc_b200_checked.so; the sanitizer is not
// available): every padded-plane index id() and interior index iq() is checked against the block's
// extents; an index outside them sets bit 1 (padded) or 2 (interior) of this flag and is clamped into
// range, so the access stays inside the arrays.  ostc_bounds_flags reads and clears it.
__device__ unsigned g_ostc_bounds = 0;

struct DevBlock {
  int mx, my, mz, g, gz, pitch, sy, sz;
  long long plane, off0, n;
  const double *met, *jac;
  // air: FP32 copies of the 9 metric planes and the Jacobian (plane 9), read by the mixed-precision
  // viscous sweep (the values it would round from met / jac); null for mixtures
  const float *met32;
  __host__ __device__ __forceinline__ long long id(int i, int j, int k) const {
#if defined(OSTC_BOUNDS_CHECK) && defined(__CUDA_ARCH__)
    if (i < -g || i >= pitch - g || j < -g || j >= sy - g || k < -gz || k >= sz - gz) {
      atomicOr(&g_ostc_bounds, 1u);
      i = min(max(i, -g), pitch - g - 1);
      j = min(max(j, -g), sy - g - 1);
      k = min(max(k, -gz), sz - gz - 1);
    }
#endif
    return off0 + ((long long)k * sy + j) * pitch + i;
  }
  // A padded-plane index formed from an accessor's index plus neighbour strides (stencil offsets,
  // ghost layers): checked in the bounds-checked build against the plane (bit 4, clamped), passed
  // through otherwise.
  __host__ __device__ __forceinline__ long long chk(long long p) const {
#if defined(OSTC_BOUNDS_CHECK) && defined(__CUDA_ARCH__)
    if (p < 0 || p >= plane) {
      atomicOr(&g_ostc_bounds, 4u);
      p = p < 0 ? 0 : plane - 1;
    }
#endif
    return p;
  }
  __host__ __device__ __forceinline__ long long iq(int i, int j, int k) const {
#if defined(OSTC_BOUNDS_CHECK) && defined(__CUDA_ARCH__)
    if (i < 0 || i >= mx || j < 0 || j >= my || k < 0 || k >= mz) {
      atomicOr(&g_ostc_bounds, 2u);
      i = min(max(i, 0), mx - 1);
      j = min(max(j, 0), my - 1);
      k = min(max(k, 0), mz - 1);
    }
#endif
    return ((long long)k * my + j) * mx + i;
  }
};

struct DevState {
  double *cv, *bv, *mul;
  // mixtures (null on the air path): mass fractions, conductivity, rho*D_k, gamma, acoustic speed
  double *sv = nullptr, *cond = nullptr, *rhod = nullptr, *gam = nullptr, *acs = nullptr;
};

struct DevFace {
  int type, face, direction, rs[3], re[3];
  double density, u, v, w, pressure, temperature, acoustic_speed, gamma, entropy, mw;
  int wall_adiabatic;  // walls: 1 adiabatic, 0 isothermal at `temperature`
  double y[16];        // inflow mass fractions (mixtures)
  // inflows: 0 constant / 2 mixing-layer profile (upper stream above, `lower` below, blended in u by
  // tanh(2 y / delta_omega)); fluct 1 adds white noise of relative intensity fluct_rms, drawn from
  // rng[] at the face node's index in a plane of rng_row nodes per row (apply_inflow's indexing)
  int inflow_type, fluct, rng_row;
  double fluct_rms, velocity, delta_omega;
  double lower[6], y_lower[16];
  const double *ycoord;  // mixing-layer inflow: y of every face node, in the kernel's enumeration
  curandState *rng;
};

struct FillVals {
  double val[16];
};

// One block interface (InnerFace after register_boundary, Mesh.cpp:38-141).
struct DevInner {
  int rs[3], ts[3], loop_dir[3], target_loop_dir[3], src_tar[3], n_point[3];
  int face, direction, face_index;  // face_index: the coincident node layer along `face`
};

__device__ __forceinline__ void cv_from_bv_node(const DevBlock &b, DevState s, long long p) {
  // compute_cv_from_bv_1_point + compute_total_energy<Air> (FieldOperation.cuh:17-38,78-105)
  const long long P = b.plane;
  const double rho = s.bv[p], u = s.bv[P + p], v = s.bv[2 * P + p], w = s.bv[3 * P + p];
  s.cv[p] = rho;
  s.cv[P + p] = rho * u;
  s.cv[2 * P + p] = rho * v;
  s.cv[3 * P + p] = rho * w;
  const double V2 = u * u + v * v + w * w;
  double te = 0.5 * V2;
  te *= rho;
  te += s.bv[4 * P + p] / (kGamma - 1);
  s.cv[4 * P + p] = te;
}

}  // namespace ostc
