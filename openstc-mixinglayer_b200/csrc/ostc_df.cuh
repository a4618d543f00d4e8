// ostc_df.cuh -- the digital-filter turbulent inflow of a mixing-layer problem (fluctuation_type 11 on
// the inflow struct, problem_type 1): DBoundCond::initialize_digital_filter and the per-application
// pipeline generate_random_numbers -> apply_convolution -> compute_fluctuations -> apply_inflow_df
// (DigitalFilter.cu:8-678, BoundCond.cuh:614-754, called in the inflow slot of the boundary order,
// BoundCond.cuh:1555-1573).
//
// The face is the i = 0 plane of its block, ghost-padded by ngg in j and k (the reference supports no
// other face).  Per face plane node (j, k) and velocity component c the filter keeps
//   r      normal draws over the plane padded by DF_N + ngg (one curand state per node and component),
//          spanwise mean removed and rms normalised over k = 0..mz-1, then extended periodically in k;
//   fy     the y convolution of r with the per-j coefficients by (j in [-ngg, my+ngg), k padded);
//   new    the z convolution of fy with bz;
//   old    the time-correlated field (Castro's exponential correlation with time scale delta_omega / u);
//   fluc   the Lund transform of it (Cholesky factor of a Gaussian Reynolds-stress profile in y).
// Arrays are [c][k][j] with j fastest, each dimension padded as stated.
#pragma once

namespace ostc {

constexpr int kDfN = 50;  // DBoundCond::DF_N (BoundCond.cuh:80): filter half width

struct DevDf {
  int my, mz, g;          // block extents and ghost layers
  int wy, wz;             // r / rng plane: my + 2 (N + g), mz + 2 (N + g)
  int py, pz;             // face plane with ghosts: my + 2 g, mz + 2 g
  curandState *rng;       // [3][wz][wy]
  double *r;              // [3][wz][wy]
  double *fy;             // [3][wz][py]   (k padded by N + g, j by g)
  double *vnew, *vold;    // [3][pz][py]
  double *fluc;           // [3][pz][py]
  double *lund;           // [6][py]
  double *by, *bz;        // [2N+1][py]
  const double *yface;    // y of the face plane nodes (i = 0), [pz][py]
  double delta_u;         // |u_upper - u_lower| (write_reference_state's DeltaU)
};

__device__ __forceinline__ long long df_w(const DevDf &d, int j, int k, int c) {
  return ((long long)c * d.wz + (k + kDfN + d.g)) * d.wy + (j + kDfN + d.g);
}
__device__ __forceinline__ long long df_f(const DevDf &d, int j, int k, int c) {
  return ((long long)c * d.wz + (k + kDfN + d.g)) * d.py + (j + d.g);
}
__device__ __forceinline__ long long df_p(const DevDf &d, int j, int k, int c) {
  return ((long long)c * d.pz + (k + d.g)) * d.py + (j + d.g);
}

// initialize_rng on the DF states (DigitalFilter.cu:230-236): state f of the reference's
// VectorField2D<curandState>(my, mz, 3, N + ngg) - flat index f = (k + G) (my + 2G) + (j + G) + c sz -
// is seeded with seed + f, subsequence f.  Our [c][k][j] layout with the same padding has the same flat
// index, so state f here is state f there.
__global__ void k_df_rng_init(curandState *st, long long n, unsigned long long seed) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    curand_init(seed + (unsigned long long)i, (unsigned long long)i, 0, &st[i]);
}

// compute_lundMat_with_assumed_gaussian_reynolds_stress (DigitalFilter.cu:409-439): Cholesky factor of
// R_ij(y) = peak_ij exp(-2 y^2), y scaled by delta_omega; ysc[j + g].
__global__ void k_df_lund(DevDf d, const double *__restrict__ ysc, double r11, double r12, double r22, double r13,
                          double r23, double r33) {
  const int j = (int)(blockIdx.x * blockDim.x + threadIdx.x) - d.g;
  if (j >= d.my + d.g) return;
  const double y = ysc[j + d.g];
  const double gy = exp(-y * y * 0.5 * 4);
  const double R11 = r11 * gy, R12 = r12 * gy, R22 = r22 * gy, R13 = r13 * gy, R23 = r23 * gy, R33 = r33 * gy;
  double *m = d.lund;
  const int q = j + d.g, P = d.py;
  m[q] = sqrt(fabs(R11));
  m[P + q] = m[q] < 1e-40 ? 0 : R12 / m[q];
  m[2 * P + q] = sqrt(fabs(R22 - m[P + q] * m[P + q]));
  m[3 * P + q] = m[q] < 1e-40 ? 0 : R13 / m[q];
  m[4 * P + q] = m[2 * P + q] < 1e-40 ? 0 : (R23 - m[3 * P + q] * m[P + q]) / m[2 * P + q];
  m[5 * P + q] = sqrt(fabs(R33 - m[3 * P + q] * m[3 * P + q] - m[4 * P + q] * m[4 * P + q]));
}

// compute_convolution_kernel (DigitalFilter.cu:441-489): exponential filter coefficients exp(-pi d |n|)
// normalised in the 2-norm, d the local y spacing (the second spacing at j = -ngg) or the mean z
// spacing, both over delta_omega.
__global__ void k_df_coeffs(DevDf d, const double *__restrict__ ysc, double dz_scaled) {
  const int j = (int)(blockIdx.x * blockDim.x + threadIdx.x) - d.g;
  if (j >= d.my + d.g) return;
  const int q = j + d.g, P = d.py;
  const double dy = j == -d.g ? ysc[2 * d.g + 1] - ysc[2 * d.g] : ysc[j + d.g] - ysc[j + d.g - 1];
  for (int pass = 0; pass < 2; ++pass) {
    double *b = pass == 0 ? d.by : d.bz;
    const double em = -kPi * (pass == 0 ? dy : dz_scaled);
    double sum = 0;
    for (int n = -kDfN; n <= kDfN; ++n) {
      const double e = exp(em * abs(n));
      b[(n + kDfN) * P + q] = e;
      sum += e * e;
    }
    sum = sqrt(sum);
    for (int n = -kDfN; n <= kDfN; ++n) b[(n + kDfN) * P + q] = b[(n + kDfN) * P + q] / sum;
  }
}

// generate_random_numbers_kernel (DigitalFilter.cu:491-503): one normal draw per padded node and
// component from its own state.
__global__ void k_df_generate(DevDf d) {
  const long long n_all = (long long)d.wy * d.wz * 3;
  for (long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x; f < n_all; f += (long long)gridDim.x * blockDim.x) {
    curandState s = d.rng[f];
    d.r[f] = curand_normal_double(&s);
    d.rng[f] = s;
  }
}

// remove_mean_spanwise (DigitalFilter.cu:505-537): per j and component, the mean over k = 0..mz-1
// removed and the result divided by the rms about it.
__global__ void k_df_remove_mean(DevDf d) {
  const int j = (int)(blockIdx.x * blockDim.x + threadIdx.x) - kDfN - d.g;
  if (j >= d.my + kDfN + d.g) return;
  double mean[3] = {0, 0, 0}, rms[3] = {0, 0, 0};
  for (int k = 0; k < d.mz; ++k)
    for (int c = 0; c < 3; ++c) {
      const double v = d.r[df_w(d, j, k, c)];
      mean[c] += v;
      rms[c] += v * v;
    }
  const double inv = 1.0 / d.mz;
  for (int c = 0; c < 3; ++c) {
    mean[c] *= inv;
    rms[c] = sqrt(rms[c] * inv - mean[c] * mean[c]);
  }
  for (int k = 0; k < d.mz; ++k)
    for (int c = 0; c < 3; ++c) {
      double &v = d.r[df_w(d, j, k, c)];
      v = (v - mean[c]) / rms[c];
    }
}

// apply_periodic_in_spanwise (DigitalFilter.cu:539-554): r(j, mz-1+k) = r(j, k) and
// r(j, -k) = r(j, mz-1-k) for k = 1..N+ngg.  The host allows the filter only where these reads stay
// in k = 0..mz-1 (mz - 1 >= N + ngg), where the reference's parallel copies do not race.
__global__ void k_df_periodic(DevDf d) {
  const int G = kDfN + d.g;
  const long long n_all = (long long)d.wy * G;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n_all; t += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(t % d.wy) - G, k = (int)(t / d.wy) + 1;
    for (int c = 0; c < 3; ++c) {
      d.r[df_w(d, j, d.mz - 1 + k, c)] = d.r[df_w(d, j, k, c)];
      d.r[df_w(d, j, -k, c)] = d.r[df_w(d, j, d.mz - 1 - k, c)];
    }
  }
}

// perform_convolution_y (DigitalFilter.cu:556-583): fy(j, k) = sum_n by(j, n) r(j + n, k), for
// j in [-ngg, my+ngg) and k in [-N-ngg, mz+N+ngg).
__global__ void k_df_conv_y(DevDf d) {
  const long long n_all = (long long)d.py * d.wz;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n_all; t += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(t % d.py) - d.g, k = (int)(t / d.py) - kDfN - d.g;
    const int q = j + d.g;
    for (int c = 0; c < 3; ++c) {
      double f = 0;
      for (int n = -kDfN; n <= kDfN; ++n) f += d.by[(n + kDfN) * d.py + q] * d.r[df_w(d, j + n, k, c)];
      d.fy[df_f(d, j, k, c)] = f;
    }
  }
}

// perform_convolution_z (DigitalFilter.cu:585-610): new(j, k) = sum_n bz(j, n) fy(j, k + n) over the
// face plane with its ghosts.
__global__ void k_df_conv_z(DevDf d) {
  const long long n_all = (long long)d.py * d.pz;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n_all; t += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(t % d.py) - d.g, k = (int)(t / d.py) - d.g;
    const int q = j + d.g;
    for (int c = 0; c < 3; ++c) {
      double f = 0;
      for (int n = -kDfN; n <= kDfN; ++n) f += d.bz[(n + kDfN) * d.py + q] * d.fy[df_f(d, j, k + n, c)];
      d.vnew[df_p(d, j, k, c)] = f;
    }
  }
}

// compute_fluctuations_first_step (DigitalFilter.cu:612-628): fluc = Lund x old.
__global__ void k_df_first(DevDf d) {
  const long long n_all = (long long)d.py * d.pz;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n_all; t += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(t % d.py) - d.g, k = (int)(t / d.py) - d.g;
    const int q = j + d.g, P = d.py;
    const double a = d.vold[df_p(d, j, k, 0)], b = d.vold[df_p(d, j, k, 1)], c = d.vold[df_p(d, j, k, 2)];
    d.fluc[df_p(d, j, k, 0)] = d.lund[q] * a;
    d.fluc[df_p(d, j, k, 1)] = d.lund[P + q] * a + d.lund[2 * P + q] * b;
    d.fluc[df_p(d, j, k, 2)] = d.lund[3 * P + q] * a + d.lund[4 * P + q] * b + d.lund[5 * P + q] * c;
  }
}

// Castro_time_correlation_and_fluc_computation (DigitalFilter.cu:630-678): with dt a third of the
// step's dt (*dtp; zero before the first step unless the step is fixed) and the integral time
// delta_omega / u(y), old = exp(-pi dt / T / 2) old + sqrt(1 - exp(-pi dt / T)) new (kept in both
// arrays), fluc = Lund x old.  u(y) is the inflow's tanh profile of the upper and lower u.
__global__ void k_df_correlate(DevDf d, const double *__restrict__ dtp, double u_upper, double u_lower,
                               double delta_omega) {
  const long long n_all = (long long)d.py * d.pz;
  const double dt = 1.0 / 3.0 * *dtp;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n_all; t += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(t % d.py) - d.g, k = (int)(t / d.py) - d.g;
    const int q = j + d.g, P = d.py;
    const double y = d.yface[(long long)(k + d.g) * d.py + q];
    const double u = 0.5 * (u_upper + u_lower) + 0.5 * (u_upper - u_lower) * tanh(2 * y / delta_omega);
    const double tlen = delta_omega / u;
    const double pdt = -kPi * dt / tlen;
    const double a1 = exp(pdt * 0.5), a2 = sqrt(1 - exp(pdt));
    double v[3];
    for (int c = 0; c < 3; ++c) {
      const long long i = df_p(d, j, k, c);
      v[c] = a1 * d.vold[i] + a2 * d.vnew[i];
      d.vnew[i] = v[c];
      d.vold[i] = v[c];
    }
    d.fluc[df_p(d, j, k, 0)] = d.lund[q] * v[0];
    d.fluc[df_p(d, j, k, 1)] = d.lund[P + q] * v[0] + d.lund[2 * P + q] * v[1];
    d.fluc[df_p(d, j, k, 2)] = d.lund[3 * P + q] * v[0] + d.lund[4 * P + q] * v[1] + d.lund[5 * P + q] * v[2];
  }
}

}  // namespace ostc
