// api_plt.cuh -- C ABI (include/ostc.h): the Tecplot flow-field file (FieldIO layout) written
// from zones packed on the device, and the restart reader.
// Part of the ostc_b200.cu translation unit (included in order; not a standalone header).
#pragma once

extern "C" {

// ---------------------------------------------------------------- Tecplot flow-field file

// The zone data of one block in the flow-field file's layout, packed on the device
// (FieldIO::print_field, FieldIO.h:560-648): variable-major arrays over the (mx+2g)(my+2g)(mz+2g) output
// nodes, i fastest; x, y, z from xyz (the same layout), then rho u v w p T, the Mach number as
// update_physical_properties stores it (FieldOperation.cuh:107-140: |V| over the mixture speed of sound,
// or over sqrt(gamma R T) for air) and the mass fractions.  2-D blocks hold no k ghosts: their output k
// layers repeat k = 0, the copies eliminate_k_gradient makes in the reference.
__global__ void k_plt_pack(DevBlock b, DevState s, const double *__restrict__ xyz, int g, int ns, int mixture,
                           double *__restrict__ out) {
  const int nx = b.mx + 2 * g, ny = b.my + 2 * g, nz = b.mz + 2 * g;
  const long long npt = (long long)nx * ny * nz, P = b.plane;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < npt; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % nx) - g;
    const long long r = q / nx;
    const int j = (int)(r % ny) - g, k = (int)(r / ny) - g;
    const long long p = b.id(i, j, b.gz ? k : 0);
    out[q] = xyz[q];
    out[npt + q] = xyz[npt + q];
    out[2 * npt + q] = xyz[2 * npt + q];
    for (int l = 0; l < 6; ++l) out[(3 + l) * npt + q] = s.bv[l * P + p];
    const double u = s.bv[P + p], v = s.bv[2 * P + p], w = s.bv[3 * P + p];
    const double vel = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(u, u), __dmul_rn(v, v)), __dmul_rn(w, w)));
    out[9 * npt + q] = mixture ? vel / s.acs[p] : vel / sqrt(kGammaAir * kRu / kMwAir * s.bv[5 * P + p]);
    for (int l = 0; l < ns; ++l) out[(10 + l) * npt + q] = s.sv[l * P + p];
  }
}

// Per-block partial minima and maxima of every packed variable (the file's min/max pairs): block x of
// row y covers variable y; part[(y * gridDim.x + x) * 2 + 0/1].
__global__ void __launch_bounds__(256) k_plt_minmax(const double *__restrict__ a, long long npt, double *__restrict__ part) {
  __shared__ double smin[256], smax[256];
  const double *v = a + (long long)blockIdx.y * npt;
  double mn = v[0], mxv = v[0];
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < npt; q += (long long)gridDim.x * blockDim.x) {
    mn = fmin(mn, v[q]);
    mxv = fmax(mxv, v[q]);
  }
  smin[threadIdx.x] = mn;
  smax[threadIdx.x] = mxv;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) {
      smin[threadIdx.x] = fmin(smin[threadIdx.x], smin[threadIdx.x + h]);
      smax[threadIdx.x] = fmax(smax[threadIdx.x], smax[threadIdx.x + h]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const long long o = ((long long)blockIdx.y * gridDim.x + blockIdx.x) * 2;
    part[o] = smin[0];
    part[o + 1] = smax[0];
  }
}

// The interior primitive state and mass fractions of one zone read from a flow-field file (its
// selected variable columns cols[6 + ns][npt] staged on the device) into [6][N] and [ns][N].
__global__ void k_plt_gather(DevBlock b, int g, int ns, const double *__restrict__ cols, double *__restrict__ bv,
                             double *__restrict__ sv) {
  const int nx = b.mx + 2 * g, ny = b.my + 2 * g;
  const long long npt = (long long)nx * ny * (b.mz + 2 * g);
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < b.n; n += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(n % b.mx);
    const long long r = n / b.mx;
    const int j = (int)(r % b.my), k = (int)(r / b.my);
    const long long q = ((long long)(k + g) * ny + (j + g)) * nx + (i + g);
    for (int l = 0; l < 6; ++l) bv[l * b.n + n] = cols[l * npt + q];
    for (int l = 0; l < ns; ++l) sv[l * b.n + n] = cols[(6 + l) * npt + q];
  }
}

// Variable names of the flow-field file: FieldIO::acquire_variable_names (FieldIO.h:450-488) for a
// laminar air or mixture case without user-defined output (UDIO.cu:9-33).
static std::vector<std::string> plt_names(const ostc_ctx *ctx) {
  std::vector<std::string> v{"x", "y", "z", "density", "u", "v", "w", "pressure", "temperature", "mach"};
  for (int l = 0; l < ctx->der.n_spec; ++l) v.push_back(ctx->chem.names[l]);
  return v;
}

int ostc_write_plt(ostc_ctx *ctx, const char *path, int ngg_out, double solution_time) {
  if (!ctx || !path) return OSTC_EINVAL;
  cudaSetDevice(ctx->device);
  if (int r = check_ready(ctx)) return r;
  if (ngg_out < 0 || ngg_out > ctx->der.ngg) {
    ctx->err = "ostc_write_plt: ngg_out must lie in [0, ngg]";
    return OSTC_EINVAL;
  }
  CK(cudaStreamSynchronize(ctx->stream));
  const std::vector<std::string> names = plt_names(ctx);
  const int nvar = (int)names.size(), ns = ctx->der.n_spec;
  std::vector<char> buf;
  auto put = [&](const void *p, size_t n) { buf.insert(buf.end(), (const char *)p, (const char *)p + n); };
  auto put_i = [&](int v) { put(&v, 4); };
  auto put_f = [&](float v) { put(&v, 4); };
  auto put_d = [&](double v) { put(&v, 8); };
  auto put_s = [&](const std::string &s) {
    for (char c : s) put_i((int)c);
    put_i(0);
  };
  // header (FieldIO::write_header, FieldIO.h:73-200)
  put("#!TDV112", 8);
  put_i(1);
  put_i(0);
  put_s("Solution file");
  put_i(nvar);
  for (const auto &n : names) put_s(n);
  const int g = ngg_out;
  for (size_t b = 0; b < ctx->blk.size(); ++b) {
    const DevBlock &db = ctx->blk[b].db;
    put_f(299.0f);
    put_s("zone " + std::to_string(b));
    put_i(-1);
    put_i(-2);
    put_d(solution_time);
    put_i(-1);
    put_i(0);
    put_i(0);
    put_i(0);
    put_i(0);
    put_i(db.mx + 2 * g);
    put_i(db.my + 2 * g);
    put_i(db.mz + 2 * g);
    put_i(0);
  }
  put_f(357.0f);
  // data sections (write_common_data_section + print_field, FieldIO.h:222-648): per zone the
  // formats, the min/max pairs and the node arrays of x, y, z, bv, mach, Y_k - packed and reduced on
  // the device, then one copy of the packed zone into the file image
  for (size_t b = 0; b < ctx->blk.size(); ++b) {
    BlockRes &B = ctx->blk[b];
    const DevBlock &db = B.db;
    const int nx = db.mx + 2 * g, ny = db.my + 2 * g, nz = db.mz + 2 * g;
    const long long npt = (long long)nx * ny * nz;
    if (!B.plt_xyz || B.plt_g != g) {
      // the zone's coordinates (ghost grid included) uploaded once per output width
      const HostBlock &hb = ctx->mesh.blocks[b];
      std::vector<double> xyz(3 * (size_t)npt);
      for (int k = -g; k < db.mz + g; ++k)
        for (int j = -g; j < db.my + g; ++j)
          for (int i = -g; i < db.mx + g; ++i) {
            const long long q = ((long long)(k + g) * ny + (j + g)) * nx + (i + g);
            const long c = hb.cidx(i, j, k);
            xyz[q] = hb.x[c];
            xyz[npt + q] = hb.y[c];
            xyz[2 * npt + q] = hb.z[c];
          }
      cudaFree(B.plt_xyz);
      B.plt_xyz = nullptr;
      CK(cudaMalloc(&B.plt_xyz, xyz.size() * sizeof(double)));
      CK(cudaMemcpy(B.plt_xyz, xyz.data(), xyz.size() * sizeof(double), cudaMemcpyHostToDevice));
      B.plt_g = g;
    }
    double *dev = nullptr, *part = nullptr;
    const int nb = (int)std::min<long long>(256, (npt + 255) / 256);
    if (cudaMalloc(&dev, (size_t)nvar * npt * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&part, (size_t)nvar * nb * 2 * sizeof(double)) != cudaSuccess) {
      cudaFree(dev);
      ctx->err = "ostc_write_plt: device allocation for the packed zone failed";
      return OSTC_ENOMEM;
    }
    k_plt_pack<<<grid_for(ctx, npt, 256), 256, 0, ctx->stream>>>(db, state_of(B, 0), B.plt_xyz, g, ns,
                                                                  ctx->mixture ? 1 : 0, dev);
    k_plt_minmax<<<dim3(nb, nvar), 256, 0, ctx->stream>>>(dev, npt, part);
    std::vector<double> hp((size_t)nvar * nb * 2);
    const cudaError_t e1 = cudaMemcpyAsync(hp.data(), part, hp.size() * sizeof(double), cudaMemcpyDeviceToHost,
                                           ctx->stream);
    put_f(299.0f);
    for (int l = 0; l < nvar; ++l) put_i(2);
    put_i(0);
    put_i(0);
    put_i(-1);
    const cudaError_t e2 = cudaStreamSynchronize(ctx->stream);
    for (int l = 0; l < nvar; ++l) {
      double mn = hp[(size_t)l * nb * 2], mxv = hp[(size_t)l * nb * 2 + 1];
      for (int x = 1; x < nb; ++x) {
        mn = std::min(mn, hp[((size_t)l * nb + x) * 2]);
        mxv = std::max(mxv, hp[((size_t)l * nb + x) * 2 + 1]);
      }
      put_d(mn);
      put_d(mxv);
    }
    const size_t at = buf.size();
    buf.resize(at + (size_t)nvar * npt * sizeof(double));
    const cudaError_t e3 =
        cudaMemcpy(buf.data() + at, dev, (size_t)nvar * npt * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(dev);
    cudaFree(part);
    if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess) {
      ctx->err = "ostc_write_plt: device packing failed";
      return OSTC_ECUDA;
    }
  }
  FILE *f = std::fopen(path, "wb");
  if (!f) {
    ctx->err = std::string("ostc_write_plt: cannot open ") + path + " for writing";
    return OSTC_EIO;
  }
  const bool ok = std::fwrite(buf.data(), 1, buf.size(), f) == buf.size();
  if (std::fclose(f) != 0 || !ok) {
    ctx->err = std::string("ostc_write_plt: write to ") + path + " failed";
    return OSTC_EIO;
  }
  return OSTC_OK;
}

int ostc_read_plt(ostc_ctx *ctx, const char *path, double *solution_time) {
  if (!ctx || !path) return OSTC_EINVAL;
  cudaSetDevice(ctx->device);
  FILE *f = std::fopen(path, "rb");
  if (!f) {
    ctx->err = std::string("ostc_read_plt: cannot open ") + path;
    return OSTC_EIO;
  }
  std::vector<char> buf;
  char chunk[1 << 16];
  size_t got;
  while ((got = std::fread(chunk, 1, sizeof(chunk), f)) > 0) buf.insert(buf.end(), chunk, chunk + got);
  std::fclose(f);
  size_t pos = 0;
  bool bad = false;
  auto take = [&](void *dst, size_t n) {
    if (pos + n > buf.size()) {
      bad = true;
      std::memset(dst, 0, n);
      return;
    }
    std::memcpy(dst, buf.data() + pos, n);
    pos += n;
  };
  auto get_i = [&]() { int v; take(&v, 4); return v; };
  auto get_f = [&]() { float v; take(&v, 4); return v; };
  auto get_d = [&]() { double v; take(&v, 8); return v; };
  auto get_s = [&]() {
    std::string s;
    for (int c = get_i(); c != 0 && !bad && s.size() < 4096; c = get_i()) s.push_back((char)c);
    return s;
  };
  auto fail = [&](const std::string &why) {
    ctx->err = std::string("ostc_read_plt: ") + path + ": " + why;
    return OSTC_EIO;
  };
  // header (read_flowfield, Initialize.cuh:102-215)
  if (buf.size() < 8 || std::memcmp(buf.data(), "#!TDV", 5) != 0) return fail("not a Tecplot binary file");
  pos = 8;
  get_i();
  get_i();
  get_s();
  const int nvar = get_i();
  if (bad || nvar <= 0 || nvar > 4096) return fail("bad variable count");
  std::vector<std::string> names(nvar);
  for (auto &n : names) n = get_s();
  std::vector<std::array<int, 3>> dims;
  double t0 = 0;
  float marker = get_f();
  while (!bad && std::fabs(marker - 299.0f) < 1e-3f) {
    get_s();
    get_i();
    get_i();
    const double t = get_d();
    if (dims.empty()) t0 = t;
    get_i();
    if (get_i() != 0) return fail("only ordered zones are read");
    if (get_i() != 0) return fail("only node-located data is read");
    get_i();
    get_i();
    const int d0 = get_i(), d1 = get_i(), d2 = get_i();
    dims.push_back({d0, d1, d2});
    if (get_i() != 0) return fail("zone auxiliary data is not read");
    marker = get_f();
  }
  if (bad || std::fabs(marker - 357.0f) > 1e-3f) return fail("header does not end with the end-of-header marker");
  if (dims.size() != ctx->blk.size()) return fail("zone count differs from the case's block count");
  auto find = [&](const std::string &n) {
    for (int l = 0; l < nvar; ++l)
      if (names[l] == n) return l;
    return -1;
  };
  static const char *const kPrim[6] = {"density", "u", "v", "w", "pressure", "temperature"};
  int col[6 + kMS];
  for (int l = 0; l < 6; ++l)
    if ((col[l] = find(kPrim[l])) < 0) return fail(std::string("no variable '") + kPrim[l] + "'");
  const int ns = ctx->der.n_spec;
  for (int l = 0; l < ns; ++l)
    if ((col[6 + l] = find(ctx->chem.names[l])) < 0) return fail("no variable for species " + ctx->chem.names[l]);
  for (size_t b = 0; b < ctx->blk.size(); ++b) {
    const DevBlock &db = ctx->blk[b].db;
    const int nx = dims[b][0], ny = dims[b][1], nz = dims[b][2];
    const int g = (nx - db.mx) / 2;
    if (g < 0 || nx != db.mx + 2 * g || ny != db.my + 2 * g || nz != db.mz + 2 * g)
      return fail("zone " + std::to_string(b) + " extents do not match block " + std::to_string(b));
    if (std::fabs(get_f() - 299.0f) > 1e-3f) return fail("missing zone data marker");
    for (int l = 0; l < nvar; ++l)
      if (get_i() != 2) return fail("only double-precision variables are read");
    if (get_i() != 0 || get_i() != 0) return fail("passive or shared variables are not read");
    get_i();
    for (int l = 0; l < 2 * nvar; ++l) get_d();
    const long long npt = (long long)nx * ny * nz;
    if (bad || pos + (size_t)nvar * npt * 8 > buf.size()) return fail("truncated zone data");
    const char *a = buf.data() + pos;
    pos += (size_t)nvar * npt * 8;
    // the zone's primitive and species columns go to the device as they lie in the file; the interior
    // is gathered there and set as the block's state
    const long long N = db.n;
    double *cols = nullptr, *st = nullptr;
    if (cudaMalloc(&cols, (size_t)(6 + ns) * npt * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&st, (size_t)(6 + ns) * N * sizeof(double)) != cudaSuccess) {
      cudaFree(cols);
      ctx->err = "ostc_read_plt: device allocation for the zone failed";
      return OSTC_ENOMEM;
    }
    bool okc = true;
    for (int l = 0; l < 6 + ns && okc; ++l)
      okc = cudaMemcpyAsync(cols + (size_t)l * npt, a + (size_t)col[l] * npt * 8, npt * sizeof(double),
                            cudaMemcpyHostToDevice, ctx->stream) == cudaSuccess;
    if (okc) k_plt_gather<<<grid_for(ctx, N, 256), 256, 0, ctx->stream>>>(db, g, ns, cols, st, st + 6 * N);
    const int r = okc ? ostc_set_state(ctx, (int)b, st, ns ? st + 6 * N : nullptr, OSTC_DEVICE) : OSTC_ECUDA;
    cudaFree(cols);
    cudaFree(st);
    if (r) return r;
  }
  // the physical time continues from the file's solution time
  CK(cudaMemcpyAsync(ctx->d_time, &t0, sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (solution_time) *solution_time = t0;
  return OSTC_OK;
}

}  // extern "C"
