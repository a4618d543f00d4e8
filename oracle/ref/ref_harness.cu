// ref_harness.cu -- runs the reference solver's own RK3 path on a case directory for parity checks.
// TEST INFRASTRUCTURE ONLY (built by oracle/ref/build_ref.sh into oracle/_ref/ref_harness).
//
// Usage (cwd = case directory holding ./input/setup.txt, grid and boundary files):
//   ref_harness state_in.bin state_out.bin
// It builds cfd::Parameter, cfd::Mesh and cfd::Driver<model, Laminar> as the reference's main() does
// (main.cu:8-136; model Air, Mixture or FR from the species/reaction keys), replaces the freshly
// initialised interior primitive variables with the ones in state_in.bin ([block][6 + n_spec][mz][my][mx]
// doubles: rho u v w p T, then the mass fractions), runs the reference's
// Driver::initialize_computation() and RK3() (RK.cuh:19-228) for total_step steps - or, when the setup
// has steady = 1, its steady_simulation() (SteadySim.cuh:15-140) for total_step iterations, or with
// temporal_scheme = 2 its dual_time_stepping() (DualTimeStepping.cuh:32-252) for total_step steps - and writes the
// interior cv[n_var], bv[6] and sv[n_spec] of every block, then the physical time, to state_out.bin.  It prints the
// wall time of the RK3 call (steps, per-step output checks and the final flow-field file included).
//
// The reference seeds the generator states of a white-noise inflow with the clock (time(), in
// DBoundCond::initialize_bc_on_GPU, BoundCond.cu:1731-1734).  build_ref.sh links this harness with
// --wrap=time, so that with OSTC_REF_TIME set the clock reads that value and the run is repeatable.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <ctime>
#include <exception>
#include <vector>

extern "C" time_t __real_time(time_t *t);
extern "C" time_t __wrap_time(time_t *t) {
  const char *v = std::getenv("OSTC_REF_TIME");
  if (!v) return __real_time(t);
  const time_t r = (time_t)std::strtoll(v, nullptr, 10);
  if (t) *t = r;
  return r;
}

#include "Parameter.h"
#include "Mesh.h"
#include "Driver.cuh"
#include "Simulate.cuh"
#include "SST.cuh"

namespace {
// element (i,j,k) of variable l of a VectorField3D with ngg ghosts (gxl_lib/Array.cuh:209-230)
long long padded_index(int mx, int my, int mz, int ngg, int i, int j, int k, int l) {
  const long long disp2 = mx + 2 * ngg;
  const long long disp1 = (my + 2 * ngg) * disp2;
  const long long dispt = (disp1 + disp2 + 1) * ngg;
  const long long sz = (long long)(mx + 2 * ngg) * (my + 2 * ngg) * (mz + 2 * ngg);
  return k * disp1 + j * disp2 + i + dispt + l * sz;
}

const char *g_stage = "start";
}  // namespace

template <MixtureModel M>
int run_model(cfd::Parameter &parameter, cfd::Mesh &mesh, const char *fin, const char *fout) {
  g_stage = "Driver";
  cfd::Driver<M, cfd::Laminar> driver(parameter, mesh);
  const int n_var = parameter.get_int("n_var"), n_spec = parameter.get_int("n_spec");

  g_stage = "state_in";
  std::FILE *f = std::fopen(fin, "rb");
  if (!f) {
    std::fprintf(stderr, "cannot open %s\n", fin);
    return 2;
  }
  for (int b = 0; b < mesh.n_block; ++b) {
    const int mx = mesh[b].mx, my = mesh[b].my, mz = mesh[b].mz, ngg = mesh[b].ngg;
    const long long n = (long long)mx * my * mz;
    const long long sz = (long long)(mx + 2 * ngg) * (my + 2 * ngg) * (mz + 2 * ngg);
    std::vector<double> in((6 + n_spec) * n), pad(6 * sz), spad(n_spec > 0 ? n_spec * sz : 1);
    if (std::fread(in.data(), sizeof(double), in.size(), f) != in.size()) {
      std::fprintf(stderr, "short state file\n");
      return 2;
    }
    cudaMemcpy(pad.data(), driver.field[b].h_ptr->bv.data(), pad.size() * sizeof(double), cudaMemcpyDeviceToHost);
    for (int l = 0; l < 6; ++l)
      for (int k = 0; k < mz; ++k)
        for (int j = 0; j < my; ++j)
          for (int i = 0; i < mx; ++i)
            pad[padded_index(mx, my, mz, ngg, i, j, k, l)] = in[l * n + ((long long)k * my + j) * mx + i];
    cudaMemcpy(driver.field[b].h_ptr->bv.data(), pad.data(), pad.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (n_spec > 0) {
      cudaMemcpy(spad.data(), driver.field[b].h_ptr->sv.data(), spad.size() * sizeof(double), cudaMemcpyDeviceToHost);
      for (int l = 0; l < n_spec; ++l)
        for (int k = 0; k < mz; ++k)
          for (int j = 0; j < my; ++j)
            for (int i = 0; i < mx; ++i)
              spad[padded_index(mx, my, mz, ngg, i, j, k, l)] = in[(6 + l) * n + ((long long)k * my + j) * mx + i];
      cudaMemcpy(driver.field[b].h_ptr->sv.data(), spad.data(), spad.size() * sizeof(double), cudaMemcpyHostToDevice);
    }
  }
  std::fclose(f);

  g_stage = "initialize_computation";
  driver.initialize_computation();
  const bool steady = parameter.get_bool("steady"), dual = !steady && parameter.get_int("temporal_scheme") == 2;
  g_stage = steady ? "steady_simulation" : dual ? "dual_time_stepping" : "RK3";
  cudaDeviceSynchronize();
  const auto t_begin = std::chrono::steady_clock::now();
  // the time-advance driver Simulate.cuh picks: the steady local-time-step loop (SteadySim.cuh), dual
  // time stepping (DualTimeStepping.cuh, temporal_scheme 2) or RK3
  if (steady) cfd::steady_simulation<M, cfd::Laminar>(driver);
  else if (dual) cfd::dual_time_stepping<M, cfd::Laminar>(driver);
  else cfd::RK3<M, cfd::Laminar>(driver);
  cudaDeviceSynchronize();
  const double rk3_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_begin).count();
  std::printf("ref_harness: rk3_seconds = %.6f\n", rk3_seconds);

  g_stage = "state_out";
  f = std::fopen(fout, "wb");
  for (int b = 0; b < mesh.n_block; ++b) {
    const int mx = mesh[b].mx, my = mesh[b].my, mz = mesh[b].mz, ngg = mesh[b].ngg;
    const long long n = (long long)mx * my * mz;
    const long long sz = (long long)(mx + 2 * ngg) * (my + 2 * ngg) * (mz + 2 * ngg);
    const int nout = n_var + 6 + n_spec;
    std::vector<double> cv(n_var * sz), bv(6 * sz), sv(n_spec > 0 ? n_spec * sz : 1), out(nout * n);
    cudaMemcpy(cv.data(), driver.field[b].h_ptr->cv.data(), cv.size() * sizeof(double), cudaMemcpyDeviceToHost);
    cudaMemcpy(bv.data(), driver.field[b].h_ptr->bv.data(), bv.size() * sizeof(double), cudaMemcpyDeviceToHost);
    if (n_spec > 0)
      cudaMemcpy(sv.data(), driver.field[b].h_ptr->sv.data(), sv.size() * sizeof(double), cudaMemcpyDeviceToHost);
    for (int l = 0; l < nout; ++l)
      for (int k = 0; k < mz; ++k)
        for (int j = 0; j < my; ++j)
          for (int i = 0; i < mx; ++i) {
            double v;
            if (l < n_var) v = cv[padded_index(mx, my, mz, ngg, i, j, k, l)];
            else if (l < n_var + 6) v = bv[padded_index(mx, my, mz, ngg, i, j, k, l - n_var)];
            else v = sv[padded_index(mx, my, mz, ngg, i, j, k, l - n_var - 6)];
            out[l * n + ((long long)k * my + j) * mx + i] = v;
          }
    std::fwrite(out.data(), sizeof(double), out.size(), f);
  }
  const double t = parameter.get_real("solution_time");
  std::fwrite(&t, sizeof(double), 1, f);
  std::fclose(f);
  const cudaError_t e = cudaGetLastError();
  std::printf("ref_harness: done (%s), t = %.17g\n", cudaGetErrorString(e), t);
  return e == cudaSuccess ? 0 : 1;
}

int run(const char *fin, const char *fout, int *argc, char ***argv) {
  g_stage = "Parameter";
  cfd::Parameter parameter(argc, argv);
  // the reference reads total_simulation_time without a default (Simulate.cuh:62, RK.cuh:64); the run
  // is bounded by total_step instead
  parameter.update_parameter("total_simulation_time", 1e30);
  g_stage = "Mesh";
  cfd::Mesh mesh(parameter);
  if (!parameter.get_bool("turbulence")) parameter.update_parameter("turbulence_method", 0);
  // model selection as main.cu:60-71 (laminar): species 1 with reaction 1 -> FR, else Mixture
  if (parameter.get_int("species") == 1) {
    if (parameter.get_int("reaction") == 1) return run_model<MixtureModel::FR>(parameter, mesh, fin, fout);
    return run_model<MixtureModel::Mixture>(parameter, mesh, fin, fout);
  }
  return run_model<MixtureModel::Air>(parameter, mesh, fin, fout);
}

int main(int argc, char *argv[]) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: ref_harness state_in.bin state_out.bin\n");
    return 2;
  }
  std::setvbuf(stdout, nullptr, _IONBF, 0);
  int one = 1;
  char **av = argv;
  try {
    return run(argv[1], argv[2], &one, &av);
  } catch (const std::exception &e) {
    std::fprintf(stderr, "ref_harness: exception in stage %s: %s\n", g_stage, e.what());
    return 5;
  }
}
