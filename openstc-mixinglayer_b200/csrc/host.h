// host.h -- host-side (C++) data of the B200 OpenSTC library: the setup.txt parameter store, the
// block geometry (ghost grid, metrics, Jacobian) and the boundary-face tables.  Everything here is
// set-up work done once per context; the per-step path is in the CUDA sources.
#pragma once

#include <array>
#include <map>
#include <string>
#include <variant>
#include <vector>

#include "chem.h"

namespace ostc {

// Physical constants (Constants.h:18,26,31-35 of the reference).
constexpr double kGammaAir = 1.4;
constexpr double kRu = 8314.462618;
constexpr double kMwAir = 28.9647;

// Typed key/value store with the grammar of cfd::Parameter::read_one_file (Parameter.cpp:39-185):
//   <int|real|bool|string> key = value      one value per line, text after it ignored
//   array <int|real|string> name [=] { ... }   values over one or more lines, closed by "}"
//   struct name = { <type> key = value ... }  closing "}" on its own line
//   range <int|real> name = { 2, 4 or 6 values }
// Lines starting with "//" or "!" and empty lines are skipped; a later definition overrides.
struct Setup {
  using StructVal = std::variant<std::string, int, double>;
  std::map<std::string, int> ints;
  std::map<std::string, double> reals;
  std::map<std::string, bool> bools;
  std::map<std::string, std::string> strings;
  std::map<std::string, std::vector<int>> int_arrays;
  std::map<std::string, std::vector<double>> real_arrays;
  std::map<std::string, std::vector<std::string>> string_arrays;
  std::map<std::string, std::map<std::string, StructVal>> structs;
  std::map<std::string, std::vector<double>> real_ranges;
  std::map<std::string, std::vector<int>> int_ranges;

  void set_defaults();  // Parameter::setup_default_settings (Parameter.cpp:439-564), path-relevant keys
  bool read_file(const std::string &path, std::string &err);
  int get_int(const std::string &k) const;
  double get_real(const std::string &k) const;
  bool get_bool(const std::string &k) const;
};

// Values derived from the setup (Parameter::deduce_known_info / deduce_sim_info,
// Parameter.cpp:187-437, 589-653) that the hot path needs.
struct Derived {
  int ngg = 2;
  int inviscid_type = 0;  // 0 pv reconstruction, 1 AWENO, 2 Roe, 3 char. WENO (FVS), 4 EP
  int n_var = 5;
  int n_scalar = 0;
  int n_spec = 0;
  int reconstruction = 2;
  int inviscid_scheme = 3;
  // Riemann solver the face flux actually uses: 1 Lax-Friedrichs, 2 Roe, 3 AUSM+, 4 HLLC.  The
  // reference's switches fall back to AUSM+ for any other inviscid_scheme (InviscidScheme.cu:145-159,
  // 345-359), and AWENO with inviscid_scheme 2 lands there too (inviscid_type 1 takes precedence).
  int riemann = 3;
  int limiter = 0;                  // 0 and 1 are both minmod (Limiter.cuh:8-17)
  double entropy_fix_factor = 0.125;
  int viscous_order = 2;
  double cfl = 1.0;
  double prandtl = 0.72;
  bool steady = true;
  int temporal_scheme = 3;
  int implicit_method = 0;   // steady driver: 0 explicit, 1 DPLUR
  int dplur_inner = 3;       // DPLUR inner iterations
  int chem_src_method = 0;   // 0 explicit, 1 EPI, 2 DA (forced 0 under RK3)
  double convergence_criteria = 1e-8;
  int output_screen = 100;   // steady driver: residual check every output_screen iterations
  int inner_iteration = 20, max_inner_iteration = 30, iteration_adjust_step = 20;  // dual time stepping
  bool fixed_time_step = false;
  double dt = 1e-8;
  double grid_scale = 1.0;
  int species = 0;
  int reaction = 0;
  int problem_type = 0;  // 0 general, 1 mixing layer (inflows take the two-stream profile)
};

bool derive(const Setup &s, Derived &d, std::string &err);

// Boundary types (labels of the reference, BoundCond.cu:232-258).
enum BcType { kWall = 2, kSymmetry = 3, kFarfield = 4, kInflow = 5, kOutflow = 6, kSubsonicInflow = 7,
              kPeriodic = 8, kBackPressure = 9 };

// One boundary face after Boundary::register_boundary (Mesh.cpp:14-32).
struct BcFace {
  int label = 0;
  int type = 0;
  int face = 0;       // normal direction 0/1/2
  int direction = 1;  // -1 on the low face, +1 on the high face
  int rs[3]{}, re[3]{};
  // far-field state (FarField ctor, BoundCond.cpp:586-669), air only on this path
  double density = 0, u = 0, v = 0, w = 0, pressure = 0, temperature = 0;
  double acoustic_speed = 0, gamma = kGammaAir, entropy = 0, mw = kMwAir;
  int wall_adiabatic = 0;  // walls: 1 adiabatic, 0 isothermal at `temperature` (Wall, BoundCond.h:87-112)
  // constant supersonic inflow (Inflow ctor, BoundCond.cpp:157-214): the struct it reads and, for
  // mixtures, its mass fractions (filled once the species tables are known)
  std::string struct_name;
  std::vector<double> y;
  // inflow kind (Inflow ctor, BoundCond.cpp:10-21): 0 constant, 2 mixing-layer profile (every inflow
  // of a problem_type 1 case); fluctuation_type 1 adds white noise of relative intensity
  // fluct_intensity to the velocity (apply_inflow, BoundCond.cuh:402-425, 500-521); velocity is the
  // Inflow's `velocity` member (the constant inflow scales its noise by it)
  int inflow_type = 0, fluctuation_type = 0;
  double fluct_intensity = 0, velocity = 0, delta_omega = 0;
  // mixing-layer profile: the lower stream (rho, u, v, w, p, T) and its mass fractions; the upper
  // stream is density .. temperature and y above
  double lower[6]{};
  std::vector<double> y_lower;
  // digital-filter inflow (fluctuation_type 11 of a mixing-layer inflow): the peak Reynolds stresses
  // R11 R12 R22 R13 R23 R33 of the assumed Gaussian profile (df_reynolds_gaussian_peak)
  std::vector<double> df_rij;
};

// The two streams of a mixing-layer problem (get_mixing_layer_info, MixingLayer.cu:9-191): rho, u, v,
// w, p, T of the upper and lower stream and their mass fractions (mixtures).
struct MixingLayerStreams {
  double upper[6]{}, lower[6]{};
  std::vector<double> y_upper, y_lower;
  double delta_omega = 0;
};
bool mixing_layer_streams(const Setup &s, const ChemTables *chem, MixingLayerStreams &m, std::string &err);


// One 1:1 block interface after InnerFace::register_boundary (Mesh.cpp:34-176): the node range of
// this block it writes (the coincident face plus ngg ghost layers), the matching start in the target
// block, and the index map src_tar / loop directions between the two.
struct InnerFace {
  int rs[3]{}, re[3]{};
  int face = 0, direction = 1;
  int ts[3]{}, te[3]{};
  int target_block = 0, target_face = 0, target_direction = 1;
  int src_tar[3]{};
  int loop_dir[3]{1, 1, 1}, target_loop_dir[3]{1, 1, 1};
  int n_point[3]{1, 1, 1};
};

struct HostBlock {
  int mx = 0, my = 0, mz = 0, ngg = 0;
  // coordinates with ngg+1 ghost layers, Fortran order (Mesh.cpp:229-231)
  std::vector<double> x, y, z;
  // Jacobian and metric with ngg ghost layers; metric as 9 planes (r-1)*3+(c-1)
  std::vector<double> jac, metric;
  std::vector<BcFace> faces;   // file order
  std::vector<InnerFace> inner;
  long cidx(int i, int j, int k) const {
    const int g = ngg + 1;
    return ((long)(k + g) * (my + 2 * g) + (j + g)) * (mx + 2 * g) + (i + g);
  }
  long gidx(int i, int j, int k) const {
    return ((long)(k + ngg) * (my + 2 * ngg) + (j + ngg)) * (mx + 2 * ngg) + (i + ngg);
  }
  long padded() const { return (long)(mx + 2 * ngg) * (my + 2 * ngg) * (mz + 2 * ngg); }
};

struct HostMesh {
  int dimension = 3;
  std::vector<HostBlock> blocks;
};

// Reads "<dir>/grid/grid   0.dat" (binary, Mesh.cpp:663-697), the boundary and inner-face files
// (Mesh.cpp:790-844), scales, builds ghost grids and metrics.
bool read_mesh(const std::string &input_dir, const Derived &d, HostMesh &mesh, std::string &err);
// Attaches types and far-field states to the faces from the setup's boundary structs
// (DBoundCond::initialize_bc_on_GPU, BoundCond.cu:162-258).
bool resolve_boundaries(const Setup &s, const Derived &d, HostMesh &mesh, std::string &err);
// Inflow face states from their structs, with the species tables of a mixture case (nullptr: air).
bool resolve_inflows(const Setup &s, const ChemTables *chem, HostMesh &mesh, std::string &err);
// rho_inf^2 v_inf^2 and v_inf of the struct named by reference_state (0, 0 without one): the scales of
// the flux-split WENO epsilon (DParameter.cu:26-29, WENO.cu:1466-1473).
bool reference_scales(const Setup &s, const ChemTables *chem, double &eps_scale, double &v_ref, std::string &err);
// The state (rho, u, v, w, p, T; mass fractions y, acoustic speed c; gamma through gamma_out) of a plain
// inflow struct, as the reference's default initialisation fills every node of a block with it
// (Field.cu:316-345).
bool inflow_state(const Setup &s, const std::string &name, const ChemTables *chem, double bv[6],
                  std::vector<double> &y, double &c, std::string &err, double *gamma_out = nullptr);
// Order in which faces are applied each stage (BoundCond.cuh:1488-1679): a list of (block, face).
std::vector<std::pair<int, int>> bc_order(const Setup &s, const HostMesh &mesh);

}  // namespace ostc
