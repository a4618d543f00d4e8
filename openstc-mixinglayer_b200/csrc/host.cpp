// host.cpp -- setup.txt parsing, derived parameters, grid/boundary file reading, ghost grids,
// metrics and boundary registration.  All of it restates the reference's host-side set-up so that
// the device path sees exactly the values the reference computes.
#include "host.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>

namespace ostc {

// ------------------------------------------------------------------------------------ setup.txt

void Setup::set_defaults() {
  ints["problem_type"] = 0;
  ints["mesh_file_type"] = 0;
  ints["gridIsBinary"] = 0;
  reals["gridScale"] = 1.0;
  bools["steady"] = true;
  ints["implicit_method"] = 0;
  ints["temporal_scheme"] = 3;
  bools["fixed_time_step"] = false;
  reals["dt"] = 1e-8;
  ints["inviscid_scheme"] = 3;
  ints["reconstruction"] = 2;
  ints["limiter"] = 0;
  reals["entropy_fix_factor"] = 0.125;
  ints["viscous_order"] = 2;
  bools["gradPInDiffusionFlux"] = false;
  bools["positive_preserving"] = false;
  ints["species"] = 0;
  ints["reaction"] = 0;
  strings["therm_file"] = "chemistry/therm.dat";
  strings["transport_file"] = "chemistry/tran.dat";
  ints["chemSrcMethod"] = 0;
  ints["DPLUR_inner_step"] = 3;         // Parameter.cpp:450
  ints["inner_iteration"] = 20;         // Parameter.cpp:466-468
  ints["max_inner_iteration"] = 30;
  ints["iteration_adjust_step"] = 20;
  reals["convergence_criteria"] = 1e-8;  // Parameter.cpp:451
  bools["turbulence"] = false;
  ints["turbulence_method"] = 1;
  ints["RANS_model"] = 2;
  ints["n_ps"] = 0;
  reals["schmidt_number"] = 0.5;
  reals["prandtl_number"] = 0.72;
  reals["turbulent_prandtl_number"] = 0.9;
  reals["turbulent_schmidt_number"] = 0.9;
  bools["limit_flow"] = false;
  bools["sponge_layer"] = false;
  reals["cfl"] = 1.0;
  ints["total_step"] = 1;
  ints["output_screen"] = 100;
  string_arrays["boundary_conditions"] = {};
}

namespace {
// Reads tokens of one line into arr until "}" (returns false: array finished) or "//" / end of
// line (returns true: continue on the next line).  Parameter::read_line_to_array, Parameter.cpp:136-160.
template <typename T>
bool read_line_to_array(std::istringstream &line, std::vector<T> &arr) {
  std::string tok;
  while (line >> tok) {
    if (tok == "}") return false;
    if (tok == "//") break;
    if constexpr (std::is_same_v<T, double>) arr.push_back(std::stod(tok));
    else if constexpr (std::is_same_v<T, int>) arr.push_back(std::stoi(tok));
    else arr.push_back(tok);
  }
  return true;
}

void next_line(std::ifstream &f, std::string &input, std::istringstream &line) {
  if (!std::getline(f, input)) input.clear();
  const auto s = input.find_first_not_of(" \t");
  input = s == std::string::npos ? std::string() : input.substr(s);
  line.clear();
  line.str(input);
}

template <typename T>
void read_array(std::ifstream &f, std::string &input, std::istringstream &line, std::vector<T> &arr) {
  while (read_line_to_array(line, arr)) {
    if (!f) break;
    next_line(f, input, line);
    if (!f && input.empty()) break;
  }
}
}  // namespace

bool Setup::read_file(const std::string &path, std::string &err) {
  std::ifstream f(path);
  if (!f) {
    err = "cannot open setup file " + path;
    return false;
  }
  std::string input, type, key, temp;
  std::istringstream line;
  try {
    while (std::getline(f, input)) {
      if (input.rfind("//", 0) == 0 || input.rfind("!", 0) == 0 || input.empty()) continue;
      line.clear();
      line.str(input);
      type.clear();
      key.clear();
      temp.clear();
      line >> type;
      line >> key >> temp;
      if (type == "int") {
        int v{};
        line >> v;
        ints[key] = v;
      } else if (type == "real") {
        double v{};
        line >> v;
        reals[key] = v;
      } else if (type == "bool") {
        bool v{};
        line >> v;
        bools[key] = v;
      } else if (type == "string") {
        std::string v;
        line >> v;
        strings[key] = v;
      } else if (type == "array") {
        const std::string name = temp;
        line >> temp >> temp;  // "= {" or "{" plus the first value (reference behaviour)
        if (key == "int") {
          std::vector<int> a;
          read_array(f, input, line, a);
          int_arrays[name] = a;
        } else if (key == "real") {
          std::vector<double> a;
          read_array(f, input, line, a);
          real_arrays[name] = a;
        } else if (key == "string") {
          std::vector<std::string> a;
          read_array(f, input, line, a);
          string_arrays[name] = a;
        }
      } else if (type == "struct") {
        std::map<std::string, StructVal> st;
        while (true) {
          next_line(f, input, line);
          if (!f && input.empty()) break;
          std::string k2, name, eq;
          line >> k2;
          if (k2 == "}") break;
          if (k2 == "string") {
            std::string v;
            line >> name >> eq >> v;
            st.emplace(name, v);
          } else if (k2 == "int") {
            int v{};
            line >> name >> eq >> v;
            st.emplace(name, v);
          } else if (k2 == "real") {
            double v{};
            line >> name >> eq >> v;
            st.emplace(name, v);
          }
        }
        structs[key] = st;
      } else if (type == "range") {
        const std::string name = temp;
        line >> temp >> temp;
        if (key == "real") {
          std::vector<double> a;
          read_array(f, input, line, a);
          if (a.size() != 2 && a.size() != 4 && a.size() != 6) {
            err = "range " + name + ": expected 2, 4 or 6 values";
            return false;
          }
          real_ranges[name] = a;
        } else if (key == "int") {
          std::vector<int> a;
          read_array(f, input, line, a);
          if (a.size() != 2 && a.size() != 4 && a.size() != 6) {
            err = "range " + name + ": expected 2, 4 or 6 values";
            return false;
          }
          int_ranges[name] = a;
        }
      }
    }
  } catch (const std::exception &e) {
    err = std::string("setup parse error: ") + e.what();
    return false;
  }
  return true;
}

int Setup::get_int(const std::string &k) const {
  auto it = ints.find(k);
  return it == ints.end() ? 0 : it->second;
}
double Setup::get_real(const std::string &k) const {
  auto it = reals.find(k);
  return it == reals.end() ? 0.0 : it->second;
}
bool Setup::get_bool(const std::string &k) const {
  auto it = bools.find(k);
  return it == bools.end() ? false : it->second;
}

bool derive(const Setup &s, Derived &d, std::string &err) {
  d.reconstruction = s.get_int("reconstruction");
  d.inviscid_scheme = s.get_int("inviscid_scheme");
  d.viscous_order = s.get_int("viscous_order");
  // ghost layers (Parameter.cpp:194-242)
  int ngg = 2;
  if (d.reconstruction == 4) ngg = 3;
  else if (d.reconstruction == 5) ngg = 4;
  const int is = d.inviscid_scheme;
  if (is == 51 || is == 52 || is == 6) ngg = 3;
  if (is == 71 || is == 72) ngg = 4;
  d.ngg = ngg;
  // inviscid_type (Parameter.cpp:264-278)
  int it = 0;
  if (is == 2) it = 2;
  if (d.reconstruction == 4 || d.reconstruction == 5) it = 1;
  if (is == 51 || is == 52 || is == 71 || is == 72) it = 3;
  if (is == 6) it = 4;
  d.inviscid_type = it;
  d.steady = s.get_bool("steady");
  d.temporal_scheme = s.get_int("temporal_scheme");
  d.fixed_time_step = s.get_bool("fixed_time_step");
  d.dt = s.get_real("dt");
  d.cfl = s.get_real("cfl");
  d.prandtl = s.get_real("prandtl_number");
  d.grid_scale = s.get_real("gridScale");
  d.species = s.get_int("species");
  d.n_spec = 0;
  d.n_scalar = 0;
  d.n_var = 5;
  d.reaction = s.get_int("reaction");
  d.problem_type = s.get_int("problem_type");
  if (d.problem_type != 0 && d.problem_type != 1) {
    err = "problem_type must be 0 (general) or 1 (mixing layer); got " + std::to_string(d.problem_type);
    return false;
  }
  if (d.problem_type == 1 && s.get_bool("compatible_mixing_layer")) {
    err = "compatible_mixing_layer = 1 (inflow and initial field from a profile file) is not provided";
    return false;
  }
  if (d.species != 0 && d.species != 1) {
    err = "species = " + std::to_string(d.species) + " (mixture-fraction / flamelet models) is not on this library's path";
    return false;
  }
  if (d.species == 1 && d.reaction != 0 && d.reaction != 1) {
    err = "reaction = " + std::to_string(d.reaction) + " (flamelet) is not on this library's path";
    return false;
  }
  if (s.get_bool("turbulence")) {
    err = "turbulence models are outside this library's path (laminar/DNS only)";
    return false;
  }
  if (!d.steady && d.temporal_scheme != 3 && d.temporal_scheme != 2) {
    err = "temporal_scheme " + std::to_string(d.temporal_scheme) +
          ": of the unsteady drivers this library runs SSP-RK3 (3) and dual time stepping (2); steady = 1 runs "
          "the steady driver";
    return false;
  }
  // steady driver settings (Parameter.cpp:449-451, 280-283): the implicit operator, its inner
  // iterations and the treatment of the chemical source; RK3 treats the source explicitly
  d.implicit_method = s.get_int("implicit_method");
  d.dplur_inner = s.get_int("DPLUR_inner_step");
  d.chem_src_method = s.get_int("chemSrcMethod");
  d.convergence_criteria = s.get_real("convergence_criteria");
  d.output_screen = s.get_int("output_screen");
  d.inner_iteration = s.get_int("inner_iteration");
  d.max_inner_iteration = s.get_int("max_inner_iteration");
  d.iteration_adjust_step = s.get_int("iteration_adjust_step");
  if (!d.steady && d.temporal_scheme == 3) d.chem_src_method = 0;
  if (d.implicit_method != 0 && d.implicit_method != 1) {
    err = "implicit_method must be 0 (explicit) or 1 (DPLUR); got " + std::to_string(d.implicit_method);
    return false;
  }
  if (d.chem_src_method < 0 || d.chem_src_method > 2) {
    err = "chemSrcMethod must be 0 (explicit), 1 (EPI) or 2 (DA); got " + std::to_string(d.chem_src_method);
    return false;
  }
  if (d.dplur_inner < 0) {
    err = "DPLUR_inner_step must not be negative";
    return false;
  }
  if (d.inviscid_type == 4) {
    err = "inviscid_scheme 6 (energy-preserving) is not on this library's path";
    return false;
  }
  if (d.inviscid_type == 3 && is != 71 && !(is == 72 && d.species == 1)) {
    // 51 / 52 stencils read outside the loaded points for the first face of every tile
    // (WENO.cu:855-856: i_shared - 3 with ngg = 3), and 72 for air runs a 5x5 loop over 7 rows
    // (WENO.cu:1319-1328): neither defines a result to match
    err = "inviscid_scheme " + std::to_string(is) + (d.species ? "" : " for air") +
          " is not supported (reference reads outside its stencil); use 71 or, for mixtures, 72";
    return false;
  }
  if (d.species == 1 && d.inviscid_type == 1) {
    // the reference's mixture AWENO_interpolation and CDSPart1D are empty stubs (AWENO.cu:8-13, 282-285)
    err = "AWENO (reconstruction 4 / 5) is not defined for mixtures in the reference; use the flux-split WENO "
          "(inviscid_scheme 71 / 72) or a primitive reconstruction (1-3) with AUSM+, HLLC or Roe";
    return false;
  }
  if (d.species == 1 && (d.inviscid_type == 0 || d.inviscid_type == 2) && is == 1) {
    err = "Lax-Friedrichs (inviscid_scheme 1) has no mixture form in the reference (riemannSolver_laxFriedrich<mixture> "
          "only prints, RiemannSolver.cuh:419-424); use AUSM+ (3), HLLC (4) or Roe (2)";
    return false;
  }
  if (d.inviscid_type == 0 || d.inviscid_type == 2) {
    // primitive reconstruction (Reconstruction.cu:5-45): 1 first order, 2 MUSCL, 3 NND2
    if (d.reconstruction < 1 || d.reconstruction > 3) {
      err = "reconstruction must be 1 (1st order), 2 (MUSCL), 3 (NND2), 4 (AWENO5) or 5 (AWENO7); got " +
            std::to_string(d.reconstruction);
      return false;
    }
  }
  d.limiter = s.get_int("limiter");
  if (d.limiter != 0 && d.limiter != 1) {
    // apply_limiter<0, 1> has no case for other values (Limiter.cuh:24-41) and returns an undefined value
    err = "limiter must be 0 or 1 (minmod); got " + std::to_string(d.limiter);
    return false;
  }
  d.entropy_fix_factor = s.get_real("entropy_fix_factor");
  if (d.inviscid_type == 2) d.riemann = 2;
  else if (is == 1) d.riemann = 1;
  else if (is == 4) d.riemann = 4;
  else d.riemann = 3;
  if (d.viscous_order != 0 && d.viscous_order != 2) {
    err = "viscous_order must be 0 or 2";
    return false;
  }
  if (s.get_bool("limit_flow") || s.get_bool("sponge_layer")) {
    err = "limit_flow / sponge_layer are not on this library's path";
    return false;
  }
  if (s.get_int("n_ps") != 0) {
    err = "passive scalars (n_ps) are not on this library's path";
    return false;
  }
  return true;
}

// ------------------------------------------------------------------------------------ mesh

namespace {

// Boundary::register_boundary (Mesh.cpp:14-32)
void register_boundary(BcFace &b, int ngg, int dim) {
  b.face = 0;
  b.direction = 1;
  for (int i = 0; i < dim; ++i) {
    if (b.rs[i] == b.re[i]) {
      b.face = i;
      if (b.rs[i] == 0) b.direction = -1;
      break;
    }
  }
  for (int i = 0; i < dim; ++i) {
    if (i == b.face) continue;
    if (b.re[i] < b.rs[i]) std::swap(b.re[i], b.rs[i]);
    b.rs[i] -= ngg;
    b.re[i] += ngg;
  }
  if (dim == 2) {
    b.rs[2] = -ngg;
    b.re[2] = ngg;
  }
}

// Face layers of the ghost grid by point reflection (Mesh.cpp:893-960).
void ghost_grid(HostBlock &B, int dimension) {
  const int mx = B.mx, my = B.my, mz = B.mz, ngg = B.ngg;
  std::array<std::vector<double> *, 3> C{&B.x, &B.y, &B.z};
  auto at = [&](int q, int i, int j, int k) -> double & { return (*C[q])[B.cidx(i, j, k)]; };
  for (int q = 0; q < 3; ++q)
    for (int k = 0; k < mz; ++k)
      for (int j = 0; j < my; ++j) {
        for (int i = -1; i >= -ngg - 1; --i) at(q, i, j, k) = 2 * at(q, 0, j, k) - at(q, -i, j, k);
        for (int i = mx; i < mx + ngg + 1; ++i) at(q, i, j, k) = 2 * at(q, mx - 1, j, k) - at(q, 2 * (mx - 1) - i, j, k);
      }
  for (int q = 0; q < 3; ++q)
    for (int k = 0; k < mz; ++k)
      for (int i = 0; i < mx; ++i) {
        for (int j = -1; j >= -ngg - 1; --j) at(q, i, j, k) = 2 * at(q, i, 0, k) - at(q, i, -j, k);
        for (int j = my; j < my + ngg + 1; ++j) at(q, i, j, k) = 2 * at(q, i, my - 1, k) - at(q, i, 2 * (my - 1) - j, k);
      }
  if (dimension == 3) {
    for (int q = 0; q < 3; ++q)
      for (int j = 0; j < my; ++j)
        for (int i = 0; i < mx; ++i) {
          for (int k = -1; k >= -ngg - 1; --k) at(q, i, j, k) = 2 * at(q, i, j, 0) - at(q, i, j, -k);
          for (int k = mz; k < mz + ngg + 1; ++k) at(q, i, j, k) = 2 * at(q, i, j, mz - 1) - at(q, i, j, 2 * (mz - 1) - k);
        }
  } else {
    for (int j = 0; j < my; ++j)
      for (int i = 0; i < mx; ++i) {
        for (int k = -1; k >= -ngg - 1; --k) {
          at(0, i, j, k) = at(0, i, j, 0);
          at(1, i, j, k) = at(1, i, j, 0);
          at(2, i, j, k) = at(2, i, j, 0) + k;
        }
        for (int k = mz; k < mz + ngg + 1; ++k) {
          at(0, i, j, k) = at(0, i, j, mz - 1);
          at(1, i, j, k) = at(1, i, j, mz - 1);
          at(2, i, j, k) = at(2, i, j, mz - 1) + k - mz + 1;
        }
      }
  }
}

// Edges and corners of the ghost grid by the parallelogram rule (Mesh.cpp:968-1041), after the face
// layers and the interface layers are in place.
void ghost_grid_edges(HostBlock &B) {
  const int mx = B.mx, my = B.my, mz = B.mz, ngg = B.ngg;
  std::array<std::vector<double> *, 3> C{&B.x, &B.y, &B.z};
  auto at = [&](int q, int i, int j, int k) -> double & { return (*C[q])[B.cidx(i, j, k)]; };
  for (int i = 1; i <= ngg + 1; ++i)
    for (int j = 1; j <= ngg + 1; ++j)
      for (int k = 0; k < mz; ++k) {
        const int i1 = -i, j1 = -j, i2 = mx - 1 + i, j2 = my - 1 + j;
        for (int q = 0; q < 3; ++q) {
          at(q, i1, j1, k) = at(q, i1, 0, k) + at(q, 0, j1, k) - at(q, 0, 0, k);
          at(q, i2, j2, k) = at(q, i2, my - 1, k) + at(q, mx - 1, j2, k) - at(q, mx - 1, my - 1, k);
          at(q, i1, j2, k) = at(q, i1, my - 1, k) + at(q, 0, j2, k) - at(q, 0, my - 1, k);
          at(q, i2, j1, k) = at(q, i2, 0, k) + at(q, mx - 1, j1, k) - at(q, mx - 1, 0, k);
        }
      }
  for (int i = 1; i <= ngg + 1; ++i)
    for (int j = 0; j < my; ++j)
      for (int k = 1; k <= ngg + 1; ++k) {
        const int i1 = -i, k1 = -k, i2 = mx - 1 + i, k2 = mz - 1 + k;
        for (int q = 0; q < 3; ++q) {
          at(q, i1, j, k1) = at(q, i1, j, 0) + at(q, 0, j, k1) - at(q, 0, j, 0);
          at(q, i2, j, k2) = at(q, i2, j, mz - 1) + at(q, mx - 1, j, k2) - at(q, mx - 1, j, mz - 1);
          at(q, i1, j, k2) = at(q, i1, j, mz - 1) + at(q, 0, j, k2) - at(q, 0, j, mz - 1);
          at(q, i2, j, k1) = at(q, i2, j, 0) + at(q, mx - 1, j, k1) - at(q, mx - 1, j, 0);
        }
      }
  for (int i = -ngg - 1; i <= mx + ngg; ++i)
    for (int j = 1; j <= ngg + 1; ++j)
      for (int k = 1; k <= ngg + 1; ++k) {
        const int j1 = -j, k1 = -k, j2 = my - 1 + j, k2 = mz - 1 + k;
        for (int q = 0; q < 3; ++q) {
          at(q, i, j1, k1) = at(q, i, j1, 0) + at(q, i, 0, k1) - at(q, i, 0, 0);
          at(q, i, j2, k2) = at(q, i, j2, mz - 1) + at(q, i, my - 1, k2) - at(q, i, my - 1, mz - 1);
          at(q, i, j1, k2) = at(q, i, j1, mz - 1) + at(q, i, 0, k2) - at(q, i, 0, mz - 1);
          at(q, i, j2, k1) = at(q, i, j2, 0) + at(q, i, my - 1, k1) - at(q, i, my - 1, 0);
        }
      }
}

// One node of Block::compute_jac_metric (Mesh.cpp:241-503)
void metric_node(HostBlock &B, int i, int j, int k, int fi, int fj, int fk) {
  auto X = [&](int a, int b, int c) { return B.x[B.cidx(a, b, c)]; };
  auto Y = [&](int a, int b, int c) { return B.y[B.cidx(a, b, c)]; };
  auto Z = [&](int a, int b, int c) { return B.z[B.cidx(a, b, c)]; };
  const double dxd1 = (X(i + 1, j, k) - X(i - 1, j, k)) * 0.5, dyd1 = (Y(i + 1, j, k) - Y(i - 1, j, k)) * 0.5,
               dzd1 = (Z(i + 1, j, k) - Z(i - 1, j, k)) * 0.5;
  const double dxd2 = (X(i, j + 1, k) - X(i, j - 1, k)) * 0.5, dyd2 = (Y(i, j + 1, k) - Y(i, j - 1, k)) * 0.5,
               dzd2 = (Z(i, j + 1, k) - Z(i, j - 1, k)) * 0.5;
  const double dxd3 = (X(i, j, k + 1) - X(i, j, k - 1)) * 0.5, dyd3 = (Y(i, j, k + 1) - Y(i, j, k - 1)) * 0.5,
               dzd3 = (Z(i, j, k + 1) - Z(i, j, k - 1)) * 0.5;
  const double jac = dxd1 * dyd2 * dzd3 + dxd2 * dyd3 * dzd1 + dxd3 * dyd1 * dzd2 - dxd1 * dyd3 * dzd2 -
                     dxd2 * dyd1 * dzd3 - dxd3 * dyd2 * dzd1;
  const long P = B.padded(), p = B.gidx(i, j, k);
  if (jac <= 0) {
    const long q = B.gidx(fi, fj, fk);
    B.jac[p] = B.jac[q];
    for (int r = 0; r < 9; ++r) B.metric[r * P + p] = B.metric[r * P + q];
    return;
  }
  B.jac[p] = jac;
  double *m = B.metric.data();
  m[0 * P + p] = (dyd2 * dzd3 - dyd3 * dzd2) / jac;
  m[1 * P + p] = (dxd3 * dzd2 - dxd2 * dzd3) / jac;
  m[2 * P + p] = (dxd2 * dyd3 - dxd3 * dyd2) / jac;
  m[3 * P + p] = (dyd3 * dzd1 - dyd1 * dzd3) / jac;
  m[4 * P + p] = (dxd1 * dzd3 - dxd3 * dzd1) / jac;
  m[5 * P + p] = (dxd3 * dyd1 - dxd1 * dyd3) / jac;
  m[6 * P + p] = (dyd1 * dzd2 - dyd2 * dzd1) / jac;
  m[7 * P + p] = (dxd2 * dzd1 - dxd1 * dzd2) / jac;
  m[8 * P + p] = (dxd1 * dyd2 - dxd2 * dyd1) / jac;
}

void compute_jac_metric(HostBlock &B) {
  const int mx = B.mx, my = B.my, mz = B.mz, ngg = B.ngg;
  for (int i = 1; i < mx - 1; ++i)
    for (int j = 1; j < my - 1; ++j) {
      int k0 = 1, k1 = mz - 1;
      if (mz == 1) {
        k0 = 0;
        k1 = 1;
      }
      for (int k = k0; k < k1; ++k) metric_node(B, i, j, k, i, j, k);
    }
  for (int i = 1; i < mx - 1; ++i)
    for (int j = 1; j < my - 1; ++j)
      for (int k = 0; k >= -ngg; --k) metric_node(B, i, j, k, i, j, k + 1);
  for (int i = 1; i < mx - 1; ++i)
    for (int j = 1; j < my - 1; ++j)
      for (int k = mz - 1; k < mz + ngg; ++k) metric_node(B, i, j, k, i, j, k - 1);
  for (int i = 1; i < mx - 1; ++i)
    for (int j = 0; j >= -ngg; --j)
      for (int k = -ngg; k < mz + ngg; ++k) metric_node(B, i, j, k, i, j + 1, k);
  for (int i = 1; i < mx - 1; ++i)
    for (int j = my - 1; j < my + ngg; ++j)
      for (int k = -ngg; k < mz + ngg; ++k) metric_node(B, i, j, k, i, j - 1, k);
  for (int i = 0; i >= -ngg; --i)
    for (int j = -ngg; j < my + ngg; ++j)
      for (int k = -ngg; k < mz + ngg; ++k) metric_node(B, i, j, k, i + 1, j, k);
  for (int i = mx - 1; i < mx + ngg; ++i)
    for (int j = -ngg; j < my + ngg; ++j)
      for (int k = -ngg; k < mz + ngg; ++k) metric_node(B, i, j, k, i - 1, j, k);
}

}  // namespace

namespace {
int sgn(int a) { return a < 0 ? -1 : 1; }  // gxl::sgn: sgn(0) = +1 (gxl_lib/Math.hpp:13-15)

// InnerFace::register_boundary (Mesh.cpp:38-141).  Input: the two 1-based index ranges of the file,
// signs marking the first tangential direction (3-D); output: the written range (face + ngg ghost
// layers, tangential extent of the face), the target start, the index map and loop directions.
void register_inner(InnerFace &f, int ngg, int dim) {
  for (int i = 0; i < dim; ++i)
    if (f.rs[i] == f.re[i]) {
      f.face = i;
      if (f.rs[i] == 1) f.direction = -1;
      f.rs[i] -= 1;
      f.re[i] -= 1;
      break;
    }
  for (int i = 0; i < dim; ++i)
    if (f.ts[i] == f.te[i]) {
      f.target_face = i;
      if (f.ts[i] == 1) f.target_direction = -1;
      f.ts[i] -= 1;
      f.te[i] -= 1;
      break;
    }
  f.src_tar[f.target_face] = -(f.direction * f.target_direction) * (f.face + 1);
  if (dim == 2) {
    const int nf = 1 - f.face, tnf = 1 - f.target_face;
    f.rs[nf] = std::abs(f.rs[nf]) - 1;
    f.re[nf] = std::abs(f.re[nf]) - 1;
    f.ts[tnf] = std::abs(f.ts[tnf]) - 1;
    f.te[tnf] = std::abs(f.te[tnf]) - 1;
    f.src_tar[tnf] = sgn((f.te[tnf] - f.ts[tnf]) * (f.re[nf] - f.rs[nf])) * (nf + 1);
    f.src_tar[2] = 3;
    f.rs[2] = f.re[2] = f.ts[2] = f.te[2] = 0;
  } else {
    int nf = 0, tnf = 0;
    for (int i = 0; i < dim; ++i)
      if (f.rs[i] < 0) {
        nf = i;
        f.rs[i] = -f.rs[i] - 1;
        f.re[i] = -f.re[i] - 1;
        break;
      }
    for (int i = 0; i < dim; ++i)
      if (f.ts[i] < 0) {
        tnf = i;
        f.ts[i] = -f.ts[i] - 1;
        f.te[i] = -f.te[i] - 1;
        break;
      }
    f.src_tar[tnf] = sgn((f.te[tnf] - f.ts[tnf]) * (f.re[nf] - f.rs[nf])) * (nf + 1);
    nf = 3 - f.face - nf;
    tnf = 3 - f.target_face - tnf;
    f.rs[nf] -= 1;
    f.re[nf] -= 1;
    f.ts[tnf] -= 1;
    f.te[tnf] -= 1;
    f.src_tar[tnf] = sgn((f.te[tnf] - f.ts[tnf]) * (f.re[nf] - f.rs[nf])) * (nf + 1);
  }
  f.rs[f.face] = f.direction < 0 ? -ngg : f.re[f.face];
  f.re[f.face] = f.direction < 0 ? 0 : f.re[f.face] + ngg;
  const int st = sgn(f.src_tar[f.target_face]);
  if (f.target_direction > 0) f.ts[f.target_face] = st > 0 ? f.te[f.target_face] - ngg : f.te[f.target_face];
  else f.ts[f.target_face] = st > 0 ? 0 : ngg;
  for (int i = 0; i < 3; ++i) {
    f.loop_dir[i] = f.rs[i] <= f.re[i] ? 1 : -1;
    f.target_loop_dir[i] = sgn(f.src_tar[i]);
    f.src_tar[i] = std::abs(f.src_tar[i]) - 1;
  }
  for (int i = 0; i < 3; ++i) f.n_point[i] = std::abs(f.rs[i] - f.re[i]) + 1;
}

// Mesh::init_inner_ghost_grid (Mesh.cpp:1049-1097): ghost coordinates across an interface are the
// neighbour's interior coordinates (ngg + 1 layers).
void inner_ghost_grid(HostMesh &mesh) {
  for (auto &B : mesh.blocks)
    for (const auto &fc : B.inner) {
      HostBlock &nB = mesh.blocks[fc.target_block];
      int mn[3] = {fc.rs[0], fc.rs[1], fc.rs[2]}, mx_[3] = {fc.re[0], fc.re[1], fc.re[2]};
      int mt[3] = {fc.ts[0], fc.ts[1], fc.ts[2]};
      if (fc.direction < 0) {
        mn[fc.face] -= 1;
        mx_[fc.face] -= 1;
      } else {
        mn[fc.face] += 1;
        mx_[fc.face] += 1;
      }
      mt[fc.target_face] += fc.target_direction > 0 ? -1 : 1;
      const int d1[3] = {fc.loop_dir[0], fc.loop_dir[1], fc.loop_dir[2]};
      int di[3];
      for (int i1 = mn[0]; d1[0] * (i1 - mx_[0]) != 1; i1 += d1[0]) {
        di[0] = i1 - mn[0];
        for (int j1 = mn[1]; d1[1] * (j1 - mx_[1]) != 1; j1 += d1[1]) {
          di[1] = j1 - mn[1];
          for (int k1 = mn[2]; d1[2] * (k1 - mx_[2]) != 1; k1 += d1[2]) {
            di[2] = k1 - mn[2];
            const int i2 = mt[0] + fc.target_loop_dir[0] * di[fc.src_tar[0]];
            const int j2 = mt[1] + fc.target_loop_dir[1] * di[fc.src_tar[1]];
            const int k2 = mt[2] + fc.target_loop_dir[2] * di[fc.src_tar[2]];
            B.x[B.cidx(i1, j1, k1)] = nB.x[nB.cidx(i2, j2, k2)];
            B.y[B.cidx(i1, j1, k1)] = nB.y[nB.cidx(i2, j2, k2)];
            B.z[B.cidx(i1, j1, k1)] = nB.z[nB.cidx(i2, j2, k2)];
          }
        }
      }
    }
}
}  // namespace

bool read_mesh(const std::string &dir, const Derived &d, HostMesh &mesh, std::string &err) {
  const std::string gpath = dir + "/grid/grid   0.dat";
  FILE *fp = std::fopen(gpath.c_str(), "rb");
  if (!fp) {
    err = "cannot open grid file " + gpath + " (binary grid, gridIsBinary = 1, is expected)";
    return false;
  }
  int nblk = 0;
  if (std::fread(&nblk, sizeof(int), 1, fp) != 1 || nblk <= 0 || nblk > 4096) {
    std::fclose(fp);
    err = "grid file: bad block count";
    return false;
  }
  mesh.blocks.assign(nblk, HostBlock{});
  for (auto &B : mesh.blocks) {
    int dims[3];
    if (std::fread(dims, sizeof(int), 3, fp) != 3 || dims[0] < 2 || dims[1] < 2 || dims[2] < 1) {
      std::fclose(fp);
      err = "grid file: bad block dimensions";
      return false;
    }
    B.mx = dims[0];
    B.my = dims[1];
    B.mz = dims[2];
    B.ngg = d.ngg;
  }
  mesh.dimension = mesh.blocks[0].mz == 1 ? 2 : 3;
  for (auto &B : mesh.blocks) {
    const int g = B.ngg + 1;
    const long n = (long)(B.mx + 2 * g) * (B.my + 2 * g) * (B.mz + 2 * g);
    B.x.assign(n, 0.0);
    B.y.assign(n, 0.0);
    B.z.assign(n, 0.0);
    const long N = (long)B.mx * B.my * B.mz;
    std::vector<double> buf(N);
    std::vector<double> *dst[3] = {&B.x, &B.y, &B.z};
    for (int q = 0; q < 3; ++q) {
      if (std::fread(buf.data(), sizeof(double), N, fp) != (size_t)N) {
        std::fclose(fp);
        err = "grid file: truncated coordinates";
        return false;
      }
      for (int k = 0; k < B.mz; ++k)
        for (int j = 0; j < B.my; ++j)
          for (int i = 0; i < B.mx; ++i) (*dst[q])[B.cidx(i, j, k)] = buf[((long)k * B.my + j) * B.mx + i];
    }
  }
  std::fclose(fp);

  // boundary file (Mesh.cpp:790-810)
  {
    const std::string bpath = dir + "/boundary_condition/boundary   0.txt";
    std::ifstream bf(bpath);
    if (!bf) {
      err = "cannot open " + bpath;
      return false;
    }
    std::string input;
    for (auto &B : mesh.blocks) {
      if (!std::getline(bf, input)) {
        err = "boundary file: missing face count";
        return false;
      }
      const int n = std::stoi(input);
      for (int f = 0; f < n; ++f) {
        std::getline(bf, input);
        std::istringstream line(input);
        BcFace b;
        line >> b.rs[0] >> b.re[0] >> b.rs[1] >> b.re[1] >> b.rs[2] >> b.re[2] >> b.label;
        if (!line) {
          err = "boundary file: malformed face line";
          return false;
        }
        // every device access of a face kernel derives from these ranges: reject anything that
        // is not a whole-face or sub-face range of this block's nodes
        const int ext[3] = {B.mx, B.my, B.mz};
        bool ok = false;
        for (int q = 0; q < mesh.dimension; ++q) {
          const int lo = std::min(b.rs[q], b.re[q]), hi = std::max(b.rs[q], b.re[q]);
          if (lo < 0 || hi > ext[q] - 1) {
            err = "boundary file: face range outside the block";
            return false;
          }
          if (b.rs[q] == b.re[q] && (b.rs[q] == 0 || b.rs[q] == ext[q] - 1)) ok = true;
        }
        if (!ok || (mesh.dimension == 2 && (b.rs[2] != 0 || b.re[2] != 0))) {
          err = "boundary file: a face must lie on a block side (one index fixed at 0 or m-1)";
          return false;
        }
        for (int q = 0; q < 3; ++q)
          if (ext[q] <= B.ngg + 1 && !(mesh.dimension == 2 && q == 2)) {
            err = "block too small for the stencil (every extent must exceed ngg + 1)";
            return false;
          }
        register_boundary(b, B.ngg, mesh.dimension);
        B.faces.push_back(b);
      }
    }
  }
  // inner-face file (Mesh.cpp:812-844)
  {
    const std::string ipath = dir + "/boundary_condition/inner   0.txt";
    std::ifstream inf(ipath);
    if (inf) {
      // Mesh::read_inner_interface (Mesh.cpp:812-844): a header line, the face count of every block,
      // a column-title line, then per face two lines: this block's 1-based range and the target's
      // range followed by the target block id.
      std::string input;
      std::getline(inf, input);
      std::vector<int> nface(mesh.blocks.size(), 0);
      for (auto &n : nface) inf >> n;
      std::getline(inf, input);
      std::getline(inf, input);
      const int nb = (int)mesh.blocks.size();
      for (int b = 0; b < nb; ++b) {
        HostBlock &B = mesh.blocks[b];
        for (int l = 0; l < nface[b]; ++l) {
          InnerFace f;
          int i7 = 0, j7 = 0;
          std::getline(inf, input);
          std::istringstream l1(input);
          l1 >> f.rs[0] >> f.re[0] >> f.rs[1] >> f.re[1] >> f.rs[2] >> f.re[2] >> i7;
          std::getline(inf, input);
          std::istringstream l2(input);
          l2 >> f.ts[0] >> f.te[0] >> f.ts[1] >> f.te[1] >> f.ts[2] >> f.te[2] >> j7;
          if (!l1 || !l2 || j7 < 1 || j7 > nb) {
            err = "inner face file: malformed face of block " + std::to_string(b + 1);
            return false;
          }
          f.target_block = j7 - 1;
          register_inner(f, B.ngg, mesh.dimension);
          // every device index of the exchange derives from these ranges: check them against both blocks
          const HostBlock &T = mesh.blocks[f.target_block];
          const int ext[3] = {B.mx, B.my, B.mz}, text[3] = {T.mx, T.my, T.mz};
          bool ok = true;
          for (int q = 0; q < 3; ++q) {
            const int lo = std::min(f.rs[q], f.re[q]), hi = std::max(f.rs[q], f.re[q]);
            const int g = q == f.face ? B.ngg : 0;
            if (lo < -g || hi > ext[q] - 1 + g) ok = false;
          }
          for (int q = 0; q < 3 && ok; ++q) {
            // the target index of the last point along each source axis
            const int dmax = f.n_point[f.src_tar[q]] - 1;
            const int a = f.ts[q], bq = f.ts[q] + f.target_loop_dir[q] * f.loop_dir[f.src_tar[q]] * dmax;
            if (std::min(a, bq) < 0 || std::max(a, bq) > text[q] - 1) ok = false;
          }
          if (!ok) {
            err = "inner face file: interface " + std::to_string(l + 1) + " of block " + std::to_string(b + 1) +
                  " reaches outside a block";
            return false;
          }
          B.inner.push_back(f);
        }
      }
    }
  }
  // scale (Mesh.cpp:613-619, 877-891)
  if (std::abs(d.grid_scale - 1.0) > 1e-15) {
    for (auto &B : mesh.blocks) {
      for (auto &v : B.x) v *= d.grid_scale;
      for (auto &v : B.y) v *= d.grid_scale;
      for (auto &v : B.z) v *= d.grid_scale;
    }
  }
  for (auto &B : mesh.blocks) ghost_grid(B, mesh.dimension);
  inner_ghost_grid(mesh);
  for (auto &B : mesh.blocks) {
    ghost_grid_edges(B);
    B.jac.assign(B.padded(), 0.0);
    B.metric.assign(9 * B.padded(), 0.0);
    compute_jac_metric(B);
    for (int k = 0; k < B.mz; ++k)
      for (int j = 0; j < B.my; ++j)
        for (int i = 0; i < B.mx; ++i)
          if (!(B.jac[B.gidx(i, j, k)] > 0)) {
            err = "negative Jacobian at interior node (" + std::to_string(i) + "," + std::to_string(j) + "," +
                  std::to_string(k) + ")";
            return false;
          }
  }
  return true;
}

namespace {
double struct_real(const std::map<std::string, Setup::StructVal> &st, const char *k, double def) {
  auto it = st.find(k);
  if (it == st.end()) return def;
  if (auto p = std::get_if<double>(&it->second)) return *p;
  if (auto q = std::get_if<int>(&it->second)) return *q;
  return def;
}
double sutherland_host(double t) { return 1.7894e-5 * std::pow(t / 288.16, 1.5) * (288.16 + 110) / (t + 110); }

// Species::compute_cp (ChemData.cpp:126-149): mass-specific cp of every species, frozen at t_low below it
void species_cp(const ChemTables &chem, double t, double *cp) {
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t;
  for (int i = 0; i < chem.n_spec; ++i) {
    double cc;
    if (t < chem.t_low[i]) {
      const double tt = chem.t_low[i], tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt;
      const double *a = &chem.low[i * 7];
      cc = a[0] + a[1] * tt + a[2] * tt2 + a[3] * tt3 + a[4] * tt4;
    } else {
      const double *a = t < chem.t_mid[i] ? &chem.low[i * 7] : &chem.high[i * 7];
      cc = a[0] + a[1] * t + a[2] * t2 + a[3] * t3 + a[4] * t4;
    }
    cp[i] = cc * (kRu / chem.mw[i]);
  }
}
}  // namespace

// State of a plain inflow struct (Inflow::Inflow, BoundCond.cpp:157-214): density from p, T and the
// mixture weight, velocity = Mach * c along (u, v, w).  Returns false with err set when the struct
// lacks mach, pressure or temperature.
bool inflow_state(const Setup &s, const std::string &name, const ChemTables *chem, double bv[6],
                  std::vector<double> &y, double &c, std::string &err, double *gamma_out) {
  auto it = s.structs.find(name);
  if (it == s.structs.end()) {
    err = "struct '" + name + "' is not defined in the setup";
    return false;
  }
  const auto &st = it->second;
  const double mach = struct_real(st, "mach", -1), pressure = struct_real(st, "pressure", -1);
  const double temperature = struct_real(st, "temperature", -1);
  if (mach < 0 || pressure < 0 || temperature < 0) {
    err = "struct '" + name + "' needs mach, pressure and temperature on this path";
    return false;
  }
  double mw = kMwAir, gamma = kGammaAir;
  y.clear();
  if (chem && chem->n_spec > 0) {
    y.assign(chem->n_spec, 0.0);
    std::vector<double> cp(chem->n_spec);
    for (int i = 0; i < chem->n_spec; ++i) y[i] = struct_real(st, chem->names[i].c_str(), 0.0);
    mw = 0;
    for (int i = 0; i < chem->n_spec; ++i) mw += y[i] / chem->mw[i];
    mw = 1 / mw;
    for (int i = 0; i < chem->n_spec; ++i) cp[i] = 0;
    species_cp(*chem, temperature, cp.data());
    double cpt = 0, cvt = 0;
    for (int i = 0; i < chem->n_spec; ++i) {
      cpt += y[i] * cp[i];
      cvt += y[i] * (cp[i] - kRu / chem->mw[i]);
    }
    gamma = cpt / cvt;
  }
  c = std::sqrt(gamma * kRu / mw * temperature);
  if (gamma_out) *gamma_out = gamma;
  const double velocity = mach * c;
  bv[0] = pressure * mw / (kRu * temperature);
  bv[1] = struct_real(st, "u", 1.0) * velocity;
  bv[2] = struct_real(st, "v", 0.0) * velocity;
  bv[3] = struct_real(st, "w", 0.0) * velocity;
  bv[4] = pressure;
  bv[5] = temperature;
  return true;
}

bool mixing_layer_streams(const Setup &s, const ChemTables *chem, MixingLayerStreams &m, std::string &err) {
  auto up = s.structs.find("upper_stream"), lo = s.structs.find("lower_stream");
  if (up == s.structs.end() || lo == s.structs.end()) {
    err = "a mixing-layer problem (problem_type = 1) needs the structs upper_stream and lower_stream";
    return false;
  }
  for (const char *k : {"ma_c", "velocity_ratio", "delta_omega"})
    if (!s.reals.count(k)) {
      err = std::string("a mixing-layer problem (problem_type = 1) needs the real ") + k;
      return false;
    }
  const auto &U = up->second, &L = lo->second;
  for (const auto *st : {&U, &L})
    for (const char *k : {"temperature", "pressure"})
      if (!st->count(k)) {
        err = std::string("upper_stream / lower_stream need ") + k;
        return false;
      }
  const double ma_c = s.get_real("ma_c"), vel_ratio = s.get_real("velocity_ratio");
  const bool upper_faster = s.get_bool("upper_faster");
  double ma_upper = struct_real(U, "mach", -1), ma_lower = struct_real(L, "mach", -1);
  const double t_upper = struct_real(U, "temperature", 0), t_lower = struct_real(L, "temperature", 0);
  const double p_upper = struct_real(U, "pressure", 0), p_lower = struct_real(L, "pressure", 0);
  double rho_upper, rho_lower, c_upper, c_lower;
  const int ns = chem ? chem->n_spec : 0;
  m.y_upper.assign(ns, 0.0);
  m.y_lower.assign(ns, 0.0);
  if (ns > 0) {
    for (int i = 0; i < ns; ++i) {
      m.y_upper[i] = struct_real(U, chem->names[i].c_str(), 0.0);
      m.y_lower[i] = struct_real(L, chem->names[i].c_str(), 0.0);
    }
    std::vector<double> cpu(ns), cpl(ns);
    species_cp(*chem, t_upper, cpu.data());
    species_cp(*chem, t_lower, cpl.data());
    double mwi_u = 0, mwi_l = 0, cp_u = 0, cp_l = 0;
    for (int i = 0; i < ns; ++i) {
      mwi_u += m.y_upper[i] / chem->mw[i];
      mwi_l += m.y_lower[i] / chem->mw[i];
      cp_u += cpu[i] * m.y_upper[i];
      cp_l += cpl[i] * m.y_lower[i];
    }
    const double g_u = cp_u / (cp_u - kRu * mwi_u), g_l = cp_l / (cp_l - kRu * mwi_l);
    c_upper = std::sqrt(g_u * kRu * mwi_u * t_upper);
    c_lower = std::sqrt(g_l * kRu * mwi_l * t_lower);
    rho_upper = p_upper / (kRu * mwi_u * t_upper);
    rho_lower = p_lower / (kRu * mwi_l * t_lower);
  } else {
    c_upper = std::sqrt(kGammaAir * kRu / kMwAir * t_upper);
    c_lower = std::sqrt(kGammaAir * kRu / kMwAir * t_lower);
    rho_upper = p_upper * kMwAir / (kRu * t_upper);
    rho_lower = p_lower * kMwAir / (kRu * t_lower);
  }
  // the stream Mach numbers from the velocity ratio, or from one given Mach number and Ma_c
  if (vel_ratio > 0) {
    double u_slow, u_fast;
    if (vel_ratio > 1) {
      u_slow = ma_c * (c_upper + c_lower) / (vel_ratio - 1);
      u_fast = vel_ratio * u_slow;
    } else {
      u_fast = ma_c * (c_upper + c_lower) / (1 - vel_ratio);
      u_slow = u_fast * vel_ratio;
    }
    ma_upper = (upper_faster ? u_fast : u_slow) / c_upper;
    ma_lower = (upper_faster ? u_slow : u_fast) / c_lower;
  } else if (ma_upper < 0 && ma_lower < 0) {
    err = "a mixing-layer problem needs velocity_ratio > 0 or a stream Mach number";
    return false;
  } else if (ma_upper > 0 && ma_lower > 0) {
    // both given: the given streams are used as they are
  } else if (ma_upper > 0) {
    ma_lower = upper_faster ? (ma_upper - ma_c) * c_upper / c_lower - ma_c : (ma_c + ma_upper) * c_upper / c_lower + ma_c;
  } else {
    ma_upper = upper_faster ? (ma_c + ma_lower) * c_lower / c_upper + ma_c : (ma_lower - ma_c) * c_lower / c_upper - ma_c;
  }
  const double u_upper = ma_upper * c_upper, u_lower = ma_lower * c_lower;
  const double a[6] = {rho_upper, u_upper, 0, 0, p_upper, t_upper}, b[6] = {rho_lower, u_lower, 0, 0, p_lower, t_lower};
  for (int l = 0; l < 6; ++l) {
    m.upper[l] = a[l];
    m.lower[l] = b[l];
  }
  m.delta_omega = s.get_real("delta_omega");
  return true;
}

bool reference_scales(const Setup &s, const ChemTables *chem, double &eps_scale, double &v_ref, std::string &err) {
  eps_scale = 0;
  v_ref = 0;
  if (s.get_int("problem_type") == 1) {
    // a mixing-layer problem: the inflow struct named by reference_state carries the upper stream
    // (Inflow ctor, BoundCond.cpp:28-62, 299-305)
    MixingLayerStreams m;
    if (!mixing_layer_streams(s, chem, m, err)) return false;
    const double *u = m.upper;
    double vel = std::sqrt(u[1] * u[1] + u[2] * u[2] + u[3] * u[3]);
    if (std::abs(vel) < 1) {
      double mw = kMwAir, gamma = kGammaAir;
      if (chem && chem->n_spec > 0) {
        std::vector<double> cp(chem->n_spec);
        species_cp(*chem, u[5], cp.data());
        double mwi = 0, cpt = 0, cvt = 0;
        for (int i = 0; i < chem->n_spec; ++i) {
          mwi += m.y_upper[i] / chem->mw[i];
          cpt += m.y_upper[i] * cp[i];
          cvt += m.y_upper[i] * (cp[i] - kRu / chem->mw[i]);
        }
        mw = 1 / mwi;
        gamma = cpt / cvt;
      }
      vel = std::sqrt(gamma * kRu / mw * u[5]);
    }
    v_ref = vel;
    eps_scale = u[0] * v_ref * u[0] * v_ref;
    return true;
  }
  auto rs = s.strings.find("reference_state");
  if (rs == s.strings.end()) return true;
  double bv[6], c;
  std::vector<double> y;
  if (!inflow_state(s, rs->second, chem, bv, y, c, err)) {
    err = "reference_state: " + err;
    return false;
  }
  // the reference state (BoundCond.cpp:299-305): v_inf = |V|, or c when |V| < 1
  const double velocity = std::sqrt(bv[1] * bv[1] + bv[2] * bv[2] + bv[3] * bv[3]);
  const auto &st = s.structs.at(rs->second);
  const double vmag = struct_real(st, "mach", -1) * c;  // Inflow's `velocity` member
  (void)velocity;
  v_ref = std::abs(vmag) < 1 ? c : vmag;
  eps_scale = bv[0] * v_ref * bv[0] * v_ref;
  return true;
}

bool resolve_boundaries(const Setup &s, const Derived &d, HostMesh &mesh, std::string &err) {
  // label -> (type, struct name) from the setup's boundary_conditions structs, then default labels
  std::map<int, std::pair<int, std::string>> lab;
  static const std::map<std::string, int> tname{{"wall", kWall},          {"inflow", kInflow},
                                                {"outflow", kOutflow},    {"symmetry", kSymmetry},
                                                {"farfield", kFarfield},  {"subsonic_inflow", kSubsonicInflow},
                                                {"back_pressure", kBackPressure}, {"periodic", kPeriodic}};
  auto bcs = s.string_arrays.find("boundary_conditions");
  if (bcs != s.string_arrays.end()) {
    for (const auto &name : bcs->second) {
      auto st = s.structs.find(name);
      if (st == s.structs.end()) continue;
      auto l = st->second.find("label");
      auto t = st->second.find("type");
      if (l == st->second.end() || t == st->second.end()) continue;
      const int label = std::get<int>(l->second);
      auto tt = tname.find(std::get<std::string>(t->second));
      if (tt != tname.end() && !lab.count(label)) lab[label] = {tt->second, name};
    }
  }
  for (auto &B : mesh.blocks)
    for (auto &f : B.faces) {
      auto it = lab.find(f.label);
      f.type = it != lab.end() ? it->second.first : f.label;
      if (f.type != kSymmetry && f.type != kFarfield && f.type != kOutflow && f.type != kPeriodic &&
          f.type != kWall && f.type != kInflow && f.type != kSubsonicInflow && f.type != kBackPressure) {
        err = "boundary label " + std::to_string(f.label) +
              " maps to a type outside this path (supported: wall 2, symmetry 3, farfield 4, inflow 5, outflow 6, "
              "subsonic_inflow 7, periodic 8, back_pressure 9)";
        return false;
      }
      if (f.type == kSubsonicInflow || f.type == kBackPressure) {
        // SubsonicInflow / BackPressure ctors (BoundCond.cpp:704-768): air only, states resolved with
        // the reference state in resolve_inflows
        if (d.species != 0) {
          err = std::string(f.type == kBackPressure ? "back pressure" : "subsonic inflow") +
                " faces do not support multi-species cases (label " + std::to_string(f.label) + ")";
          return false;
        }
        if (it == lab.end()) {
          err = "label " + std::to_string(f.label) + " needs a struct in boundary_conditions";
          return false;
        }
        f.struct_name = it->second.second;
        if (f.type == kSubsonicInflow) {
          // the total-state ratios have no default (SubsonicInflow::SubsonicInflow reads them with
          // info.at, BoundCond.cpp:714-715)
          const auto &st = s.structs.at(f.struct_name);
          for (const char *key : {"pt_pRef_ratio", "Tt_TRef_ratio"})
            if (!st.count(key)) {
              err = "subsonic inflow struct '" + f.struct_name + "' has no " + key;
              return false;
            }
        }
        continue;
      }
      if (f.type == kInflow) {
        // apply_inflow (BoundCond.cuh:235-613): a constant state (inflow_type 0) or, in a mixing-layer
        // problem, the two-stream tanh profile (inflow_type 2, forced by problem_type 1; Inflow ctor
        // BoundCond.cpp:10-21), either with optional white noise on the velocity (fluctuation_type 1).
        // Profile-file inflows (1), stability-mode and receptivity fluctuations (2, 3) and the digital
        // filter (11) are not on this path.
        if (it == lab.end()) {
          err = "inflow label " + std::to_string(f.label) + " needs a struct in boundary_conditions";
          return false;
        }
        const auto &st = s.structs.at(it->second.second);
        auto get_int = [&](const char *k) {
          auto q = st.find(k);
          return q != st.end() && std::holds_alternative<int>(q->second) ? std::get<int>(q->second) : 0;
        };
        int itype = get_int("inflow_type"), ftype = get_int("fluctuation_type");
        if (d.problem_type == 1) itype = 2;
        if (d.problem_type == 0 && itype == 2) itype = 0;
        if (itype != 2 && ftype == 11) ftype = 0;
        if (itype != 0 && itype != 2) {
          err = "inflow label " + std::to_string(f.label) + ": inflow_type " + std::to_string(itype) +
                " (profile file) is not provided; constant (0) and mixing-layer (problem_type 1) inflows are";
          return false;
        }
        if (ftype != 0 && ftype != 1 && ftype != 11) {
          err = "inflow label " + std::to_string(f.label) + ": fluctuation_type " + std::to_string(ftype) +
                " is not provided (stability-mode and receptivity fluctuations); white noise (1) and, for "
                "mixing-layer inflows, the digital filter (11) are";
          return false;
        }
        if (ftype == 11) {
          // DBoundCond::initialize_digital_filter (DigitalFilter.cu:8-120): the inflow plane i = 0 of a
          // 3-D block, z periodic; the Gaussian Reynolds-stress supplier (reynolds_stress_supplier 2)
          if (f.face != 0 || f.direction != -1 || mesh.dimension != 3) {
            err = "inflow label " + std::to_string(f.label) +
                  ": the digital filter needs the i = 0 face of a 3-D block (the reference supports no other)";
            return false;
          }
          if (B.mz - 1 < 50 + B.ngg) {
            // apply_periodic_in_spanwise copies k = 1..50+ngg from k = 0..mz-1; with fewer planes its
            // parallel copies read ghosts other threads write (DigitalFilter.cu:539-554)
            err = "the digital filter needs mz - 1 >= 50 + ngg spanwise nodes (its periodic extension is "
                  "otherwise undefined in the reference)";
            return false;
          }
          if (s.get_int("reynolds_stress_supplier") != 2) {
            err = "the digital filter supports reynolds_stress_supplier = 2 (Gaussian Reynolds stresses) only";
            return false;
          }
          auto rij = s.real_arrays.find("df_reynolds_gaussian_peak");
          if (rij == s.real_arrays.end() || rij->second.size() < 6) {
            err = "the digital filter needs the array df_reynolds_gaussian_peak (R11 R12 R22 R13 R23 R33)";
            return false;
          }
          f.df_rij.assign(rij->second.begin(), rij->second.begin() + 6);
        }
        f.inflow_type = itype;
        f.fluctuation_type = ftype;
        f.fluct_intensity = ftype == 1 ? struct_real(st, "fluctuation_intensity", 0.0) : 0.0;
        f.struct_name = it->second.second;
        continue;
      }
      if (f.type == kWall) {
        // Wall::Wall (BoundCond.cpp:497-560): isothermal (default, 300 K) or adiabatic; the radiative
        // wall needs wall distances and the blowing / fluctuating walls their forcing, neither on
        // this path
        f.temperature = 300.0;
        f.wall_adiabatic = 0;
        if (it != lab.end()) {
          const auto &st = s.structs.at(it->second.second);
          auto tt = st.find("thermal_type");
          const std::string th = tt == st.end() ? "isothermal" : std::get<std::string>(tt->second);
          if (th == "adiabatic") {
            f.wall_adiabatic = 1;
          } else if (th == "equilibrium_radiation") {
            err = "wall label " + std::to_string(f.label) +
                  ": thermal_type equilibrium_radiation is not provided (isothermal and adiabatic are)";
            return false;
          }
          f.temperature = struct_real(st, "temperature", 300.0);
          auto fl = st.find("fluctuation_type");
          if (fl != st.end() && std::holds_alternative<int>(fl->second) && std::get<int>(fl->second) != 0) {
            err = "wall label " + std::to_string(f.label) + ": wall fluctuations (fluctuation_type) are not provided";
            return false;
          }
        }
        continue;
      }
      if (f.type == kFarfield) {
        if (it == lab.end()) {
          err = "farfield label " + std::to_string(f.label) + " needs a struct in boundary_conditions";
          return false;
        }
        if (d.species != 0) {
          // mixtures: the state needs the species tables (resolve_inflows)
          f.struct_name = it->second.second;
          continue;
        }
        const auto &st = s.structs.at(it->second.second);
        // FarField::FarField (BoundCond.cpp:586-669), air
        double mach = struct_real(st, "mach", -1), pressure = struct_real(st, "pressure", -1),
               temperature = struct_real(st, "temperature", -1), velocity = struct_real(st, "velocity", 0),
               density = struct_real(st, "density", -1), u = struct_real(st, "u", 1), v = struct_real(st, "v", 0),
               w = struct_real(st, "w", 0), re = struct_real(st, "reynolds_number", -1);
        const double mw = kMwAir, gamma = kGammaAir;
        if (temperature < 0) temperature = pressure * mw / (density * kRu);
        const double viscosity = sutherland_host(temperature);
        const double c = std::sqrt(gamma * kRu / mw * temperature);
        if (mach < 0) mach = velocity / c;
        else velocity = mach * c;
        u *= velocity;
        v *= velocity;
        w *= velocity;
        if (pressure < 0) {
          density = viscosity * re / velocity;
          pressure = density * temperature * kRu / mw;
        }
        if (density < 0) density = pressure * mw / (kRu * temperature);
        f.density = density;
        f.u = u;
        f.v = v;
        f.w = w;
        f.pressure = pressure;
        f.temperature = temperature;
        f.acoustic_speed = c;
        f.gamma = gamma;
        f.entropy = pressure / std::pow(density, gamma);
        f.mw = mw;
      }
    }
  return true;
}

bool resolve_inflows(const Setup &s, const ChemTables *chem, HostMesh &mesh, std::string &err) {
  // p_inf, T_inf: the reference state's pressure and temperature (Inflow ctor, BoundCond.cpp:299-310)
  auto ref_pt = [&](double &p_inf, double &t_inf) {
    auto rs = s.strings.find("reference_state");
    if (rs == s.strings.end()) {
      err = "a pressure or temperature ratio needs the reference_state struct (p_inf, T_inf)";
      return false;
    }
    double bv[6], c;
    std::vector<double> y;
    if (!inflow_state(s, rs->second, chem, bv, y, c, err)) return false;
    p_inf = bv[4];
    t_inf = bv[5];
    return true;
  };
  for (auto &B : mesh.blocks)
    for (auto &f : B.faces) {
      if (f.type == kBackPressure) {
        const auto &st = s.structs.at(f.struct_name);
        f.pressure = struct_real(st, "pressure", -1);
        if (f.pressure < 0) {
          double p_inf, t_inf;
          if (!ref_pt(p_inf, t_inf)) return false;
          f.pressure = struct_real(st, "p_pRef_ratio", 1.0) * p_inf;
        }
        continue;
      }
      if (f.type == kSubsonicInflow) {
        const auto &st = s.structs.at(f.struct_name);
        double p_inf, t_inf;
        if (!ref_pt(p_inf, t_inf)) return false;
        f.pressure = struct_real(st, "pt_pRef_ratio", 1.0) * p_inf;     // total pressure
        f.temperature = struct_real(st, "Tt_TRef_ratio", 1.0) * t_inf;  // total temperature
        f.u = struct_real(st, "u", 1.0);
        f.v = struct_real(st, "v", 0.0);
        f.w = struct_real(st, "w", 0.0);
        continue;
      }
      if (f.type == kFarfield && chem && chem->n_spec > 0) {
        // FarField::FarField for mixtures (BoundCond.cpp:586-669): (mach, pressure, temperature) with the
        // struct's mass fractions; gamma from cp and cv of the composition at the temperature
        const auto &st = s.structs.at(f.struct_name);
        if (struct_real(st, "pressure", -1) < 0 || struct_real(st, "temperature", -1) < 0 ||
            struct_real(st, "mach", -1) < 0) {
          err = "far-field struct '" + f.struct_name + "' of a mixture needs mach, pressure and temperature on this path";
          return false;
        }
        double bv[6], c, gamma;
        if (!inflow_state(s, f.struct_name, chem, bv, f.y, c, err, &gamma)) return false;
        double mw = 0;
        for (int i = 0; i < chem->n_spec; ++i) mw += f.y[i] / chem->mw[i];
        mw = 1 / mw;
        f.density = bv[0];
        f.u = bv[1];
        f.v = bv[2];
        f.w = bv[3];
        f.pressure = bv[4];
        f.temperature = bv[5];
        f.acoustic_speed = c;
        f.gamma = gamma;
        f.mw = mw;
        f.entropy = bv[4] / std::pow(bv[0], f.gamma);
        continue;
      }
      if (f.type != kInflow) continue;
      if (f.inflow_type == 2) {
        // the mixing-layer inflow (Inflow ctor, BoundCond.cpp:28-98): the upper stream in the face's
        // constant-state members, the lower stream beside it
        MixingLayerStreams m;
        if (!mixing_layer_streams(s, chem, m, err)) return false;
        f.density = m.upper[0];
        f.u = m.upper[1];
        f.v = m.upper[2];
        f.w = m.upper[3];
        f.pressure = m.upper[4];
        f.temperature = m.upper[5];
        f.velocity = std::sqrt(f.u * f.u + f.v * f.v + f.w * f.w);
        f.y = m.y_upper;
        for (int l = 0; l < 6; ++l) f.lower[l] = m.lower[l];
        f.y_lower = m.y_lower;
        f.delta_omega = m.delta_omega;
        continue;
      }
      double bv[6], c;
      if (!inflow_state(s, f.struct_name, chem, bv, f.y, c, err)) return false;
      f.density = bv[0];
      f.u = bv[1];
      f.v = bv[2];
      f.w = bv[3];
      f.pressure = bv[4];
      f.temperature = bv[5];
      // the Inflow's velocity member: Mach times the speed of sound (BoundCond.cpp:217-223)
      f.velocity = struct_real(s.structs.at(f.struct_name), "mach", -1) * c;
    }
  return true;
}

std::vector<std::pair<int, int>> bc_order(const Setup &s, const HostMesh &mesh) {
  // label order per type: first the labels named in boundary_conditions (in that order), then the
  // remaining labels in order of first appearance (BoundCond.cu:163-258)
  std::vector<int> seen;
  for (const auto &B : mesh.blocks)
    for (const auto &f : B.faces)
      if (std::find(seen.begin(), seen.end(), f.label) == seen.end()) seen.push_back(f.label);
  std::vector<int> ordered;
  auto bcs = s.string_arrays.find("boundary_conditions");
  if (bcs != s.string_arrays.end())
    for (const auto &name : bcs->second) {
      auto st = s.structs.find(name);
      if (st == s.structs.end()) continue;
      auto l = st->second.find("label");
      if (l == st->second.end()) continue;
      const int label = std::get<int>(l->second);
      auto it = std::find(seen.begin(), seen.end(), label);
      if (it != seen.end()) {
        ordered.push_back(label);
        seen.erase(it);
      }
    }
  for (int l : seen) ordered.push_back(l);
  static const int prio[] = {kFarfield, kOutflow, kBackPressure, kInflow, kSubsonicInflow, kSymmetry, kWall, kPeriodic};
  std::vector<std::pair<int, int>> out;
  for (size_t b = 0; b < mesh.blocks.size(); ++b) {
    const auto &B = mesh.blocks[b];
    for (int t : prio)
      for (int label : ordered)
        for (size_t f = 0; f < B.faces.size(); ++f)
          if (B.faces[f].label == label && B.faces[f].type == t) out.emplace_back((int)b, (int)f);
  }
  return out;
}

}  // namespace ostc
