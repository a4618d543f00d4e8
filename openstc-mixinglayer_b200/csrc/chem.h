// chem.h -- species, thermodynamic, transport and reaction tables of a multi-component mixture, read
// from CHEMKIN-format files the way the reference's Species and Reaction constructors do
// (ChemData.cpp:11-948, Element.cpp:8-160).  Host-side set-up; the device copies live in the CUDA
// sources.
#pragma once

#include <map>
#include <string>
#include <vector>

namespace ostc {

constexpr int kMaxSpec = 16;   // device tables are sized for at most this many species
constexpr int kMaxReac = 64;   // and this many reactions (after merging duplicates)

// Physical constants of the reference (Constants.h:11-34).
constexpr double kRc = 1.98720425864083;    // cal/(mol K)
constexpr double kPatm = 101325.0;
constexpr double kBoltzmann = 1.380649e-23;
constexpr double kPi = 3.1415926535;

struct ChemTables {
  int n_spec = 0, n_reac = 0;
  std::vector<std::string> names;   // species in mechanism order
  std::vector<double> mw;           // kg/kmol
  // NASA-7, two ranges (Combustion2Part): coefficients [n_spec][7]
  std::vector<double> t_low, t_mid, t_high, low, high;
  // transport (read_tran, ChemData.cpp:500-597)
  std::vector<double> geometry, lj_potent_inv, vis_coeff;
  std::vector<double> wj_div_wi_1_4;    // [n][n]  (mw_j / mw_i)^(1/4)
  std::vector<double> sqrt_wiwj_8;      // [n][n]  1 / sqrt(8 (1 + mw_i / mw_j))
  std::vector<double> binary_diff;      // [n][n]
  std::vector<double> kb_over_eps_jk;   // [n][n]  (diagonal 0, as the reference leaves it)
  // reactions (Reaction, ChemData.cpp:614-948); label: 0 irreversible, 1 reversible, 3 duplicate
  // pair, 4 third body, 5 Lindemann, 6 Troe-3, 7 Troe-4
  std::vector<int> label, rev_type, order, stoi_f, stoi_b;   // stoi: [n_reac][n_spec]
  std::vector<double> A, b, Ea, A2, b2, Ea2, third_body, troe_alpha, troe_t3, troe_t1, troe_t2;

  // Species::compute_cp / compute_enthalpy (ChemData.cpp:148-198), J/kg
  void cp_and_h(double t, double *cp, double *h) const;
};

// Reads "<input_dir>/<mechanism_file>" (species, optional THERMO / TRANSPORT sections and REACTIONS),
// "<input_dir>/<therm_file>" and "<input_dir>/<transport_file>" when the mechanism does not carry them.
// with_reactions: parse the REACTIONS section (setup key reaction = 1).
bool read_chemistry(const std::string &input_dir, const std::string &mechanism, const std::string &therm,
                    const std::string &tran, bool with_reactions, ChemTables &c, std::string &err);

}  // namespace ostc
