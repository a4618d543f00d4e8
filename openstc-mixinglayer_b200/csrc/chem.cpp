// chem.cpp -- CHEMKIN-format species / thermo / transport / reaction reader (see chem.h).
#include "chem.h"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <fstream>
#include <sstream>

namespace ostc {
namespace {

// IUPAC standard atomic weights (abridged), the values the reference's element table holds for
// the elements a combustion mechanism uses (Element.cpp:13-31).
double atomic_weight(const std::string &sym) {
  static const std::map<std::string, double> w = {
      {"H", 1.008},   {"HE", 4.002602}, {"C", 12.011}, {"N", 14.007}, {"O", 15.999},
      {"F", 18.998403163}, {"NE", 20.1797}, {"S", 32.06}, {"CL", 35.45}, {"AR", 39.95}};
  auto it = w.find(sym);
  return it == w.end() ? -1.0 : it->second;
}

std::string upper(std::string s) {
  for (auto &ch : s) ch = (char)std::toupper((unsigned char)ch);
  return s;
}

std::string trim_left(const std::string &s) {
  size_t p = 0;
  while (p < s.size() && std::isspace((unsigned char)s[p])) ++p;
  return s.substr(p);
}

// gxl::getline with Case::upper (gxl_lib/MyString.cpp:15-28): left-trimmed, upper-cased line
bool getline_up(std::istream &f, std::string &line) {
  if (!std::getline(f, line)) return false;
  line = upper(trim_left(line));
  return true;
}

std::string field(const std::string &line, size_t pos, size_t len) {
  return pos < line.size() ? line.substr(pos, len) : std::string();
}

bool to_double(const std::string &s, double &v) {
  try {
    size_t used = 0;
    v = std::stod(s, &used);
    return used > 0;
  } catch (...) {
    return false;
  }
}

struct Reader {
  ChemTables &c;
  std::map<std::string, int> spec;   // name -> index (mechanism order)
  std::map<std::string, int> elem;   // symbol -> column
  std::vector<std::vector<int>> comp;
  std::string err;

  explicit Reader(ChemTables &t) : c(t) {}

  // ELEMENTS and SPECIES sections (Species ctor, ChemData.cpp:11-75).  Returns the token that ended
  // the species list ("REACTIONS"/"REAC"/"THERMO" or empty at end of file).
  std::string read_species(std::istream &f) {
    std::string tok;
    while (f >> tok) {
      if (tok[0] == '!') { std::getline(f, tok); continue; }
      if (tok == "ELEMENTS" || tok == "ELEM") break;
    }
    while (f >> tok) {
      if (tok[0] == '!') { std::getline(f, tok); continue; }
      tok = upper(tok);
      if (tok == "END") continue;
      if (tok == "SPECIES" || tok == "SPEC") break;
      const int n = (int)elem.size();
      elem.emplace(tok, n);
    }
    std::string stop;
    while (f >> tok) {
      if (tok[0] == '!') { std::getline(f, tok); continue; }
      tok = upper(tok);
      if (tok == "END") continue;
      if (tok == "REACTIONS" || tok == "REAC" || tok == "THERMO") { stop = tok; break; }
      const int n = (int)spec.size();
      if (spec.emplace(tok, n).second) c.names.push_back(tok);
    }
    c.n_spec = (int)spec.size();
    const int ns = c.n_spec;
    c.mw.assign(ns, 0.0);
    c.t_low.assign(ns, 300.0);
    c.t_mid.assign(ns, 1000.0);
    c.t_high.assign(ns, 5000.0);
    c.low.assign(ns * 7, 0.0);
    c.high.assign(ns * 7, 0.0);
    comp.assign(ns, std::vector<int>(elem.size(), 0));
    return stop;
  }

  // read_therm (ChemData.cpp:222-498, the two-range branch).  Returns true when a TRANSPORT section
  // follows in the same stream.
  bool read_therm(std::istream &f, bool in_mechanism) {
    std::string line;
    if (!in_mechanism) {
      while (getline_up(f, line))
        if (line.rfind("THERMO", 0) == 0) break;
    }
    double tl = 300, tm = 1000, th = 5000;
    while (std::getline(f, line)) {
      if (line.empty() || line[0] == '!') continue;
      std::istringstream s(line);
      s >> tl >> tm >> th;
      break;
    }
    std::fill(c.t_low.begin(), c.t_low.end(), tl);
    std::fill(c.t_mid.begin(), c.t_mid.end(), tm);
    std::fill(c.t_high.begin(), c.t_high.end(), th);
    std::vector<char> seen(c.n_spec, 0);
    int n_read = 0;
    while (getline_up(f, line)) {
      if (line.empty() || line[0] == '!') continue;
      std::istringstream s(line);
      std::string key;
      s >> key;
      if (key == "END") continue;
      if (key == "REACTIONS" || line == "REAC") break;
      if (key == "TRANSPORT" || key == "TRAN") return true;
      if (n_read >= c.n_spec) break;
      std::istringstream s18(field(line, 0, 18));
      key.clear();
      s18 >> key;
      std::string l2, l3, l4;
      auto it = spec.find(key);
      if (it == spec.end() || seen[it->second]) {
        std::getline(f, l2);
        std::getline(f, l3);
        std::getline(f, l4);
        if (it != spec.end()) {
          // an already-read species: the reference also consumes the following header line
          std::getline(f, l2);
        }
        continue;
      }
      const int sp = it->second;
      double v;
      if (to_double(field(line, 45, 10), v)) c.t_low[sp] = v;
      if (to_double(field(line, 55, 10), v)) c.t_high[sp] = v;
      {
        std::istringstream sm(field(line, 65, 10));
        std::string t;
        if (sm >> t && to_double(t, v)) c.t_mid[sp] = v;
      }
      for (int q = 0; q < 4; ++q) {
        const std::string cs = trim_left(field(line, 24 + q * 5, 5));
        if (cs.empty() || cs[0] == '0') break;
        std::istringstream se(cs);
        std::string sym;
        int cnt = 0;
        se >> sym;
        auto e = elem.find(sym);
        if (e == elem.end()) continue;
        se >> cnt;
        comp[sp][e->second] = cnt;
      }
      // molecular weight, summed over the element list in symbol order
      double w = 0;
      for (const auto &[sym, col] : elem) w += atomic_weight(sym) * comp[sp][col];
      c.mw[sp] = w;
      std::getline(f, l2);
      std::getline(f, l3);
      std::getline(f, l4);
      double *hi = &c.high[sp * 7], *lo = &c.low[sp * 7];
      bool ok = true;
      for (int q = 0; q < 5; ++q) ok = ok && to_double(field(l2, q * 15, 15), hi[q]);
      ok = ok && to_double(field(l3, 0, 15), hi[5]) && to_double(field(l3, 15, 15), hi[6]);
      for (int q = 0; q < 3; ++q) ok = ok && to_double(field(l3, 30 + q * 15, 15), lo[q]);
      for (int q = 0; q < 4; ++q) ok = ok && to_double(field(l4, q * 15, 15), lo[3 + q]);
      if (!ok) {
        err = "malformed NASA-7 coefficients for species " + key;
        return false;
      }
      seen[sp] = 1;
      ++n_read;
    }
    return false;
  }

  // read_tran and the derived pair tables (ChemData.cpp:500-612)
  bool read_tran(std::istream &f) {
    const int ns = c.n_spec;
    std::vector<double> eps(ns, 0), sigma(ns, 0), mu(ns, 0), alpha(ns, 0), zrot(ns, 0);
    c.geometry.assign(ns, 0);
    c.lj_potent_inv.assign(ns, 0);
    c.vis_coeff.assign(ns, 0);
    std::vector<char> seen(ns, 0);
    int n_read = 0;
    std::string line;
    while (getline_up(f, line)) {
      if (line.empty() || line[0] == '!') continue;
      std::istringstream s(line);
      std::string key;
      s >> key;
      if (key.rfind("END", 0) == 0 || key.rfind("REAC", 0) == 0) break;
      auto it = spec.find(key);
      if (it == spec.end()) continue;
      if (n_read >= ns) break;
      const int sp = it->second;
      if (seen[sp]) continue;
      s >> c.geometry[sp] >> eps[sp] >> sigma[sp] >> mu[sp] >> alpha[sp] >> zrot[sp];
      c.lj_potent_inv[sp] = 1.0 / eps[sp];
      c.vis_coeff[sp] = 2.6693e-6 * std::sqrt(c.mw[sp]) / (sigma[sp] * sigma[sp]);
      seen[sp] = 1;
      ++n_read;
    }
    if (n_read < ns) {
      err = "transport data missing for " + std::to_string(ns - n_read) + " species";
      return false;
    }
    c.wj_div_wi_1_4.assign(ns * ns, 0);
    c.sqrt_wiwj_8.assign(ns * ns, 0);
    c.binary_diff.assign(ns * ns, 0);
    c.kb_over_eps_jk.assign(ns * ns, 0);
    for (int i = 0; i < ns; ++i)
      for (int j = 0; j < ns; ++j) {
        c.wj_div_wi_1_4[i * ns + j] = std::pow(c.mw[j] / c.mw[i], 0.25);
        c.sqrt_wiwj_8[i * ns + j] = 1.0 / std::sqrt(8 * (1 + c.mw[i] / c.mw[j]));
      }
    // reduced dipole moment (compute_reduced_dipole_moment, ChemData.cpp:600-611): Debye -> cm^(3/2)
    // J^(1/2), Angstrom -> cm
    const double conv = 1e-18 * std::sqrt(1e-7) * std::pow(1e+8, 1.5) / std::sqrt(kBoltzmann);
    auto red_mu = [&](int i) { return mu[i] == 0 ? 0.0 : conv * mu[i] / std::sqrt(eps[i] * sigma[i] * sigma[i] * sigma[i]); };
    for (int j = 0; j < ns; ++j) {
      const double wjj = c.mw[j] * 0.5;
      c.binary_diff[j * ns + j] = 0.0188324 / (std::sqrt(wjj) * sigma[j] * sigma[j]);
      for (int k = j + 1; k < ns; ++k) {
        const double wjk = c.mw[j] * c.mw[k] / (c.mw[j] + c.mw[k]);
        double xi = 1;
        if ((mu[j] != 0) != (mu[k] != 0)) {
          // polar / non-polar pair (compute_xi, ChemData.cpp:584-598)
          const int p = mu[j] != 0 ? j : k, n = mu[j] != 0 ? k : j;
          const double an = alpha[n] / std::pow(sigma[n], 3);
          const double mp = red_mu(p);
          xi = 1.0 + 0.25 * an * mp * mp * std::sqrt(eps[p] / eps[n]);
        }
        const double sjk = 0.5 * (sigma[j] + sigma[k]) * std::pow(xi, -1.0 / 6.0);
        c.binary_diff[j * ns + k] = c.binary_diff[k * ns + j] = 0.0188324 / (std::sqrt(wjk) * sjk * sjk);
        const double ejk = xi * xi * std::sqrt(eps[j] * eps[k]);
        c.kb_over_eps_jk[j * ns + k] = c.kb_over_eps_jk[k * ns + j] = 1.0 / ejk;
      }
    }
    return true;
  }

  int sp_index(const std::string &name) {
    auto it = spec.find(name);
    if (it == spec.end()) {
      err = "reaction names unknown species '" + name + "'";
      return -1;
    }
    return it->second;
  }

  // one side of an equation: "2O+H2" -> stoichiometric counts (read_reaction_line, ChemData.cpp:697-775)
  bool side(std::string s, int *st, int &order, int sign) {
    while (!s.empty()) {
      size_t plus = s.find('+');
      if (plus != std::string::npos && plus + 1 < s.size() && s[plus + 1] == '+') ++plus;
      std::string term = plus == std::string::npos ? s : s.substr(0, plus);
      s = plus == std::string::npos ? std::string() : s.substr(plus + 1);
      int nu = 1;
      if (!term.empty() && std::isdigit((unsigned char)term[0])) {
        nu = term[0] - '0';
        term = term.substr(1);
      }
      const int sp = sp_index(term);
      if (sp < 0) return false;
      st[sp] += nu;
      order += sign * nu;
    }
    return true;
  }

  bool reaction_line(std::string line, int r) {
    const int ns = c.n_spec;
    // catalysts: "+M" (third body) and "(+M)" (fall-off); both are removed from the equation
    size_t lp = line.find("(+");
    if (line.find("+M") != std::string::npos) {
      c.label[r] = 4;
      if (lp != std::string::npos) {
        c.label[r] = 5;
        line.erase(lp, line.find(')', lp) - lp + 1);
        lp = line.find("(+");
        line.erase(lp, line.find_last_of(')') - lp + 1);
      } else {
        line.erase(line.find("+M"), 2);
        line.erase(line.find("+M"), 2);
      }
    }
    size_t lt = line.find('<');
    if (lt == std::string::npos) lt = line.find('=');
    std::replace(line.begin(), line.begin() + std::min(line.size(), lt + 1), ' ', '<');
    std::istringstream s(line);
    std::string eq;
    s >> eq >> c.A[r] >> c.b[r] >> c.Ea[r];
    c.Ea[r] /= kRc;
    size_t small = eq.find('<'), e = eq.find('='), big = eq.find('>');
    if (small == std::string::npos) {
      if (big != std::string::npos) c.label[r] = 0;
      else big = e;
      small = e;
    }
    int *sf = &c.stoi_f[r * ns], *sb = &c.stoi_b[r * ns];
    return side(eq.substr(0, small), sf, c.order[r], -1) && side(eq.substr(big + 1), sb, c.order[r], +1);
  }

  bool read_reactions(std::istream &f) {
    const int ns = c.n_spec;
    std::string line;
    // skip to the line that starts with the REACTIONS keyword (case kept, gxl::read_until)
    while (std::getline(f, line)) {
      const std::string t = trim_left(line);
      if (t.rfind("REACTIONS", 0) == 0 || t.rfind("REAC", 0) == 0) break;
    }
    auto grow = [&](int nr) {
      c.label.resize(nr, 1);
      c.rev_type.resize(nr, 0);
      c.order.resize(nr, 0);
      c.stoi_f.resize((size_t)nr * ns, 0);
      c.stoi_b.resize((size_t)nr * ns, 0);
      for (auto *v : {&c.A, &c.b, &c.Ea, &c.A2, &c.b2, &c.Ea2, &c.troe_alpha, &c.troe_t3, &c.troe_t1, &c.troe_t2})
        v->resize(nr, 0.0);
      c.third_body.resize((size_t)nr * ns, 1.0);
    };
    int cap = 100;
    grow(cap);
    int nr = 0;
    std::vector<int> dups;
    if (!getline_up(f, line)) line = "END";
    while (line != "END" && f) {
      if (line.empty() || line[0] == '!') {
        if (!getline_up(f, line)) break;
        continue;
      }
      if (nr >= cap) grow(cap += 100);
      if (!reaction_line(line, nr)) return false;
      // auxiliary lines (get_auxi_info, ChemData.cpp:777-840)
      bool dup = false;
      std::string aux;
      line = "END";
      while (getline_up(f, aux)) {
        std::string a = aux;
        std::replace(a.begin(), a.end(), '/', ' ');
        std::istringstream s(a);
        std::string key;
        s >> key;
        if (aux.empty() || aux[0] == '!') continue;
        if (key == "END") { line = aux; break; }
        if (aux.find('=') != std::string::npos) { line = aux; break; }
        if (key == "PLOG") continue;
        if (key == "DUPLICATE" || key == "DUP") {
          dup = true;
          c.label[nr] = 3;
          continue;
        }
        if (key == "REV") {
          s >> c.A2[nr] >> c.b2[nr] >> c.Ea2[nr];
          c.Ea2[nr] /= kRc;
          c.rev_type[nr] = 1;
        } else if (key == "LOW") {
          s >> c.A2[nr] >> c.b2[nr] >> c.Ea2[nr];
          c.Ea2[nr] /= kRc;
        } else if (key == "TROE") {
          c.label[nr] = 6;
          s >> c.troe_alpha[nr] >> c.troe_t3[nr] >> c.troe_t1[nr];
          std::string t2;
          if (s >> t2) {
            c.troe_t2[nr] = std::stod(t2);
            c.label[nr] = 7;
          }
        } else {
          std::istringstream s2(a);
          std::string name;
          double coe = 0;
          while (s2 >> name) {
            s2 >> coe;
            const int sp = sp_index(name);
            if (sp < 0) return false;
            c.third_body[(size_t)nr * ns + sp] = coe;
          }
        }
      }
      if (line == "END" && !f) line = "END";
      {
        // a line such as "END" may carry trailing blanks
        std::istringstream s(line);
        std::string k;
        s >> k;
        if (k == "END") line = "END";
      }
      if (dup) {
        int found = -1;
        for (size_t q = 0; q < dups.size() && found < 0; ++q) {
          const int d = dups[q];
          bool same = true;
          for (int l = 0; l < ns && same; ++l)
            same = c.stoi_f[d * ns + l] == c.stoi_f[nr * ns + l] && c.stoi_b[d * ns + l] == c.stoi_b[nr * ns + l];
          if (same) found = (int)q;
        }
        if (found >= 0) {
          const int d = dups[found];
          c.A2[d] = c.A[nr];
          c.b2[d] = c.b[nr];
          c.Ea2[d] = c.Ea[nr];
          dups.erase(dups.begin() + found);
          for (int l = 0; l < ns; ++l) c.stoi_f[nr * ns + l] = c.stoi_b[nr * ns + l] = 0;
          c.label[nr] = 1;
          c.order[nr] = 0;
        } else {
          dups.push_back(nr);
          ++nr;
        }
        continue;
      }
      ++nr;
    }
    c.n_reac = nr;
    c.label.resize(nr);
    c.rev_type.resize(nr);
    c.order.resize(nr);
    c.stoi_f.resize((size_t)nr * ns);
    c.stoi_b.resize((size_t)nr * ns);
    for (auto *v : {&c.A, &c.b, &c.Ea, &c.A2, &c.b2, &c.Ea2, &c.troe_alpha, &c.troe_t3, &c.troe_t1, &c.troe_t2})
      v->resize(nr);
    c.third_body.resize((size_t)nr * ns);
    return true;
  }
};

}  // namespace

void ChemTables::cp_and_h(double t, double *cp, double *h) const {
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t, t5 = t4 * t;
  for (int i = 0; i < n_spec; ++i) {
    if (t < t_low[i]) {
      const double tt = t_low[i], tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt, tt5 = tt4 * tt;
      const double *a = &low[i * 7];
      h[i] = a[0] * tt + 0.5 * a[1] * tt2 + a[2] * tt3 / 3 + 0.25 * a[3] * tt4 + 0.2 * a[4] * tt5 + a[5];
      cp[i] = a[0] + a[1] * tt + a[2] * tt2 + a[3] * tt3 + a[4] * tt4;
      h[i] += cp[i] * (t - tt);
    } else {
      const double *a = t < t_mid[i] ? &low[i * 7] : &high[i * 7];
      h[i] = a[0] * t + 0.5 * a[1] * t2 + a[2] * t3 / 3 + 0.25 * a[3] * t4 + 0.2 * a[4] * t5 + a[5];
      cp[i] = a[0] + a[1] * t + a[2] * t2 + a[3] * t3 + a[4] * t4;
    }
    h[i] *= 8314.462618 / mw[i];
    cp[i] *= 8314.462618 / mw[i];
  }
}

bool read_chemistry(const std::string &input_dir, const std::string &mechanism, const std::string &therm,
                    const std::string &tran, bool with_reactions, ChemTables &c, std::string &err) {
  c = ChemTables{};
  Reader rd(c);
  std::ifstream mech(input_dir + "/" + mechanism);
  if (!mech) {
    err = "cannot open mechanism file " + input_dir + "/" + mechanism;
    return false;
  }
  const std::string stop = rd.read_species(mech);
  if (c.n_spec == 0) {
    err = "no species in " + mechanism;
    return false;
  }
  if (c.n_spec > kMaxSpec) {
    err = "mechanism has " + std::to_string(c.n_spec) + " species; this library supports at most " +
          std::to_string(kMaxSpec);
    return false;
  }
  bool has_tran = false;
  if (stop == "THERMO") {
    has_tran = rd.read_therm(mech, true);
  } else {
    std::ifstream th(input_dir + "/" + therm);
    if (!th) {
      err = "cannot open thermodynamic data " + input_dir + "/" + therm;
      return false;
    }
    has_tran = rd.read_therm(th, false);
  }
  if (!rd.err.empty()) {
    err = rd.err;
    return false;
  }
  for (int i = 0; i < c.n_spec; ++i)
    if (c.mw[i] <= 0) {
      err = "no thermodynamic data (or unknown element) for species " + c.names[i];
      return false;
    }
  bool ok;
  if (has_tran) {
    ok = rd.read_tran(mech);
  } else {
    std::ifstream tr(input_dir + "/" + tran);
    if (!tr) {
      err = "cannot open transport data " + input_dir + "/" + tran;
      return false;
    }
    ok = rd.read_tran(tr);
  }
  if (!ok) {
    err = rd.err;
    return false;
  }
  if (with_reactions) {
    std::ifstream m2(input_dir + "/" + mechanism);
    if (!rd.read_reactions(m2)) {
      err = rd.err;
      return false;
    }
    if (c.n_reac > kMaxReac) {
      err = "mechanism has " + std::to_string(c.n_reac) + " reactions; this library supports at most " +
            std::to_string(kMaxReac);
      return false;
    }
  }
  return true;
}

}  // namespace ostc
