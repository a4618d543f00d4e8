"""Synthetic mixing-layer cases in the reference's input format.

A case is a single-block grid, a list of boundary faces, a setup.txt and a seeded initial primitive
state.  `write_case` lays them out exactly as the reference reads them:
  <dir>/setup.txt                                  (Parameter::read_one_file grammar)
  <dir>/grid/grid   0.dat                          (binary: nblk, mx my mz, x[] y[] z[]; Mesh.cpp:663-697)
  <dir>/boundary_condition/boundary   0.txt        (face count, then "x1 x2 y1 y2 z1 z2 label"; Mesh.cpp:790-810)
  <dir>/boundary_condition/inner   0.txt           (no interfaces)
The named workloads follow the benchmark configurations: a 2-D temporal mixing layer (256 x 128
cells, WENO5-Z + AUSM+, periodic x, slip walls in y) and a 3-D one (512 x 256 x 128, WENO7-Z + HLLC,
periodic x and z, far-field y).  All inputs are synthetic and seeded.
"""
from __future__ import annotations

import dataclasses
import math
import os
import re
from pathlib import Path

import numpy as np

GAMMA = 1.4
R_U = 8314.462618
MW_AIR = 28.9647
R_AIR = R_U / MW_AIR


def sutherland(t):
    return 1.7894e-5 * (t / 288.16) ** 1.5 * (288.16 + 110) / (t + 110)


@dataclasses.dataclass
class Face:
    raw: tuple  # x1 x2 y1 y2 z1 z2 (0-based node indices)
    label: int


@dataclasses.dataclass
class Case:
    name: str
    mx: int
    my: int
    mz: int
    x: np.ndarray  # [mz, my, mx] grid units
    y: np.ndarray
    z: np.ndarray
    grid_scale: float
    faces: list
    bc_structs: dict  # name -> {key: (type, value)}
    scheme: dict      # reconstruction, inviscid_scheme, viscous_order, cfl, prandtl_number
    bv: np.ndarray    # [6, mz, my, mx] initial primitive state
    steps: int = 100
    # multi-component mixtures: sv [n_spec, mz, my, mx] mass fractions; mixture = dict(tables (a
    # SpeciesThermo: names, molecular weights, NASA-7 polynomials), finite_rate, chem_dir (directory holding
    # the CHEMKIN files), mechanism, therm, tran); freestream = reference state (mach, pressure,
    # temperature, Y {name: value}) written as the inflow struct "freestream"
    sv: np.ndarray | None = None
    mixture: dict | None = None
    freestream: dict | None = None
    # generator parameters a harness may need afterwards (e.g. the velocity difference du)
    extra: dict | None = None
    # struct names listed in boundary_conditions besides bc_structs (the freestream struct when a face
    # applies it as an inflow)
    extra_bc: tuple = ()
    # mixing-layer problem (problem_type 1): ma_c, delta_omega (m), velocity_ratio, upper_faster and the
    # upper / lower stream structs {key: value} (temperature, pressure, mass fractions by species name,
    # mixture_fraction); every inflow then takes the two-stream profile
    mixing_layer: dict | None = None

    @property
    def nodes(self) -> int:
        return self.mx * self.my * self.mz

    def setup_text(self) -> str:
        s = self.scheme
        lines = [
            "// synthetic mixing layer",
            "bool parallel = 0",
            f"int problem_type = {1 if getattr(self, 'mixing_layer', None) else 0}",
            "int mesh_file_type = 0",
            "int gridIsBinary = 1",
            f"real gridScale = {self.grid_scale!r}",
            "int initial = 1",
            f"int total_step = {self.steps}",
            "int output_file = 1000000",
            "int output_screen = 1000000",
            f"bool steady = {int(bool(s.get('steady', 0)))}",
            f"int temporal_scheme = {s.get('temporal_scheme', 3)}",
            f"int inner_iteration = {s.get('inner_iteration', 20)}",
            f"int max_inner_iteration = {s.get('max_inner_iteration', 30)}",
            f"int iteration_adjust_step = {s.get('iteration_adjust_step', 20)}",
            f"int implicit_method = {s.get('implicit_method', 0)}",
            f"int DPLUR_inner_step = {s.get('dplur_inner_step', 3)}",
            f"int chemSrcMethod = {s.get('chem_src_method', 0)}",
            f"real convergence_criteria = {s.get('convergence_criteria', 1e-8)!r}",
            f"real cfl = {s['cfl']!r}",
            f"bool fixed_time_step = {int(bool(s.get('fixed_time_step', 0)))}",
            f"real dt = {s.get('dt', 1e-8)!r}",
            f"int reconstruction = {s['reconstruction']}",
            f"int inviscid_scheme = {s['inviscid_scheme']}",
            f"int viscous_order = {s['viscous_order']}",
            f"real prandtl_number = {s['prandtl_number']!r}",
            f"int limiter = {s.get('limiter', 0)}",
            f"real entropy_fix_factor = {s.get('entropy_fix_factor', 0.125)!r}",
            f"int species = {1 if self.mixture else 0}",
            f"int reaction = {1 if self.mixture and self.mixture['finite_rate'] else 0}",
            "bool turbulence = 0",
            "bool limit_flow = 0",
            "array string boundary_conditions {",
            "    " + " ".join(list(self.bc_structs.keys()) + list(getattr(self, "extra_bc", ()))),
            "}",
        ]
        if self.mixture:
            m = self.mixture
            lines += [f"string mechanism_file = chemistry/{m['mechanism']}", f"string therm_file = chemistry/{m['therm']}",
                      f"string transport_file = chemistry/{m['tran']}"]
        if self.freestream:
            f = self.freestream
            lines += ["string reference_state = freestream", "string default_init = freestream",
                      "struct freestream = {", "    string type = inflow",
                      "    int label = 5", f"    real mach = {f['mach']!r}", f"    real pressure = {f['pressure']!r}",
                      f"    real temperature = {f['temperature']!r}", "    real u = 1.0", "    real v = 0.0",
                      "    real w = 0.0"]
            lines += [f"    real {k} = {v!r}" for k, v in f.get("Y", {}).items()]
            lines.append("}")
        for name, st in self.bc_structs.items():
            lines.append(f"struct {name} = {{")
            for k, (t, v) in st.items():
                lines.append(f"    {t} {k} = {v!r}" if t == "real" else f"    {t} {k} = {v}")
            lines.append("}")
        if getattr(self, "mixing_layer", None):
            m = self.mixing_layer
            lines += [f"real ma_c = {m['ma_c']!r}", f"real delta_omega = {m['delta_omega']!r}",
                      f"real velocity_ratio = {m['velocity_ratio']!r}", f"bool upper_faster = {int(m['upper_faster'])}",
                      "bool compatible_mixing_layer = 0"]
            if "freestream" in self.bc_structs and not self.freestream:
                lines.append("string reference_state = freestream")
            if "df_rij" in m:
                # the digital filter's Gaussian Reynolds-stress supplier (DigitalFilter.cu:309-345)
                lines += ["int reynolds_stress_supplier = 2", "array real df_reynolds_gaussian_peak {",
                          "    " + " ".join(repr(float(v)) for v in m["df_rij"]), "}"]
            for side in ("upper", "lower"):
                lines.append(f"struct {side}_stream = {{")
                lines += [f"    real {k} = {v!r}" for k, v in m[side].items()]
                lines.append("}")
        return "\n".join(lines) + "\n"

    def mixing_layer_streams(self):
        """get_mixing_layer_info (MixingLayer.cu:9-191), laminar: rho, u, v, w, p, T and the mass
        fractions of the upper and lower streams of a problem_type 1 case."""
        m = self.mixing_layer
        up, lo = m["upper"], m["lower"]
        tu, tl, pu, pl = up["temperature"], lo["temperature"], up["pressure"], lo["pressure"]
        ma_u, ma_l = up.get("mach", -1.0), lo.get("mach", -1.0)
        ns = self.mixture["tables"].n_spec if self.mixture else 0
        yu, yl = [0.0] * ns, [0.0] * ns
        if ns:
            tb = self.mixture["tables"]
            for i, name in enumerate(tb.names):
                yu[i], yl[i] = float(up.get(name, 0.0)), float(lo.get(name, 0.0))
            cpu, cpl = species_cp(tb, tu), species_cp(tb, tl)
            mwu = mwl = cp_u = cp_l = 0.0
            for i in range(ns):
                mwu += yu[i] / tb.mw[i]
                mwl += yl[i] / tb.mw[i]
                cp_u += cpu[i] * yu[i]
                cp_l += cpl[i] * yl[i]
            gu, gl = cp_u / (cp_u - R_U * mwu), cp_l / (cp_l - R_U * mwl)
            cu, cl = math.sqrt(gu * R_U * mwu * tu), math.sqrt(gl * R_U * mwl * tl)
            rho_u, rho_l = pu / (R_U * mwu * tu), pl / (R_U * mwl * tl)
        else:
            cu, cl = math.sqrt(GAMMA * R_U / MW_AIR * tu), math.sqrt(GAMMA * R_U / MW_AIR * tl)
            rho_u, rho_l = pu * MW_AIR / (R_U * tu), pl * MW_AIR / (R_U * tl)
        ma_c, vr, uf = m["ma_c"], m["velocity_ratio"], bool(m["upper_faster"])
        if vr > 0:
            if vr > 1:
                slow = ma_c * (cu + cl) / (vr - 1)
                fast = vr * slow
            else:
                fast = ma_c * (cu + cl) / (1 - vr)
                slow = fast * vr
            ma_u, ma_l = (fast if uf else slow) / cu, (slow if uf else fast) / cl
        elif ma_u > 0 and ma_l < 0:
            ma_l = (ma_u - ma_c) * cu / cl - ma_c if uf else (ma_c + ma_u) * cu / cl + ma_c
        elif ma_l > 0 and ma_u < 0:
            ma_u = (ma_c + ma_l) * cl / cu + ma_c if uf else (ma_l - ma_c) * cl / cu - ma_c
        return dict(upper=[rho_u, ma_u * cu, 0.0, 0.0, pu, tu], lower=[rho_l, ma_l * cl, 0.0, 0.0, pl, tl],
                    y_upper=yu, y_lower=yl, delta_omega=m["delta_omega"])

    def farfield_states(self):
        """FarField ctor (BoundCond.cpp:586-669) from (mach, pressure, temperature): label -> state dict;
        for mixtures with the struct's mass fractions y, their molecular weight and gamma = cp / cv."""
        out = {}
        for name, st in self.bc_structs.items():
            if st.get("type", (None, None))[1] != "farfield":
                continue
            g = {k: v for k, (t, v) in st.items()}
            mach, p, t = g.get("mach", -1.0), g.get("pressure", -1.0), g.get("temperature", -1.0)
            u, v, w = g.get("u", 1.0), g.get("v", 0.0), g.get("w", 0.0)
            mw, gamma, y = MW_AIR, GAMMA, [0.0] * 16
            if self.mixture:
                tb = self.mixture["tables"]
                yk = [float(g.get(n, 0.0)) for n in tb.names]
                mw = 0.0
                for i in range(tb.n_spec):
                    mw += yk[i] / tb.mw[i]
                mw = 1 / mw
                cpi = species_cp(tb, t)
                cp = cv = 0.0
                for i in range(tb.n_spec):
                    cp += yk[i] * cpi[i]
                    cv += yk[i] * (cpi[i] - R_U / tb.mw[i])
                gamma = cp / cv
                y[:tb.n_spec] = yk
            c = math.sqrt(gamma * R_U / mw * t)
            vel = mach * c
            rho = p * mw / (R_U * t)
            out[g["label"]] = dict(density=rho, u=u * vel, v=v * vel, w=w * vel, pressure=p, temperature=t,
                                   acoustic_speed=c, gamma=gamma, entropy=p / rho ** gamma, mw=mw, y=y)
        return out

    def default_state(self):
        """(bv[6], Y) of the default initialisation (the freestream struct), or None."""
        f = self.freestream
        if not f:
            return None
        t, p, mach = f["temperature"], f["pressure"], f["mach"]
        y = []
        if self.mixture:
            tb = self.mixture["tables"]
            y = [0.0] * tb.n_spec
            for k, v in f.get("Y", {}).items():
                y[tb.names.index(k)] = v
            mw = 0.0
            for i in range(tb.n_spec):
                mw += y[i] / tb.mw[i]
            mw = 1 / mw
            cpi = species_cp(tb, t)
            cp = cv = 0.0
            for i in range(tb.n_spec):
                cp += y[i] * cpi[i]
                cv += y[i] * (cpi[i] - R_U / tb.mw[i])
            gamma = cp / cv
        else:
            mw, gamma = MW_AIR, GAMMA
        c = math.sqrt(gamma * R_U / mw * t)
        vel = mach * c
        return [p * mw / (R_U * t), 1.0 * vel, 0.0 * vel, 0.0 * vel, p, t], y

    def reference_scales(self):
        """(rho_inf^2 v_inf^2, v_inf) of the reference state as the reference's Inflow ctor computes
        them (BoundCond.cpp:157-214, 299-305); (0, 0) without one.  In a mixing-layer problem the
        reference state is the upper stream of the inflow struct it names (BoundCond.cpp:28-62)."""
        if getattr(self, "mixing_layer", None):
            ml = self.mixing_layer_streams()
            up = ml["upper"]
            vel = math.sqrt(up[1] ** 2 + up[2] ** 2 + up[3] ** 2)
            if abs(vel) < 1:
                # the Inflow's speed of sound: gamma = cp / cv of the upper stream (BoundCond.cpp:56-66)
                mw, gamma = MW_AIR, GAMMA
                if self.mixture:
                    tb = self.mixture["tables"]
                    yk = ml["y_upper"]
                    mw = 1 / sum(yk[i] / tb.mw[i] for i in range(tb.n_spec))
                    cpi = species_cp(tb, up[5])
                    cp = sum(yk[i] * cpi[i] for i in range(tb.n_spec))
                    cv = sum(yk[i] * (cpi[i] - R_U / tb.mw[i]) for i in range(tb.n_spec))
                    gamma = cp / cv
                vel = math.sqrt(gamma * R_U / mw * up[5])
            return up[0] * vel * up[0] * vel, vel
        f = self.freestream
        if not f:
            return 0.0, 0.0
        t, p, mach = f["temperature"], f["pressure"], f["mach"]
        if self.mixture:
            tb = self.mixture["tables"]
            y = np.zeros(tb.n_spec)
            for k, v in f.get("Y", {}).items():
                y[tb.names.index(k)] = v
            mw = 0.0
            for i in range(tb.n_spec):
                mw += y[i] / tb.mw[i]
            mw = 1 / mw
            cpi = species_cp(tb, t)
            cp = cv = 0.0
            for i in range(tb.n_spec):
                cp += y[i] * cpi[i]
                cv += y[i] * (cpi[i] - R_U / tb.mw[i])
            gamma = cp / cv
        else:
            mw, gamma = MW_AIR, GAMMA
        c = math.sqrt(gamma * R_U / mw * t)
        vel = mach * c
        rho = p * mw / (R_U * t)
        v_inf = c if abs(vel) < 1 else vel
        return rho * vel * rho * vel if abs(vel) >= 1 else rho * c * rho * c, v_inf

    def inflow_states(self):
        """Inflow ctor (BoundCond.cpp:157-214) of constant inflows: label -> density, velocity
        (Mach times the speed of sound along (u, v, w)), pressure, temperature and mass fractions y."""
        out = {}
        ml = self.mixing_layer_streams() if getattr(self, "mixing_layer", None) else None
        for st in self.face_structs():
            if st.get("type", (None, None))[1] != "inflow":
                continue
            g = {k: v for k, (t, v) in st.items()}
            if ml is not None:
                # problem_type 1: the mixing-layer inflow (inflow_type 2) with the two streams
                y, yl = [0.0] * 16, [0.0] * 16
                y[:len(ml["y_upper"])] = ml["y_upper"]
                yl[:len(ml["y_lower"])] = ml["y_lower"]
                up = ml["upper"]
                out[g["label"]] = dict(density=up[0], u=up[1], v=up[2], w=up[3], pressure=up[4], temperature=up[5],
                                       y=y, inflow_type=2, delta_omega=ml["delta_omega"], lower=ml["lower"],
                                       y_lower=yl)
                continue
            t, p, mach = float(g["temperature"]), float(g["pressure"]), float(g["mach"])
            y = [0.0] * 16
            mw, gamma = MW_AIR, GAMMA
            if self.mixture:
                tb = self.mixture["tables"]
                yk = [float(g.get(n, 0.0)) for n in tb.names]
                mw = 0.0
                for i in range(tb.n_spec):
                    mw += yk[i] / tb.mw[i]
                mw = 1 / mw
                cpi = species_cp(tb, t)
                cp = cv = 0.0
                for i in range(tb.n_spec):
                    cp += yk[i] * cpi[i]
                    cv += yk[i] * (cpi[i] - R_U / tb.mw[i])
                gamma = cp / cv
                y[:tb.n_spec] = yk
            vel = mach * math.sqrt(gamma * R_U / mw * t)
            out[g["label"]] = dict(density=p * mw / (R_U * t), u=g.get("u", 1.0) * vel, v=g.get("v", 0.0) * vel,
                                   w=g.get("w", 0.0) * vel, pressure=p, temperature=t, y=y)
        return out

    def characteristic_states(self):
        """SubsonicInflow / BackPressure ctors (BoundCond.cpp:704-768), air: label -> total pressure and
        temperature (ratios times the reference state's p and T) with the flow direction, or the back
        pressure (given, or its ratio times the reference pressure)."""
        out = {}
        f = self.freestream or {}
        for st in self.bc_structs.values():
            kind = st.get("type", (None, None))[1]
            if kind not in ("subsonic_inflow", "back_pressure"):
                continue
            g = {k: v for k, (t, v) in st.items()}
            if kind == "back_pressure":
                p = float(g.get("pressure", -1.0))
                if p < 0:
                    p = float(g.get("p_pRef_ratio", 1.0)) * f["pressure"]
                out[g["label"]] = dict(pressure=p)
            else:
                out[g["label"]] = dict(pressure=float(g.get("pt_pRef_ratio", 1.0)) * f["pressure"],
                                       temperature=float(g.get("Tt_TRef_ratio", 1.0)) * f["temperature"],
                                       u=float(g.get("u", 1.0)), v=float(g.get("v", 0.0)), w=float(g.get("w", 0.0)))
        return out

    def wall_states(self):
        """Wall ctor (BoundCond.cpp:497-560): label -> isothermal wall temperature (300 K by default)
        and the adiabatic flag."""
        out = {}
        for st in self.bc_structs.values():
            if st.get("type", (None, None))[1] != "wall":
                continue
            g = {k: v for k, (t, v) in st.items()}
            out[g["label"]] = dict(temperature=float(g.get("temperature", 300.0)),
                                   wall_adiabatic=int(g.get("thermal_type", "isothermal") == "adiabatic"))
        return out

    def face_structs(self):
        """The boundary structs faces may apply: bc_structs, plus the freestream struct when
        boundary_conditions lists it (extra_bc)."""
        out = list(self.bc_structs.values())
        if "freestream" in getattr(self, "extra_bc", ()) and self.freestream:
            f = self.freestream
            st = {"type": ("string", "inflow"), "label": ("int", 5), "mach": ("real", f["mach"]),
                  "pressure": ("real", f["pressure"]), "temperature": ("real", f["temperature"]),
                  "u": ("real", 1.0), "v": ("real", 0.0), "w": ("real", 0.0)}
            for k, v in f.get("Y", {}).items():
                st[k] = ("real", v)
            out.append(st)
        return out

    def label_types(self):
        types = {"wall": 2, "symmetry": 3, "farfield": 4, "inflow": 5, "outflow": 6, "subsonic_inflow": 7,
                 "periodic": 8, "back_pressure": 9}
        m = {}
        for st in self.face_structs():
            m[st["label"][1]] = types[st["type"][1]]
        return m


# element weights (kg/kmol) the species molecular weights are summed from
_ATOMIC_WEIGHT = {"H": 1.008, "HE": 4.002602, "C": 12.011, "N": 14.007, "O": 15.999, "AR": 39.95}


class SpeciesThermo:
    """Species names (mechanism order), molecular weights and NASA-7 polynomials: what a synthetic
    initial state and its freestream need from the CHEMKIN files (the library itself reads the full
    mechanism, thermodynamics and transport from the same files)."""
    names: list
    n_spec: int
    mw: np.ndarray
    t_low: np.ndarray
    t_mid: np.ndarray
    t_high: np.ndarray
    low: np.ndarray   # [n_spec, 7] below t_mid
    high: np.ndarray  # [n_spec, 7] above t_mid


def read_species(chem_dir: os.PathLike, mechanism: str, therm: str) -> SpeciesThermo:
    """Species of the mechanism's SPECIES block and their therm.dat entries (fixed-column CHEMKIN
    layout: name in columns 1-18, up to four element/count pairs of 5 columns from column 25, the
    temperature range in columns 46-75, then 5 + 5 + 4 coefficients of 15 columns on three lines)."""
    text = Path(chem_dir, mechanism).read_text().upper()
    text = "\n".join(line.split("!")[0] for line in text.split("\n"))
    m = re.search(r"\bSPEC(?:IES)?\b(.*?)\bEND\b", text, re.S)
    if m is None:
        raise ValueError(f"{mechanism}: no SPECIES block")
    names = list(dict.fromkeys(m.group(1).split()))
    ns = len(names)
    st = SpeciesThermo()
    st.names, st.n_spec = names, ns
    st.mw = np.zeros(ns)
    st.t_low, st.t_mid, st.t_high = np.full(ns, 300.0), np.full(ns, 1000.0), np.full(ns, 5000.0)
    st.low, st.high = np.zeros((ns, 7)), np.zeros((ns, 7))
    lines = Path(chem_dir, therm).read_text().split("\n")
    i = next(k for k, line in enumerate(lines) if line.upper().startswith("THERMO")) + 1
    while not lines[i].strip() or lines[i].lstrip().startswith("!"):
        i += 1
    st.t_low[:], st.t_mid[:], st.t_high[:] = (float(v) for v in lines[i].split()[:3])
    i += 1
    found = set()
    while i < len(lines) and len(found) < ns:
        head = lines[i].upper()
        word = head[:18].split()
        if not word or head.lstrip().startswith("!") or word[0] == "END" or word[0] not in names or word[0] in found:
            i += 1
            continue
        k = names.index(word[0])
        for col, arr in ((45, st.t_low), (55, st.t_high), (65, st.t_mid)):
            field = head[col:col + 10].split()
            if field:
                arr[k] = float(field[0])
        for q in range(4):
            pair = head[24 + 5 * q:29 + 5 * q].split()
            if len(pair) == 2 and pair[0] in _ATOMIC_WEIGHT:
                st.mw[k] += _ATOMIC_WEIGHT[pair[0]] * int(float(pair[1]))
        c = [float(lines[i + 1 + r][15 * q:15 * q + 15]) for r, nq in enumerate((5, 5, 4)) for q in range(nq)]
        st.high[k] = c[0:7]
        st.low[k] = c[7:14]
        found.add(word[0])
        i += 4
    if len(found) < ns:
        raise ValueError(f"{therm}: no entry for {sorted(set(names) - found)}")
    return st


def species_cp(tb, t):
    """Species::compute_cp (ChemData.cpp:148-171): cp_k(T) in J/(kg K), constant below t_low."""
    out = np.empty(tb.n_spec)
    for i in range(tb.n_spec):
        tt = t
        if t < tb.t_low[i]:
            tt = tb.t_low[i]
            a = tb.low[i]
            tt2 = tt * tt
            tt3 = tt2 * tt
            tt4 = tt3 * tt
            out[i] = a[0] + a[1] * tt + a[2] * tt2 + a[3] * tt3 + a[4] * tt4
        else:
            a = tb.low[i] if tt < tb.t_mid[i] else tb.high[i]
            t2 = t * t
            t3 = t2 * t
            t4 = t3 * t
            out[i] = a[0] + a[1] * tt + a[2] * t2 + a[3] * t3 + a[4] * t4
        out[i] *= R_U / tb.mw[i]
    return out


@dataclasses.dataclass
class Block:
    mx: int
    my: int
    mz: int
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    faces: list
    bv: np.ndarray
    inner: list = dataclasses.field(default_factory=list)  # (this 7 ints, target 7 ints), 1-based
    sv: np.ndarray | None = None

    @property
    def nodes(self) -> int:
        return self.mx * self.my * self.mz


@dataclasses.dataclass
class MultiCase:
    """Several blocks joined by 1:1 interfaces (inner-face file), with one setup."""
    name: str
    blocks: list
    grid_scale: float
    bc_structs: dict
    scheme: dict
    steps: int = 100
    mixture: dict | None = None
    freestream: dict | None = None

    @property
    def nodes(self) -> int:
        return sum(b.nodes for b in self.blocks)

    def setup_text(self) -> str:
        return Case.setup_text(self)

    def farfield_states(self):
        return Case.farfield_states(self)

    def face_structs(self):
        return Case.face_structs(self)

    def label_types(self):
        return Case.label_types(self)

    def wall_states(self):
        return Case.wall_states(self)

    def inflow_states(self):
        return Case.inflow_states(self)

    def characteristic_states(self):
        return Case.characteristic_states(self)

    def reference_scales(self):
        return Case.reference_scales(self)

    def default_state(self):
        return Case.default_state(self)


def write_case(case, directory: os.PathLike) -> Path:
    if isinstance(case, MultiCase):
        return _write_multi(case, directory)
    d = Path(directory)
    (d / "grid").mkdir(parents=True, exist_ok=True)
    if case.mixture:
        import shutil
        (d / "chemistry").mkdir(parents=True, exist_ok=True)
        for k in ("mechanism", "therm", "tran"):
            shutil.copyfile(Path(case.mixture["chem_dir"]) / case.mixture[k], d / "chemistry" / case.mixture[k])
    (d / "boundary_condition").mkdir(parents=True, exist_ok=True)
    (d / "setup.txt").write_text(case.setup_text())
    with open(d / "grid" / "grid   0.dat", "wb") as f:
        np.array([1, case.mx, case.my, case.mz], dtype=np.int32).tofile(f)
        for a in (case.x, case.y, case.z):
            np.ascontiguousarray(a, dtype=np.float64).tofile(f)
    with open(d / "boundary_condition" / "boundary   0.txt", "w") as f:
        f.write(f"{len(case.faces):7d}\n")
        for fc in case.faces:
            f.write("".join(f"{v:7d}" for v in fc.raw) + f"{fc.label:7d}\n")
    with open(d / "boundary_condition" / "inner   0.txt", "w") as f:
        f.write("        1        0\n        0\niMin  iMax  jMin  jMax  kMin  kMax   id\n")
    return d


def _write_multi(case: MultiCase, directory: os.PathLike) -> Path:
    d = Path(directory)
    (d / "grid").mkdir(parents=True, exist_ok=True)
    (d / "boundary_condition").mkdir(parents=True, exist_ok=True)
    (d / "setup.txt").write_text(case.setup_text())
    with open(d / "grid" / "grid   0.dat", "wb") as f:
        np.array([len(case.blocks)], dtype=np.int32).tofile(f)
        for b in case.blocks:
            np.array([b.mx, b.my, b.mz], dtype=np.int32).tofile(f)
        for b in case.blocks:
            for a in (b.x, b.y, b.z):
                np.ascontiguousarray(a, dtype=np.float64).tofile(f)
    with open(d / "boundary_condition" / "boundary   0.txt", "w") as f:
        for b in case.blocks:
            f.write(f"{len(b.faces):7d}\n")
            for fc in b.faces:
                f.write("".join(f"{v:7d}" for v in fc.raw) + f"{fc.label:7d}\n")
    with open(d / "boundary_condition" / "inner   0.txt", "w") as f:
        f.write(f"{len(case.blocks):9d}{0:9d}\n")
        f.write("".join(f"{len(b.inner):9d}" for b in case.blocks) + "\n")
        f.write("iMin  iMax  jMin  jMax  kMin  kMax   id\n")
        for b in case.blocks:
            for src, tar in b.inner:
                f.write("".join(f"{v:7d}" for v in src) + "\n")
                f.write("".join(f"{v:7d}" for v in tar) + "\n")
    if case.mixture:
        import shutil
        (d / "chemistry").mkdir(parents=True, exist_ok=True)
        for k in ("mechanism", "therm", "tran"):
            shutil.copyfile(Path(case.mixture["chem_dir"]) / case.mixture[k], d / "chemistry" / case.mixture[k])
    return d


def multiblock_mixing_layer_3d(nb=12, lo=32, hi=256, my=None, mz=None, seed=0, steps=100, mc=0.5, re=1000.0,
                               t0=300.0, delta0=1e-3, h=0.125, reconstruction=5, inviscid_scheme=4, cfl=0.5,
                               dims=None, uneven_axes=False) -> MultiCase:
    """nb blocks chained along x, joined by 1:1 interfaces (block b's i-max face on block b+1's i-min
    face, coincident nodes).  Outflow at the two x ends, far-field y, periodic z within every block.
    Shear layer u = dU/2 tanh(2y/delta0), Mc = 0.5, with 1e-2 dU N(0,1) exp(-(y/delta0)^2) seeded noise in
    u, v, w.

    Extents: seeded uneven i extents (uniform in [lo, hi]; `dims` overrides) with common j / k extents
    (drawn once in [lo, hi] unless given); or, with uneven_axes, every block's three extents drawn
    (uniform in [lo, hi]; `dims` may give (mx, my, mz) tuples).  Then neighbouring blocks share the
    part of their x faces where both have nodes: block b's node j sits at y = (j - (my_b - 1) // 2) h
    and node k at z = k h, the interface covers the overlapping j and k ranges, and the rest of each
    x face is an outflow patch."""
    rng = np.random.default_rng(seed)
    if uneven_axes:
        ext = [tuple(int(v) for v in e) for e in dims] if dims is not None else \
            [tuple(int(v) for v in rng.integers(lo, hi + 1, 3)) for _ in range(nb)]
    else:
        mxs = list(dims) if dims is not None else [int(v) for v in rng.integers(lo, hi + 1, nb)]
        # the chain shares its j and k extents (1:1 faces); unless given they are drawn once from the seed
        if my is None:
            my = int(rng.integers(lo, hi + 1))
        if mz is None:
            mz = int(rng.integers(lo, hi + 1))
        ext = [(m, my, mz) for m in mxs]
    nb = len(ext)
    c0 = math.sqrt(GAMMA * R_AIR * t0)
    du = 2 * mc * c0
    rho0 = re * sutherland(t0) / (du * delta0)
    p0 = rho0 * R_AIR * t0
    two_d = all(e[2] == 1 for e in ext)
    cen = [(e[1] - 1) // 2 for e in ext]

    def overlap(b):
        """j range of block b and of block b + 1, and the shared k count, of their common x face."""
        (_, myb, mzb), (_, myn, mzn) = ext[b], ext[b + 1]
        d = cen[b] - cen[b + 1]  # j of block b = j of block b+1 + d
        jlo, jhi = max(0, d), min(myb - 1, myn - 1 + d)
        return jlo, jhi, jlo - d, jhi - d, min(mzb, mzn)

    def x_face(i, myb, mzb, jlo, jhi, kn, label_open, faces):
        """Outflow patches of an x face outside the interface's j [jlo, jhi] x k [0, kn) rectangle."""
        if jlo > 0:
            faces.append(Face((i, i, 0, jlo - 1, 0, mzb - 1), label_open))
        if jhi < myb - 1:
            faces.append(Face((i, i, jhi + 1, myb - 1, 0, mzb - 1), label_open))
        if kn < mzb:
            faces.append(Face((i, i, jlo, jhi, kn, mzb - 1), label_open))

    blocks = []
    x0 = 0.0
    for b, (mx, myb, mzb) in enumerate(ext):
        xs = x0 + np.arange(mx) * h
        ys = (np.arange(myb) - (myb - 1) / 2) * h if not uneven_axes else (np.arange(myb) - cen[b]) * h
        zs = np.arange(mzb) * h
        Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
        x0 = xs[-1]
        env = np.exp(-Y ** 2)
        bv = np.empty((6, mzb, myb, mx))
        bv[0] = rho0
        bv[1] = 0.5 * du * np.tanh(2 * Y) + 1e-2 * du * rng.standard_normal(X.shape) * env
        bv[2] = 1e-2 * du * rng.standard_normal(X.shape) * env
        bv[3] = 0.0 if two_d else 1e-2 * du * rng.standard_normal(X.shape) * env
        bv[4] = p0
        bv[5] = t0
        faces = []
        if b == 0:
            faces.append(Face((0, 0, 0, myb - 1, 0, mzb - 1), 6))
        if b == nb - 1:
            faces.append(Face((mx - 1, mx - 1, 0, myb - 1, 0, mzb - 1), 6))
        inner = []
        if b > 0:
            _, _, jlo, jhi, kn = overlap(b - 1)
            plo, phi, _, _, _ = overlap(b - 1)
            x_face(0, myb, mzb, jlo, jhi, kn, 6, faces)
            pm = ext[b - 1][0]
            inner.append(([1, 1, -(jlo + 1), -(jhi + 1), 1, kn, b + 1], [pm, pm, -(plo + 1), -(phi + 1), 1, kn, b]))
        if b < nb - 1:
            jlo, jhi, nlo, nhi, kn = overlap(b)
            x_face(mx - 1, myb, mzb, jlo, jhi, kn, 6, faces)
            inner.append(([mx, mx, -(jlo + 1), -(jhi + 1), 1, kn, b + 1], [1, 1, -(nlo + 1), -(nhi + 1), 1, kn, b + 2]))
        faces += [Face((0, mx - 1, 0, 0, 0, mzb - 1), 41), Face((0, mx - 1, myb - 1, myb - 1, 0, mzb - 1), 4)]
        if not two_d:
            faces += [Face((0, mx - 1, 0, myb - 1, 0, 0), 8), Face((0, mx - 1, 0, myb - 1, mzb - 1, mzb - 1), 8)]
        blocks.append(Block(mx, myb, mzb, X, Y, Z, faces, bv, inner))
    structs = {"outflow": {"type": ("string", "outflow"), "label": ("int", 6)},
               "farfield_upper": {"type": ("string", "farfield"), "label": ("int", 4), "mach": ("real", mc),
                                  "pressure": ("real", p0), "temperature": ("real", t0), "u": ("real", 1.0),
                                  "v": ("real", 0.0), "w": ("real", 0.0)},
               "farfield_lower": {"type": ("string", "farfield"), "label": ("int", 41), "mach": ("real", mc),
                                  "pressure": ("real", p0), "temperature": ("real", t0), "u": ("real", -1.0),
                                  "v": ("real", 0.0), "w": ("real", 0.0)}}
    if not two_d:
        structs["periodic"] = {"type": ("string", "periodic"), "label": ("int", 8)}
    scheme = dict(reconstruction=reconstruction, inviscid_scheme=inviscid_scheme, viscous_order=2, cfl=cfl,
                  prandtl_number=0.72, limiter=0, entropy_fix_factor=0.125)
    return MultiCase("multiblock_mixing_layer", blocks, delta0, structs, scheme, steps,
                     freestream=dict(mach=mc, pressure=p0, temperature=t0))


def _inflow_x(faces, structs, mach, p, t, y=None, noise=0.0):
    """Turn the periodic x faces into a constant supersonic inflow at i = 0 (label 5) and an outflow at
    i = mx - 1 (label 6); y: inflow mass fractions {name: value} of a mixture; noise > 0: white noise of
    that relative intensity on the inflow velocity (fluctuation_type 1)."""
    faces[0] = Face(faces[0].raw, 5)
    faces[1] = Face(faces[1].raw, 6)
    st = {"type": ("string", "inflow"), "label": ("int", 5), "mach": ("real", float(mach)),
          "pressure": ("real", float(p)), "temperature": ("real", float(t)), "u": ("real", 1.0), "v": ("real", 0.0),
          "w": ("real", 0.0)}
    if noise > 0:
        st["fluctuation_type"] = ("int", 1)
        st["fluctuation_intensity"] = ("real", float(noise))
    for k, v in (y or {}).items():
        st[k] = ("real", float(v))
    structs["inflow"] = st
    structs.setdefault("outflow", {"type": ("string", "outflow"), "label": ("int", 6)})


def _wall_struct(thermal, t_wall):
    """No-slip wall struct (label 2): isothermal at t_wall, or adiabatic."""
    st = {"type": ("string", "wall"), "label": ("int", 2), "thermal_type": ("string", thermal)}
    if thermal == "isothermal":
        st["temperature"] = ("real", float(t_wall))
    return st


def _box_faces(mx, my, mz, xlab, ylab_lo, ylab_hi, zlab):
    f = [Face((0, 0, 0, my - 1, 0, mz - 1), xlab), Face((mx - 1, mx - 1, 0, my - 1, 0, mz - 1), xlab),
         Face((0, mx - 1, 0, 0, 0, mz - 1), ylab_lo), Face((0, mx - 1, my - 1, my - 1, 0, mz - 1), ylab_hi)]
    if mz > 1:
        f += [Face((0, mx - 1, 0, my - 1, 0, 0), zlab), Face((0, mx - 1, 0, my - 1, mz - 1, mz - 1), zlab)]
    return f


def mixing_layer_2d(mx=257, my=129, seed=0, steps=100, mc=0.4, re=1000.0, t0=300.0, delta0=1e-3,
                    reconstruction=4, inviscid_scheme=3, cfl=0.5, entropy_fix_factor=0.125, ybc="symmetry",
                    wall_thermal="isothermal", steady=None) -> Case:
    """2-D temporal mixing layer: 256 x 128 cells on 2*pi x pi (node-coincident periodic x, mx = 257),
    u = dU/2 tanh(2y/delta0), Mc = dU/(2c), Re = rho dU delta0 / mu(T) , T and p uniform, and
    v' = 1e-3 dU sum_{m=1..8} a_m cos(m x + phi_m) exp(-(y/delta0)^2), a_m = 1/8, phi_m ~ U[0,2pi)."""
    rng = np.random.default_rng(seed)
    xs = np.linspace(0.0, 2 * math.pi, mx)
    ys = np.linspace(-math.pi / 2, math.pi / 2, my)
    Y, X = np.meshgrid(ys, xs, indexing="ij")
    x = X[None].copy()
    y = Y[None].copy()
    z = np.zeros_like(x)
    c0 = math.sqrt(GAMMA * R_AIR * t0)
    du = 2 * mc * c0
    rho0 = re * sutherland(t0) / (du * delta0)
    p0 = rho0 * R_AIR * t0
    phi = rng.uniform(0, 2 * math.pi, 8)
    a = np.full(8, 1 / 8)
    yy = y  # grid units = y / delta0
    vprime = 1e-3 * du * sum(a[m] * np.cos((m + 1) * x + phi[m]) for m in range(8)) * np.exp(-yy ** 2)
    bv = np.empty((6, 1, my, mx))
    bv[0] = rho0
    bv[1] = 0.5 * du * np.tanh(2 * yy)
    bv[2] = vprime
    bv[3] = 0.0
    bv[4] = p0
    bv[5] = t0
    if ybc == "wall":
        faces = _box_faces(mx, my, 1, 8, 2, 2, 8)
        structs = {"wall": _wall_struct(wall_thermal, t0), "periodic": {"type": ("string", "periodic"), "label": ("int", 8)}}
    elif ybc == "outflow":
        faces = _box_faces(mx, my, 1, 8, 6, 6, 8)
        structs = {"outflow": {"type": ("string", "outflow"), "label": ("int", 6)},
                   "periodic": {"type": ("string", "periodic"), "label": ("int", 8)}}
    else:
        faces = _box_faces(mx, my, 1, 8, 3, 3, 8)
        structs = {"slipwall": {"type": ("string", "symmetry"), "label": ("int", 3)},
                   "periodic": {"type": ("string", "periodic"), "label": ("int", 8)}}
    scheme = dict(reconstruction=reconstruction, inviscid_scheme=inviscid_scheme, viscous_order=2, cfl=cfl,
                  prandtl_number=0.72, limiter=0, entropy_fix_factor=entropy_fix_factor)
    scheme.update(steady or {})
    return Case("mixing_layer_2d", mx, my, 1, x, y, z, delta0, faces, structs, scheme, bv, steps)


def mixing_layer_3d(mx=512, my=256, mz=128, seed=0, steps=200, mc=0.7, re=1000.0, t0=300.0, delta0=1e-3,
                    h=0.125, reconstruction=5, inviscid_scheme=4, cfl=0.5, ybc="farfield",
                    entropy_fix_factor=0.125, wall_thermal="isothermal", xbc="periodic", ref_face=False,
                    steady=None, inflow_noise=0.0) -> Case:
    """3-D temporal mixing layer: uniform spacing h*delta0, periodic x and z (node-coincident),
    far-field (Riemann-invariant, label 4/41) or outflow (label 6) y faces; u = dU/2 tanh(2y/delta0),
    Mc = 0.7, plus 1e-2 dU N(0,1) exp(-(y/delta0)^2) seeded white noise in u, v, w.
    ref_face (with xbc="subsonic"): the j = 0 face applies the reference state as a constant inflow
    (label 5), the configuration in which the reference sets its reference values before it builds a
    subsonic inflow (its FarField and Inflow faces set them, BoundCond.cu:258-261, BoundCond.cpp:300-310)."""
    rng = np.random.default_rng(seed)
    xs = np.arange(mx) * h
    ys = (np.arange(my) - (my - 1) / 2) * h
    zs = np.arange(mz) * h
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    c0 = math.sqrt(GAMMA * R_AIR * t0)
    du = 2 * mc * c0
    rho0 = re * sutherland(t0) / (du * delta0)
    p0 = rho0 * R_AIR * t0
    env = np.exp(-Y ** 2)
    bv = np.empty((6, mz, my, mx))
    bv[0] = rho0
    bv[1] = 0.5 * du * np.tanh(2 * Y) + 1e-2 * du * rng.standard_normal(X.shape) * env
    bv[2] = 1e-2 * du * rng.standard_normal(X.shape) * env
    bv[3] = 1e-2 * du * rng.standard_normal(X.shape) * env
    bv[4] = p0
    bv[5] = t0
    if ybc == "farfield":
        faces = _box_faces(mx, my, mz, 8, 41, 4, 8)
        structs = {"periodic": {"type": ("string", "periodic"), "label": ("int", 8)},
                   "farfield_upper": {"type": ("string", "farfield"), "label": ("int", 4), "mach": ("real", mc),
                                      "pressure": ("real", p0), "temperature": ("real", t0), "u": ("real", 1.0),
                                      "v": ("real", 0.0), "w": ("real", 0.0)},
                   "farfield_lower": {"type": ("string", "farfield"), "label": ("int", 41), "mach": ("real", mc),
                                      "pressure": ("real", p0), "temperature": ("real", t0), "u": ("real", -1.0),
                                      "v": ("real", 0.0), "w": ("real", 0.0)}}
    elif ybc == "wall":
        faces = _box_faces(mx, my, mz, 8, 2, 2, 8)
        structs = {"periodic": {"type": ("string", "periodic"), "label": ("int", 8)},
                   "wall": _wall_struct(wall_thermal, t0)}
    else:
        faces = _box_faces(mx, my, mz, 8, 6, 6, 8)
        structs = {"periodic": {"type": ("string", "periodic"), "label": ("int", 8)},
                   "outflow": {"type": ("string", "outflow"), "label": ("int", 6)}}
    freestream = None
    extra_bc = ()
    if xbc == "inflow":
        _inflow_x(faces, structs, 1.5, p0, t0, noise=inflow_noise)
    elif xbc == "subsonic":
        # subsonic inflow at i = 0 (total state 1.2 p0, 1.05 T0) and back pressure p0 at i = mx - 1,
        # both relative to the reference state (Mach mc, p0, T0)
        faces[0] = Face(faces[0].raw, 7)
        faces[1] = Face(faces[1].raw, 9)
        structs["subsonic_inflow"] = {"type": ("string", "subsonic_inflow"), "label": ("int", 7),
                                      "pt_pRef_ratio": ("real", 1.2), "Tt_TRef_ratio": ("real", 1.05),
                                      "u": ("real", 1.0), "v": ("real", 0.0), "w": ("real", 0.0)}
        structs["back_pressure"] = {"type": ("string", "back_pressure"), "label": ("int", 9),
                                    "p_pRef_ratio": ("real", 1.0)}
        freestream = dict(mach=mc, pressure=p0, temperature=t0)
        if ref_face:
            faces[2] = Face(faces[2].raw, 5)
            extra_bc = ("freestream",)
    scheme = dict(reconstruction=reconstruction, inviscid_scheme=inviscid_scheme, viscous_order=2, cfl=cfl,
                  prandtl_number=0.72, limiter=0, entropy_fix_factor=entropy_fix_factor)
    scheme.update(steady or {})
    return Case("mixing_layer_3d", mx, my, mz, X, Y, Z, delta0, faces, structs, scheme, bv, steps,
                freestream=freestream, extra_bc=extra_bc)


CHEM_FIXTURE = Path(__file__).resolve().parents[2] / "tests" / "golden" / "chem"


def reacting_mixing_layer_3d(mx=384, my=192, mz=96, seed=0, steps=100, h=0.125, delta0=1e-3, mc=0.4,
                             p0=101325.0, inviscid_scheme=72, finite_rate=True, ybc="outflow",
                             chem_dir=None, fuel=None, oxidiser=None, wall_thermal="isothermal",
                             xbc="periodic", steady=None, reconstruction=2) -> Case:
    """Reacting H2/air temporal mixing layer (9 species, 19 reactions after merging duplicates):
    fuel Y_H2 = 0.05 in N2 at 300 K (y > 0) over vitiated air at 1500 K (y < 0): Y_O2 = 0.20, Y_H2O = 0.10,
    radicals Y_OH = 1e-3, Y_O = 1e-4, Y_H = 1e-5, Y_HO2 = 1e-6, Y_H2O2 = 1e-7 (so that every reaction
    runs from the first step), N2 the rest; T and Y blended by (1 + tanh(2y/delta0))/2, uniform p0, u = dU/2 tanh(2y/delta0)
    with dU = 2 Mc (c_fuel + c_ox)/2 and 1e-2 dU N(0,1) exp(-(y/delta0)^2) seeded noise in u, v, w;
    periodic x and z, outflow y; flux-split characteristic WENO7-Z (inviscid_scheme 72), or, with
    inviscid_scheme 2 / 3 / 4, the primitive reconstruction `reconstruction` (1 first order, 2 MUSCL,
    3 NND2) with Roe, AUSM+ or HLLC."""
    chem_dir = Path(chem_dir) if chem_dir else CHEM_FIXTURE
    tb = read_species(chem_dir, "H2_mech.inp", "therm.dat")
    ns = tb.n_spec
    fuel = fuel or {"H2": 0.05, "N2": 0.95}
    oxidiser = oxidiser or {"O2": 0.20, "H2O": 0.10, "OH": 1e-3, "O": 1e-4, "H": 1e-5, "HO2": 1e-6, "H2O2": 1e-7,
                            "N2": 0.70 - 1e-3 - 1e-4 - 1e-5 - 1e-6 - 1e-7}
    yf, yo = np.zeros(ns), np.zeros(ns)
    for k, v in fuel.items():
        yf[tb.names.index(k)] = v
    for k, v in oxidiser.items():
        yo[tb.names.index(k)] = v
    tf, to = 300.0, 1500.0
    rng = np.random.default_rng(seed)
    xs = np.arange(mx) * h
    ys = (np.arange(my) - (my - 1) / 2) * h
    zs = np.arange(mz) * h
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    mwf = 1 / np.sum(yf / tb.mw)
    mwo = 1 / np.sum(yo / tb.mw)
    cf = math.sqrt(GAMMA * R_U / mwf * tf)
    co = math.sqrt(GAMMA * R_U / mwo * to)
    du = mc * (cf + co)
    f = 0.5 * (1 + np.tanh(2 * Y))
    sv = np.empty((ns,) + X.shape)
    for l in range(ns):
        sv[l] = f * yf[l] + (1 - f) * yo[l]
    T = f * tf + (1 - f) * to
    mw = 1 / np.einsum("l...,l->...", sv, 1 / tb.mw)
    env = np.exp(-Y ** 2)
    bv = np.empty((6,) + X.shape)
    bv[0] = p0 * mw / (R_U * T)
    bv[1] = 0.5 * du * np.tanh(2 * Y) + 1e-2 * du * rng.standard_normal(X.shape) * env
    bv[2] = 1e-2 * du * rng.standard_normal(X.shape) * env
    bv[3] = 1e-2 * du * rng.standard_normal(X.shape) * env
    bv[4] = p0
    bv[5] = T
    if ybc == "wall":
        faces = _box_faces(mx, my, mz, 8, 2, 2, 8)
        structs = {"periodic": {"type": ("string", "periodic"), "label": ("int", 8)},
                   "wall": _wall_struct(wall_thermal, 300.0)}
    elif ybc == "outflow":
        faces = _box_faces(mx, my, mz, 8, 6, 6, 8)
        structs = {"periodic": {"type": ("string", "periodic"), "label": ("int", 8)},
                   "outflow": {"type": ("string", "outflow"), "label": ("int", 6)}}
    elif ybc == "farfield":
        # far-field (Riemann-invariant) y faces: the fuel stream above (u = +dU/2), the vitiated air below
        # (u = -dU/2), each at its own temperature and composition and the uniform pressure
        faces = _box_faces(mx, my, mz, 8, 41, 4, 8)
        up = {"type": ("string", "farfield"), "label": ("int", 4), "mach": ("real", 0.5 * du / cf),
              "pressure": ("real", p0), "temperature": ("real", tf), "u": ("real", 1.0), "v": ("real", 0.0),
              "w": ("real", 0.0)}
        lo = {"type": ("string", "farfield"), "label": ("int", 41), "mach": ("real", 0.5 * du / co),
              "pressure": ("real", p0), "temperature": ("real", to), "u": ("real", -1.0), "v": ("real", 0.0),
              "w": ("real", 0.0)}
        for k, v in fuel.items():
            up[k] = ("real", float(v))
        for k, v in oxidiser.items():
            lo[k] = ("real", float(v))
        structs = {"periodic": {"type": ("string", "periodic"), "label": ("int", 8)},
                   "farfield_upper": up, "farfield_lower": lo}
    else:
        raise ValueError("the reacting case uses outflow, wall or far-field y faces")
    if xbc == "inflow":
        _inflow_x(faces, structs, 1.2, p0, to, oxidiser)
    scheme = dict(reconstruction=reconstruction, inviscid_scheme=inviscid_scheme, viscous_order=2, cfl=0.5,
                  prandtl_number=0.72, limiter=0, entropy_fix_factor=0.125)
    scheme.update(steady or {})
    mixture = dict(tables=tb, finite_rate=finite_rate, chem_dir=str(chem_dir), mechanism="H2_mech.inp",
                   therm="therm.dat", tran="tran.dat")
    freestream = dict(mach=0.5, pressure=p0, temperature=to, Y=dict(oxidiser))
    return Case("reacting_mixing_layer_3d", mx, my, mz, X, Y, Z, delta0, faces, structs, scheme, bv, steps,
                sv=sv, mixture=mixture, freestream=freestream, extra=dict(du=du, h=h))



def spatial_mixing_layer_3d(mx=64, my=48, mz=12, seed=0, steps=20, h=0.125, delta_omega=1e-3, ma_c=0.3,
                            velocity_ratio=1.5, upper_faster=False, species=False, fluctuation_type=0,
                            intensity=0.01, inviscid_scheme=None, chem_dir=None, finite_rate=False,
                            noise=0.0) -> Case:
    """Spatially developing mixing layer (problem_type 1, the layout of the reference's shipped input):
    the two-stream inflow profile at i = 0 (u blended by tanh(2 y / delta_omega), upper / lower stream
    state by the sign of y), optionally with white noise on its velocity (fluctuation_type 1, relative
    intensity `intensity`, within |y| < 4 delta_omega) or the digital filter's turbulent fluctuations
    (fluctuation_type 11, 3-D with mz - 1 >= 50 + ngg); outflow at the other x face and both y faces;
    periodic z (3-D).  Air: upper 300 K, lower 500 K at 1 bar; species: H2/N2 fuel above (300 K) over
    air (600 K) with the 9-species mechanism, frozen unless finite_rate.  Stream Mach numbers from
    ma_c and the velocity ratio (lower stream faster unless upper_faster).  Grid in units of
    delta_omega (gridScale = delta_omega), y = (j - (my - 1) / 2) h.  The initial field is the profile
    plus `noise` dU N(0,1) exp(-(y/delta_omega)^2) seeded noise in u, v, w (noise = 0: the profile alone,
    as the reference starts a mixing-layer problem)."""
    rng = np.random.default_rng(seed)
    xs = np.arange(mx) * h
    ys = (np.arange(my) - (my - 1) / 2) * h
    zs = np.arange(mz) * h
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    if species:
        chem_dir = Path(chem_dir) if chem_dir else CHEM_FIXTURE
        tb = read_species(chem_dir, "H2_mech.inp", "therm.dat")
        upper = {"temperature": 300.0, "pressure": 101325.0, "H2": 0.1, "N2": 0.9, "mixture_fraction": 1.0}
        lower = {"temperature": 600.0, "pressure": 101325.0, "O2": 0.232, "N2": 0.768, "mixture_fraction": 0.0}
        mixture = dict(tables=tb, finite_rate=finite_rate, chem_dir=str(chem_dir), mechanism="H2_mech.inp",
                       therm="therm.dat", tran="tran.dat")
        scheme_id = inviscid_scheme or 72
    else:
        upper = {"temperature": 300.0, "pressure": 101325.0}
        lower = {"temperature": 500.0, "pressure": 101325.0}
        mixture = None
        scheme_id = inviscid_scheme or 4
    ml = dict(ma_c=ma_c, delta_omega=delta_omega, velocity_ratio=velocity_ratio, upper_faster=upper_faster,
              upper=upper, lower=lower)
    if fluctuation_type == 11:
        # the digital filter's peak Reynolds stresses R11 R12 R22 R13 R23 R33 (the reference's input values)
        ml["df_rij"] = [0.15, 0.09, 0.12, 0.05, 0.05, 0.118]
    faces = [Face((0, 0, 0, my - 1, 0, mz - 1), 5), Face((mx - 1, mx - 1, 0, my - 1, 0, mz - 1), 6),
             Face((0, mx - 1, 0, 0, 0, mz - 1), 6), Face((0, mx - 1, my - 1, my - 1, 0, mz - 1), 6)]
    if mz > 1:
        faces += [Face((0, mx - 1, 0, my - 1, 0, 0), 8), Face((0, mx - 1, 0, my - 1, mz - 1, mz - 1), 8)]
    # the inflow struct is also the reference state, as in the reference's shipped input
    structs = {"freestream": {"type": ("string", "inflow"), "label": ("int", 5), "inflow_type": ("int", 1),
                              "fluctuation_type": ("int", fluctuation_type),
                              "fluctuation_intensity": ("real", float(intensity))},
               "outflow": {"type": ("string", "outflow"), "label": ("int", 6)}}
    if mz > 1:
        structs["periodic"] = {"type": ("string", "periodic"), "label": ("int", 8)}
    recon = 5 if scheme_id in (1, 3, 4) else 2
    scheme = dict(reconstruction=recon, inviscid_scheme=scheme_id, viscous_order=2, cfl=0.5, prandtl_number=0.72,
                  limiter=0, entropy_fix_factor=0.125)
    case = Case("spatial_mixing_layer", mx, my, mz, X, Y, Z, delta_omega, faces, structs, scheme,
                np.zeros((6,) + X.shape), steps, mixture=mixture, mixing_layer=ml)
    st = case.mixing_layer_streams()
    up, lo = st["upper"], st["lower"]
    yphys = Y * delta_omega
    above = yphys >= 0
    du = abs(up[1] - lo[1])
    env = np.exp(-Y ** 2)
    bv = case.bv
    for l in (0, 4, 5):
        bv[l] = np.where(above, up[l], lo[l])
    bv[1] = 0.5 * (up[1] + lo[1]) + 0.5 * (up[1] - lo[1]) * np.tanh(2 * yphys / delta_omega)
    bv[1] += noise * du * rng.standard_normal(X.shape) * env
    bv[2] = noise * du * rng.standard_normal(X.shape) * env
    bv[3] = 0.0 if mz == 1 else noise * du * rng.standard_normal(X.shape) * env
    if species:
        ns = tb.n_spec
        case.sv = np.empty((ns,) + X.shape)
        for l in range(ns):
            case.sv[l] = np.where(above, st["y_upper"][l], st["y_lower"][l])
    case.extra = dict(du=du, h=h)
    return case

# ---- sensitivity of the momentum thickness to inflow mode amplitudes (adjoint harness)

def mode_shapes(case: Case, n_modes: int = 8, seed: int = 0, amp: float = 1e-3) -> np.ndarray:
    """v' shapes phi_m = amp du cos(2 pi m x / Lx + phase_m) exp(-y^2) (x, y in grid units, Lx the
    periodic length (mx - 1) h, the layer's own envelope), phases U[0, 2 pi) from the seed: the
    perturbation sum_m a_m phi_m added to v.  Returns [n_modes, mz, my, mx]."""
    rng = np.random.default_rng(seed)
    phases = rng.uniform(0.0, 2 * np.pi, n_modes)
    lx = (case.mx - 1) * case.extra["h"]
    env = np.exp(-case.y ** 2)
    return np.stack([amp * case.extra["du"] * np.cos(2 * np.pi * (m + 1) * case.x / lx + phases[m]) * env
                     for m in range(n_modes)])


def add_modes(case: Case, a, shapes: np.ndarray) -> Case:
    """A copy of the case with v += sum_m a_m shapes[m]."""
    c = dataclasses.replace(case, bv=case.bv.copy(), sv=None if case.sv is None else case.sv.copy())
    c.bv[2] = c.bv[2] + np.tensordot(np.asarray(a, dtype=float), shapes, axes=1)
    return c


def dcv_dmodes(cv: np.ndarray, shapes: np.ndarray) -> np.ndarray:
    """d cv / d a_m at the state cv (v enters rho v and rho E = ... + rho |V|^2 / 2):
    [n_modes, n_var, mz, my, mx]."""
    rho, v = cv[0], cv[2] / cv[0]
    out = np.zeros((shapes.shape[0],) + cv.shape)
    out[:, 2] = rho * shapes
    out[:, 4] = rho * v * shapes
    return out


def momentum_thickness(cv: np.ndarray, du: float, rho0: float, dy: float):
    """theta = 1 / (rho0 du^2) sum_y <rho> (du/2 - u~)(du/2 + u~) dy, <.> the (x, z) average and
    u~ = <rho u> / <rho> the Favre average; returns theta and d theta / d cv (zero but in rho, rho u)."""
    rm = cv[0].mean(axis=(0, 2))
    ru = cv[1].mean(axis=(0, 2))
    ut = ru / rm
    c = dy / (rho0 * du * du)
    theta = float(c * np.sum(0.25 * du * du * rm - ru * ut))
    nxz = cv.shape[1] * cv.shape[3]
    g = np.zeros_like(cv)
    g[0] = (c * (0.25 * du * du + ut * ut) / nxz)[None, :, None]
    g[1] = (c * (-2.0 * ut) / nxz)[None, :, None]
    return theta, g


def relative_errors(a: np.ndarray, b: np.ndarray, momentum_group: bool = True):
    """Per conserved variable (rho, rho u, rho v, rho w, rho E): (max-abs error / scale, L2 error / L2 scale).

    The scale of a scalar variable is its own max-abs (or L2 norm).  With momentum_group, the three
    momentum components share one scale, the momentum vector's max-abs (L2) magnitude: a transverse
    component that is only a small perturbation (rho v in a shear layer) is then measured against the
    momentum it is part of, not against its own near-zero size."""
    out = []
    mom = slice(1, 4)
    mom_max = float(np.max(np.sqrt(np.sum(b[mom] ** 2, axis=0))))
    mom_l2 = float(np.linalg.norm(b[mom]))
    for l in range(a.shape[0]):
        if momentum_group and 1 <= l <= 3:
            smax, sl2 = mom_max, mom_l2
        else:
            smax, sl2 = float(np.max(np.abs(b[l]))), float(np.linalg.norm(b[l]))
        d = a[l] - b[l]
        mx = float(np.max(np.abs(d)) / smax) if smax > 0 else float(np.max(np.abs(d)))
        l2 = float(np.linalg.norm(d) / sl2) if sl2 > 0 else float(np.linalg.norm(d))
        out.append((mx, l2))
    return out
