"""CHEMKIN species / thermo / transport / reaction reader for the CPU oracle.

TEST INFRASTRUCTURE: an independent restatement of the reference's Species and Reaction constructors
(ChemData.cpp:11-948, element weights Element.cpp:13-31) used by the oracle to build its mixture
tables; the product has its own C++ reader.  Line handling follows the reference: section lines are
read left-trimmed and upper-cased (gxl_lib/MyString.cpp:15-50), NASA-7 coefficient lines raw in
15-column fields, the REACTIONS keyword is matched case-sensitively at the line start.
"""
from __future__ import annotations

import math
from pathlib import Path

import numpy as np

R_C = 1.98720425864083
BOLTZMANN = 1.380649e-23
ATOMIC_WEIGHT = {"H": 1.008, "HE": 4.002602, "C": 12.011, "N": 14.007, "O": 15.999, "F": 18.998403163,
                 "NE": 20.1797, "S": 32.06, "CL": 35.45, "AR": 39.95}


class Tables:
    pass


def _tokens(text):
    """Token stream with '!' comments removed up to the end of their line (file >> input)."""
    for line in text.split("\n"):
        for tok in line.split():
            if tok.startswith("!"):
                break
            yield tok


def _up(line):
    return line.lstrip().upper()


def read(input_dir, mechanism="chemistry/H2_mech.inp", therm="chemistry/therm.dat",
         tran="chemistry/tran.dat", reactions=True) -> Tables:
    d = Path(input_dir)
    mech_text = (d / mechanism).read_text()
    t = Tables()
    it = _tokens(mech_text)
    for tok in it:
        if tok in ("ELEMENTS", "ELEM"):
            break
    elems = {}
    for tok in it:
        tok = tok.upper()
        if tok == "END":
            continue
        if tok in ("SPECIES", "SPEC"):
            break
        elems.setdefault(tok, len(elems))
    spec = {}
    stop = ""
    for tok in it:
        tok = tok.upper()
        if tok == "END":
            continue
        if tok in ("REACTIONS", "REAC", "THERMO"):
            stop = tok
            break
        spec.setdefault(tok, len(spec))
    ns = len(spec)
    t.names = sorted(spec, key=spec.get)
    t.n_spec = ns
    t.mw = np.zeros(ns)
    t.t_low, t.t_mid, t.t_high = np.full(ns, 300.0), np.full(ns, 1000.0), np.full(ns, 5000.0)
    t.low, t.high = np.zeros((ns, 7)), np.zeros((ns, 7))
    if stop == "THERMO":
        raise NotImplementedError("THERMO inside the mechanism file")
    lines = (d / therm).read_text().split("\n")
    p = 0
    while p < len(lines) and not _up(lines[p]).startswith("THERMO"):
        p += 1
    p += 1
    while p < len(lines) and (not lines[p] or lines[p][0] == "!"):
        p += 1
    tl, tm, th = (float(x) for x in lines[p].split()[:3])
    p += 1
    t.t_low[:], t.t_mid[:], t.t_high[:] = tl, tm, th
    seen = set()
    while p < len(lines):
        line = _up(lines[p])
        p += 1
        if not line or line[0] == "!":
            continue
        key = line.split()[0]
        if key == "END":
            continue
        if key in ("REACTIONS", "TRANSPORT", "TRAN") or line == "REAC":
            break
        if len(seen) >= ns:
            break
        name = line[:18].split()[0] if line[:18].split() else ""
        if name not in spec or name in seen:
            p += 3 + (1 if name in spec else 0)
            continue
        sp = spec[name]
        try:
            t.t_low[sp] = float(line[45:55])
        except ValueError:
            pass
        try:
            t.t_high[sp] = float(line[55:65])
        except ValueError:
            pass
        if line[65:75].split():
            t.t_mid[sp] = float(line[65:75].split()[0])
        comp = {}
        for q in range(4):
            cs = line[24 + 5 * q: 29 + 5 * q].lstrip()
            if not cs or cs[0] == "0":
                break
            parts = cs.split()
            if parts[0] not in elems:
                continue
            comp[parts[0]] = int(parts[1]) if len(parts) > 1 else 0
        w = 0.0
        for sym in sorted(elems):
            w += ATOMIC_WEIGHT[sym] * comp.get(sym, 0)
        t.mw[sp] = w
        l2, l3, l4 = lines[p], lines[p + 1], lines[p + 2]
        p += 3
        f = lambda s, q: float(s[15 * q: 15 * q + 15])  # noqa: E731
        t.high[sp, :5] = [f(l2, q) for q in range(5)]
        t.high[sp, 5:7] = [f(l3, 0), f(l3, 1)]
        t.low[sp, :3] = [f(l3, q) for q in range(2, 5)]
        t.low[sp, 3:7] = [f(l4, q) for q in range(4)]
        seen.add(name)

    # transport (ChemData.cpp:500-597)
    eps, sigma, mu, alpha = np.zeros(ns), np.zeros(ns), np.zeros(ns), np.zeros(ns)
    t.geometry, t.lj_potent_inv, t.vis_coeff = np.zeros(ns), np.zeros(ns), np.zeros(ns)
    seen = set()
    for raw in (d / tran).read_text().split("\n"):
        line = _up(raw)
        if not line or line[0] == "!":
            continue
        parts = line.split()
        if parts[0].startswith("END") or parts[0].startswith("REAC"):
            break
        if parts[0] not in spec or parts[0] in seen:
            continue
        sp = spec[parts[0]]
        g, e, s, m, a = (float(x) for x in parts[1:6])
        t.geometry[sp], eps[sp], sigma[sp], mu[sp], alpha[sp] = g, e, s, m, a
        t.lj_potent_inv[sp] = 1.0 / e
        t.vis_coeff[sp] = 2.6693e-6 * math.sqrt(t.mw[sp]) / (s * s)
        seen.add(parts[0])
    mwv = t.mw
    t.wj_div_wi_1_4 = np.array([[math.pow(mwv[j] / mwv[i], 0.25) for j in range(ns)] for i in range(ns)])
    t.sqrt_wiwj_8 = np.array([[1.0 / math.sqrt(8 * (1 + mwv[i] / mwv[j])) for j in range(ns)] for i in range(ns)])
    conv = 1e-18 * math.sqrt(1e-7) * math.pow(1e8, 1.5) / math.sqrt(BOLTZMANN)

    def red_mu(i):
        return 0.0 if mu[i] == 0 else conv * mu[i] / math.sqrt(eps[i] * sigma[i] * sigma[i] * sigma[i])

    t.binary_diff = np.zeros((ns, ns))
    t.kb_over_eps_jk = np.zeros((ns, ns))
    for j in range(ns):
        t.binary_diff[j, j] = 0.0188324 / (math.sqrt(mwv[j] * 0.5) * sigma[j] * sigma[j])
        for k in range(j + 1, ns):
            wjk = mwv[j] * mwv[k] / (mwv[j] + mwv[k])
            xi = 1.0
            if (mu[j] != 0) != (mu[k] != 0):
                pp, nn = (j, k) if mu[j] != 0 else (k, j)
                an = alpha[nn] / math.pow(sigma[nn], 3)
                mp = red_mu(pp)
                xi = 1.0 + 0.25 * an * mp * mp * math.sqrt(eps[pp] / eps[nn])
            sjk = 0.5 * (sigma[j] + sigma[k]) * math.pow(xi, -1.0 / 6.0)
            t.binary_diff[j, k] = t.binary_diff[k, j] = 0.0188324 / (math.sqrt(wjk) * sjk * sjk)
            t.kb_over_eps_jk[j, k] = t.kb_over_eps_jk[k, j] = 1.0 / (xi * xi * math.sqrt(eps[j] * eps[k]))

    t.n_reac = 0
    if reactions:
        _read_reactions(t, spec, mech_text)
    return t


def _side(s, spec, st, sign):
    order = 0
    while s:
        p = s.find("+")
        if p != -1 and p + 1 < len(s) and s[p + 1] == "+":
            p += 1
        term, s = (s, "") if p == -1 else (s[:p], s[p + 1:])
        nu = 1
        if term and term[0].isdigit():
            nu, term = int(term[0]), term[1:]
        st[spec[term]] += nu
        order += sign * nu
    return order


def _read_reactions(t, spec, text):
    ns = t.n_spec
    lines = text.split("\n")
    p = 0
    while p < len(lines):
        tl = lines[p].lstrip()
        p += 1
        if tl.startswith("REACTIONS") or tl.startswith("REAC"):
            break
    R = []
    dups = []

    def getline():
        nonlocal p
        if p >= len(lines):
            return None
        s = _up(lines[p])
        p += 1
        return s

    line = getline() or "END"
    while line is not None and line != "END":
        if not line or line[0] == "!":
            line = getline()
            continue
        r = dict(label=1, rev_type=0, order=0, sf=np.zeros(ns, int), sb=np.zeros(ns, int), A=0.0, b=0.0, Ea=0.0,
                 A2=0.0, b2=0.0, Ea2=0.0, tb=np.ones(ns), ta=0.0, t3=0.0, t1=0.0, t2=0.0)
        eqline = line
        if "+M" in eqline:
            r["label"] = 4
            lp = eqline.find("(+")
            if lp != -1:
                r["label"] = 5
                eqline = eqline[:lp] + eqline[eqline.find(")", lp) + 1:]
                lp = eqline.find("(+")
                eqline = eqline[:lp] + eqline[eqline.rfind(")") + 1:]
            else:
                q = eqline.find("+M")
                eqline = eqline[:q] + eqline[q + 2:]
                q = eqline.find("+M")
                eqline = eqline[:q] + eqline[q + 2:]
        lt = eqline.find("<")
        if lt == -1:
            lt = eqline.find("=")
        eqline = eqline[:lt + 1].replace(" ", "<") + eqline[lt + 1:]
        parts = eqline.split()
        eq = parts[0]
        r["A"], r["b"], r["Ea"] = float(parts[1]), float(parts[2]), float(parts[3]) / R_C
        small, e, big = eq.find("<"), eq.find("="), eq.find(">")
        if small == -1:
            if big != -1:
                r["label"] = 0
            else:
                big = e
            small = e
        r["order"] = _side(eq[:small], spec, r["sf"], -1) + _side(eq[big + 1:], spec, r["sb"], +1)
        dup = False
        line = None
        while True:
            aux = getline()
            if aux is None:
                break
            a = aux.replace("/", " ")
            toks = a.split()
            if not aux or aux[0] == "!":
                continue
            key = toks[0] if toks else ""
            if key == "END" or "=" in aux:
                line = "END" if key == "END" else aux
                break
            if key == "PLOG":
                continue
            if key in ("DUPLICATE", "DUP"):
                dup = True
                r["label"] = 3
                continue
            if key in ("REV", "LOW"):
                r["A2"], r["b2"], r["Ea2"] = float(toks[1]), float(toks[2]), float(toks[3]) / R_C
                if key == "REV":
                    r["rev_type"] = 1
            elif key == "TROE":
                r["label"] = 6
                r["ta"], r["t3"], r["t1"] = float(toks[1]), float(toks[2]), float(toks[3])
                if len(toks) > 4:
                    r["t2"] = float(toks[4])
                    r["label"] = 7
            else:
                for q in range(0, len(toks) - 1, 2):
                    r["tb"][spec[toks[q]]] = float(toks[q + 1])
        if dup:
            hit = None
            for q, di in enumerate(dups):
                if np.array_equal(R[di]["sf"], r["sf"]) and np.array_equal(R[di]["sb"], r["sb"]):
                    hit = q
                    break
            if hit is not None:
                di = dups.pop(hit)
                R[di]["A2"], R[di]["b2"], R[di]["Ea2"] = r["A"], r["b"], r["Ea"]
                continue
            dups.append(len(R))
        R.append(r)
    nr = len(R)
    t.n_reac = nr
    t.label = np.array([r["label"] for r in R], dtype=np.int32)
    t.rev_type = np.array([r["rev_type"] for r in R], dtype=np.int32)
    t.order = np.array([r["order"] for r in R], dtype=np.int32)
    t.stoi_f = np.array([r["sf"] for r in R], dtype=np.int32).reshape(nr, ns)
    t.stoi_b = np.array([r["sb"] for r in R], dtype=np.int32).reshape(nr, ns)
    for k in ("A", "b", "Ea", "A2", "b2", "Ea2"):
        setattr(t, k, np.array([r[k] for r in R]))
    t.third_body = np.array([r["tb"] for r in R]).reshape(nr, ns)
    t.troe_alpha = np.array([r["ta"] for r in R])
    t.troe_t3 = np.array([r["t3"] for r in R])
    t.troe_t1 = np.array([r["t1"] for r in R])
    t.troe_t2 = np.array([r["t2"] for r in R])
