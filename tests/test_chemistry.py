"""Host-side checks of the chemistry restatements (no GPU): the CHEMKIN readers agree, the
point-implicit treatment tends to the explicit one as dt -> 0, and the reacting case conserves
element mass through the chemical source."""
import numpy as np
import pytest

import ostc_cases as oc
from oracle import Oracle


def test_h2_mechanism_tables(built):
    case = oc.reacting_mixing_layer_3d(mx=8, my=8, mz=6)
    t = Oracle(case).tables
    assert case.mixture["tables"].names == t.names
    assert np.array_equal(case.mixture["tables"].mw, t.mw)
    assert np.array_equal(case.mixture["tables"].low, t.low) and np.array_equal(case.mixture["tables"].high, t.high)
    assert t.n_spec == 9 and t.n_reac == 19  # 21 reactions, two DUPLICATE pairs merged
    assert t.names == ["H", "H2", "H2O", "H2O2", "HO2", "O", "O2", "OH", "N2"]
    # Troe fall-off reactions (label 6) and third-body reactions (label 4) of the mechanism
    assert int(np.sum(t.label == 6)) == 2 and int(np.sum(t.label == 4)) == 4 and int(np.sum(t.label == 3)) == 2
    # molecular weights from the element table
    assert abs(t.mw[t.names.index("H2O")] - (2 * 1.008 + 15.999)) < 1e-12


def test_chemical_source_conserves_mass(built):
    """sum_k omega_k = 0: the source moves mass between species and creates none."""
    case = oc.reacting_mixing_layer_3d(mx=10, my=12, mz=6)
    o = Oracle(case)
    o.set_state(case.bv)
    dq = o.rhs(4)
    s = dq[5:].sum(axis=0)
    assert np.max(np.abs(s)) <= 1e-9 * np.max(np.abs(dq[5:]))


def test_point_implicit_reduces_to_explicit(built):
    """Before any step the oracle's step size is 0, so (I - dt J) is the identity and the
    point-implicit RHS (source added after the fluxes) equals the explicit one to rounding."""
    case = oc.reacting_mixing_layer_3d(mx=10, my=12, mz=6)
    oe = Oracle(case)
    oe.set_state(case.bv)
    oi = Oracle(case, chem_mode=1)
    oi.set_state(case.bv)
    de = oe.rhs(7)
    di = oi.rhs(7)
    assert np.allclose(di, de, rtol=1e-12, atol=1e-12 * np.max(np.abs(de)))


def _element_matrix(names):
    """Atoms of H, O, N per species from the formula names of the mechanism (H2O2 -> H 2, O 2)."""
    import re

    elems = ["H", "O", "N"]
    m = np.zeros((len(elems), len(names)))
    for k, n in enumerate(names):
        for sym, cnt in re.findall(r"([A-Z][a-z]?)(\d*)", n):
            m[elems.index(sym), k] += int(cnt) if cnt else 1
    return m


def test_chemical_source_conserves_elements(built):
    """sum_k a_ek omega_k / W_k = 0 for the elements H, O, N: reactions rearrange atoms only."""
    case = oc.reacting_mixing_layer_3d(mx=10, my=12, mz=6)
    t = case.mixture["tables"]
    o = Oracle(case)
    o.set_state(case.bv)
    w = o.rhs(4)[5:]  # J omega_k
    a = _element_matrix(t.names) / np.asarray(t.mw)[None, :]
    moles = np.einsum("ek,k...->e...", a, w)
    scale = np.einsum("ek,k...->e...", a, np.abs(w))
    assert np.all(np.abs(moles) <= 1e-12 * np.max(scale, axis=tuple(range(1, scale.ndim)), keepdims=True)), \
        np.max(np.abs(moles))
