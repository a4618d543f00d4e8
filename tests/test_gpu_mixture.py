"""The multi-component path (species = 1) on the GPU against the CPU oracle, through the C ABI: the
9-species H2/air mechanism with finite-rate chemistry (MixtureModel FR) or without (Mixture), the
flux-split characteristic WENO7-Z (inviscid_scheme 72) or component-wise WENO7-Z (71), or the primitive
reconstructions (1st order, MUSCL, NND2) with the mixture AUSM+, HLLC and Roe solvers, mixture transport
and the temperature Newton iteration.

Tolerance: 1e-12 relative per conserved variable (max norm; momentum against the momentum magnitude)
for the RHS terms and for RK3 trajectories; the physical time to 1e-13.
"""
import numpy as np
import pytest

import ostc_cases as oc
from oracle import Oracle

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _pair(case, tmp_path):
    import ostc

    d = oc.write_case(case, tmp_path / "case")
    s = ostc.Solver(str(d))
    s.set_state(case.bv, sv=case.sv)
    o = Oracle(case)
    o.set_state(case.bv)
    return s, o


def _rel(a, b, floor=0.0):
    return [0.0 if max(np.max(np.abs(b[l])), floor) == 0 else
            float(np.max(np.abs(a[l] - b[l])) / max(np.max(np.abs(b[l])), floor)) for l in range(a.shape[0])]


PV_SCHEMES = [dict(inviscid_scheme=3, reconstruction=2), dict(inviscid_scheme=4, reconstruction=3, finite_rate=False),
              dict(inviscid_scheme=2, reconstruction=1), dict(inviscid_scheme=2, reconstruction=2),
              dict(inviscid_scheme=4, reconstruction=1), dict(inviscid_scheme=3, reconstruction=3)]
PV_IDS = ["muscl_ausm", "nnd_hllc_frozen", "first_roe", "muscl_roe", "first_hllc", "nnd_ausm"]


@pytest.mark.parametrize("kw", [dict(inviscid_scheme=72), dict(inviscid_scheme=72, finite_rate=False),
                                dict(inviscid_scheme=71)] + PV_SCHEMES, ids=["fr72", "mix72", "fr71"] + PV_IDS)
def test_mixture_rhs_terms(built, tmp_path, kw):
    case = oc.reacting_mixing_layer_3d(mx=24, my=18, mz=12, **kw)
    s, o = _pair(case, tmp_path)
    cg, _ = s.get_state()
    co, _, _ = o.get_state()
    assert max(_rel(cg, co)) < 1e-13
    for mask in (4, 1, 2, 7):
        dg, dc = s.rhs(mask), o.rhs(mask)
        if not np.any(dc):
            assert not np.any(dg)
            continue
        err = _rel(dg, dc, np.max(np.abs(dc)) * 1e-9)
        assert max(err) < TOL * 100, (mask, err)


@pytest.mark.parametrize("dims,kw,steps", [((24, 18, 12), dict(inviscid_scheme=72), 10),
                                           ((24, 18, 12), dict(inviscid_scheme=71, finite_rate=False), 10),
                                           ((40, 24, 1), dict(inviscid_scheme=72), 20),
                                           ((24, 18, 12), PV_SCHEMES[0], 10), ((24, 18, 12), PV_SCHEMES[1], 10),
                                           ((24, 18, 12), PV_SCHEMES[2], 10), ((40, 24, 1), PV_SCHEMES[3], 20),
                                           ((40, 24, 1), PV_SCHEMES[1], 20)],
                         ids=["fr72_3d", "mix71_3d", "fr72_2d", "muscl_ausm_3d", "nnd_hllc_3d", "first_roe_3d",
                              "muscl_roe_2d", "nnd_hllc_2d"])
def test_mixture_trajectory(built, tmp_path, dims, kw, steps):
    mx, my, mz = dims
    case = oc.reacting_mixing_layer_3d(mx=mx, my=my, mz=mz, **kw)
    s, o = _pair(case, tmp_path)
    s.step(steps)
    o.step(steps)
    cg, bg = s.get_state()
    co, bo, _ = o.get_state()
    err = oc.relative_errors(cg, co)
    assert all(m < TOL and l2 < TOL for m, l2 in err), err
    assert abs(s.time() - o.time()) <= 1e-13 * o.time()
    sg = s.get_species()
    assert np.max(np.abs(sg - o.mixture()["sv"])) < 1e-12
    assert s.error_flags() == 0


@pytest.mark.parametrize("dims,steps", [((24, 18, 12), 10), ((40, 24, 1), 20)], ids=["3d", "2d"])
def test_point_implicit_chemistry_matches_oracle(built, tmp_path, dims, steps):
    """Chem mode 1 (extension): the batched per-cell 9x9 column-pivoted LU of (I - dt J_chem) on the
    GPU against the oracle's restatement of EPI / solve_chem_system."""
    import ostc

    mx, my, mz = dims
    case = oc.reacting_mixing_layer_3d(mx=mx, my=my, mz=mz)
    d = oc.write_case(case, tmp_path / "case")
    s = ostc.Solver(str(d))
    s.set_chem_mode(ostc.CHEM_POINT_IMPLICIT)
    s.set_state(case.bv, sv=case.sv)
    o = Oracle(case, chem_mode=1)
    o.set_state(case.bv)
    s.step(steps)
    o.step(steps)
    cg, _ = s.get_state()
    co, _, _ = o.get_state()
    err = oc.relative_errors(cg, co)
    assert all(m < TOL and l2 < TOL for m, l2 in err), err
    assert s.error_flags() == 0


@pytest.mark.parametrize("kw", [dict(inviscid_scheme=72), dict(inviscid_scheme=71, finite_rate=False)],
                         ids=["fr72", "mix71"])
def test_mixture_mixed_precision(built, tmp_path, kw):
    """Mixed precision on the multi-component path (FP32 split fluxes, viscous fluxes and transport
    properties; FP64 state, Newton temperature and chemistry) against the FP64 path after 12 steps:
    relative L2 error per conserved variable (momentum components against the momentum magnitude),
    every species density rho*Y_k included, below 1e-5, and the species mass fractions within 1e-6
    absolute."""
    import ostc

    case = oc.reacting_mixing_layer_3d(mx=40, my=32, mz=16, **kw)
    d = oc.write_case(case, tmp_path / "case")
    out = {}
    for prec in (ostc.PREC_FP64, ostc.PREC_MIXED):
        s = ostc.Solver(str(d))
        s.set_precision(prec)
        s.set_state(case.bv, sv=case.sv)
        s.step(12)
        cv, _ = s.get_state()
        out[prec] = (cv, s.get_species(), s.error_flags())
    (c64, y64, f64), (c32, y32, f32) = out[ostc.PREC_FP64], out[ostc.PREC_MIXED]
    assert f64 == 0 and f32 == 0
    l2 = [e[1] for e in oc.relative_errors(c32, c64)]
    assert max(l2) < 1e-5, l2
    assert np.max(np.abs(y32 - y64)) < 1e-6


def test_chemical_source_conserves_elements_gpu(built, tmp_path):
    """The product's chemical source rearranges atoms only: sum_k a_ek omega_k / W_k = 0 (H, O, N)."""
    import re

    import ostc

    case = oc.reacting_mixing_layer_3d(mx=16, my=12, mz=8)
    t = case.mixture["tables"]
    d = oc.write_case(case, tmp_path / "case")
    s = ostc.Solver(str(d))
    s.set_state(case.bv, sv=case.sv)
    w = s.rhs(4)[5:]
    elems = ["H", "O", "N"]
    a = np.zeros((3, len(t.names)))
    for k, n in enumerate(t.names):
        for sym, cnt in re.findall(r"([A-Z][a-z]?)(\d*)", n):
            a[elems.index(sym), k] += int(cnt) if cnt else 1
    a /= np.asarray(t.mw)[None, :]
    moles = np.einsum("ek,k...->e...", a, w)
    scale = np.einsum("ek,k...->e...", a, np.abs(w)).max(axis=(1, 2, 3))
    assert np.all(np.abs(moles).max(axis=(1, 2, 3)) <= 1e-12 * scale)


def test_temperature_newton_round_trip(built, tmp_path):
    """e(T) -> T: the conservative state of a known (rho, u, p, T, Y) set back through the Newton
    iteration (ostc_set_conservative) started 20 % off recovers T and p to 1e-6: the iteration stops
    once a correction is below 1e-3 relative (FieldOperation.cu:19-37), after which the quadratic
    convergence leaves at most ~1e-6."""
    import ostc

    case = oc.reacting_mixing_layer_3d(mx=16, my=12, mz=8)
    d = oc.write_case(case, tmp_path / "case")
    s = ostc.Solver(str(d))
    s.set_state(case.bv, sv=case.sv)
    cv0, bv0 = s.get_state()
    off = case.bv.copy()
    off[5] *= 1.2
    s.set_state(off, sv=case.sv)
    s.set_conservative(cv0)
    _, bv1 = s.get_state()
    assert np.max(np.abs(bv1[5] / bv0[5] - 1)) < 1e-6
    assert np.max(np.abs(bv1[4] / bv0[4] - 1)) < 1e-6
