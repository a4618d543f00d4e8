"""The primitive-reconstruction schemes (1st order / MUSCL / NND2 with Lax-Friedrichs, Roe, AUSM+ or
HLLC: inviscid_type 0 and 2 of the reference) and the AWENO variants with Lax-Friedrichs, on the GPU
against the CPU oracle, through the C ABI; plus their host-side properties on the CPU.

Tolerance as in test_gpu_parity: 1e-12 relative per conserved variable (max norm) for the FP64 path.
The mixed path (FP32 fluxes, FP64 state) is checked at 1e-5 relative after a few steps.
"""
import numpy as np
import pytest

import ostc_cases as oc
from oracle import Oracle

TOL = 1e-12

# (reconstruction, inviscid_scheme): MUSCL/NND/1st order with every solver, AWENO with LF, and
# AWENO with inviscid_scheme 2, which the reference runs as AUSM+ (inviscid_type 1 wins)
SCHEMES = [(1, 3), (2, 2), (3, 4), (2, 1), (1, 2), (3, 3), (2, 4), (4, 1), (5, 1), (5, 2)]


def _case(dims, recon, rs, **kw):
    mx, my, mz = dims
    if mz == 1:
        return oc.mixing_layer_2d(mx=mx, my=my, reconstruction=recon, inviscid_scheme=rs, **kw)
    return oc.mixing_layer_3d(mx=mx, my=my, mz=mz, reconstruction=recon, inviscid_scheme=rs, **kw)


def _rel(a, b, floor=0.0):
    out = []
    for l in range(a.shape[0]):
        scale = max(np.max(np.abs(b[l])), floor)
        out.append(0.0 if scale == 0 else float(np.max(np.abs(a[l] - b[l])) / scale))
    return out


@pytest.mark.parametrize("recon,rs", [(1, 3), (2, 2), (3, 4), (2, 1)])
def test_oracle_uniform_flow_is_steady(built, recon, rs):
    """Free-stream preservation: a uniform state on a uniform grid has a zero inviscid RHS away from
    the far-field faces (the sweeps difference identical face fluxes)."""
    case = oc.mixing_layer_3d(mx=12, my=10, mz=8, reconstruction=recon, inviscid_scheme=rs, ybc="outflow")
    case.bv[1], case.bv[2], case.bv[3] = 100.0, 30.0, -20.0
    o = Oracle(case)
    o.set_state(case.bv)
    dq = o.rhs(1)
    assert np.max(np.abs(dq)) < 1e-12 * np.max(np.abs(case.bv[4]))


@pytest.mark.parametrize("recon,rs", [(2, 2), (3, 1), (1, 4), (2, 3)])
def test_oracle_periodic_conservation(built, recon, rs):
    """A state that varies along the periodic x only: the y and z sweeps vanish and the x sweep
    telescopes, so the RHS summed over one period (nodes 0..mx-2; node mx-1 duplicates node 0)
    vanishes to rounding for every conserved variable."""
    case = oc.mixing_layer_3d(mx=17, my=8, mz=6, reconstruction=recon, inviscid_scheme=rs, ybc="outflow")
    ph = 2 * np.pi * np.arange(case.mx) / (case.mx - 1)
    rho0, p0 = case.bv[0].mean(), case.bv[4].mean()
    case.bv[0] = rho0 * (1 + 0.2 * np.sin(ph))
    case.bv[1] = 80.0 * np.cos(ph) + 20.0
    case.bv[2] = 10.0 * np.sin(2 * ph)
    case.bv[3] = -5.0
    case.bv[4] = p0 * (1 + 0.1 * np.cos(3 * ph))
    case.bv[5] = case.bv[4] / (case.bv[0] * oc.R_AIR)
    o = Oracle(case)
    o.set_state(case.bv)
    dq = o.rhs(1)
    for l in range(5):
        total = np.abs(np.sum(dq[l][:, :, : case.mx - 1], axis=2)).max()
        assert total <= 1e-12 * np.abs(dq[l]).max() * case.mx + 1e-300, (l, total)


@pytest.mark.gpu
@pytest.mark.parametrize("recon,rs", SCHEMES)
@pytest.mark.parametrize("dims", [(65, 33, 1), (36, 20, 16)])
def test_gpu_rhs_matches_oracle(built, tmp_path, dims, recon, rs):
    import ostc

    case = _case(dims, recon, rs)
    d = oc.write_case(case, tmp_path / "case")
    s = ostc.Solver(str(d))
    s.set_state(case.bv)
    o = Oracle(case)
    o.set_state(case.bv)
    for mask in (1, 3):
        dg, dc = s.rhs(mask), o.rhs(mask)
        err = _rel(dg, dc, np.max(np.abs(dc)) * 1e-6)
        assert max(err) < TOL * 100, (mask, err)


@pytest.mark.gpu
@pytest.mark.parametrize("recon,rs", SCHEMES)
@pytest.mark.parametrize("dims,steps", [((65, 33, 1), 40), ((36, 20, 16), 10)])
def test_gpu_trajectory_matches_oracle(built, tmp_path, dims, steps, recon, rs):
    import ostc

    case = _case(dims, recon, rs)
    d = oc.write_case(case, tmp_path / "case")
    s = ostc.Solver(str(d))
    s.set_state(case.bv)
    o = Oracle(case)
    o.set_state(case.bv)
    s.step(steps)
    o.step(steps)
    cg, _ = s.get_state()
    co, _, _ = o.get_state()
    err = oc.relative_errors(cg, co)
    assert all(m < TOL and l2 < TOL for m, l2 in err), err
    assert abs(s.time() - o.time()) <= 1e-13 * o.time()
    assert s.error_flags() == 0


@pytest.mark.gpu
@pytest.mark.parametrize("recon,rs", [(2, 2), (3, 4), (1, 1)])
def test_gpu_mixed_precision_low_order(built, tmp_path, recon, rs):
    import ostc

    case = _case((36, 20, 16), recon, rs)
    d = oc.write_case(case, tmp_path / "case")
    s = ostc.Solver(str(d))
    s.set_precision(ostc.PREC_MIXED)
    s.set_state(case.bv)
    o = Oracle(case)
    o.set_state(case.bv)
    s.step(10)
    o.step(10)
    cg, _ = s.get_state()
    co, _, _ = o.get_state()
    err = oc.relative_errors(cg, co)
    assert all(l2 < 1e-5 for _, l2 in err), err
