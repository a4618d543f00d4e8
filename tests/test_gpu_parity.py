"""GPU parity of the RHS and SSP-RK3 path against the CPU oracle, through the C ABI.

Tolerance: the plain FP64 path must match the oracle to 1e-12 relative, per conserved variable, in the
max norm and in L2 (ostc_cases.relative_errors: scalars against their own magnitude, momentum
components against the momentum magnitude).  The remaining differences are FMA contraction and libm
rounding in CUDA, both present in the reference's own CUDA build as well.
"""
import numpy as np
import pytest

import ostc
import ostc_cases as oc
from oracle import Oracle

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _pair(case, tmp_path):
    d = oc.write_case(case, tmp_path / case.name)
    s = ostc.Solver(str(d))
    s.set_state(case.bv)
    o = Oracle(case)
    o.set_state(case.bv)
    return s, o


def _rel(a, b, floor=0.0):
    out = []
    for l in range(a.shape[0]):
        scale = max(np.max(np.abs(b[l])), floor)
        out.append(0.0 if scale == 0 else float(np.max(np.abs(a[l] - b[l])) / scale))
    return out


@pytest.mark.parametrize("dims,recon,rs", [((65, 33, 1), 4, 3), ((65, 33, 1), 5, 4), ((40, 24, 20), 5, 4),
                                           ((36, 20, 16), 4, 3)])
def test_rhs_terms(built, tmp_path, dims, recon, rs):
    mx, my, mz = dims
    if mz == 1:
        case = oc.mixing_layer_2d(mx=mx, my=my, reconstruction=recon, inviscid_scheme=rs)
    else:
        case = oc.mixing_layer_3d(mx=mx, my=my, mz=mz, reconstruction=recon, inviscid_scheme=rs)
    s, o = _pair(case, tmp_path)
    for mask in (1, 2, 3):
        dg = s.rhs(mask)
        dc = o.rhs(mask)
        # scale by the largest |dq| of the momentum/energy group: dq[0] is tiny for viscous-only
        floor = np.max(np.abs(dc))
        err = _rel(dg, dc, floor * 1e-6)
        assert max(err) < TOL * 100, (mask, err)


def test_initial_state_and_dt(built, tmp_path):
    case = oc.mixing_layer_3d(mx=40, my=24, mz=20)
    s, o = _pair(case, tmp_path)
    cg, bg = s.get_state()
    co, bo, _ = o.get_state()
    assert max(_rel(cg, co)) < 1e-14
    assert max(_rel(bg, bo)) < 1e-14
    dt_g = s.step(1)
    o.step(1)
    assert abs(dt_g - o.time()) / o.time() < 1e-13


@pytest.mark.parametrize("dims,recon,rs,steps", [((65, 33, 1), 4, 3, 100), ((65, 33, 1), 5, 4, 50),
                                                 ((40, 24, 20), 5, 4, 20), ((36, 20, 16), 4, 3, 20)])
def test_rk3_trajectory(built, tmp_path, dims, recon, rs, steps):
    mx, my, mz = dims
    if mz == 1:
        case = oc.mixing_layer_2d(mx=mx, my=my, reconstruction=recon, inviscid_scheme=rs)
    else:
        case = oc.mixing_layer_3d(mx=mx, my=my, mz=mz, reconstruction=recon, inviscid_scheme=rs)
    s, o = _pair(case, tmp_path)
    s.step(steps)
    o.step(steps)
    cg, bg = s.get_state()
    co, bo, _ = o.get_state()
    err = oc.relative_errors(cg, co)
    assert all(m < TOL and l2 < TOL for m, l2 in err), err
    assert abs(s.time() - o.time()) / o.time() < 1e-12
    assert s.error_flags() == 0


def test_mixed_precision_accuracy(built, tmp_path):
    """Mixed path (FP32 reconstruction/Riemann/viscous arithmetic, FP64 state and EOS) against the
    FP64 path after 100 steps: relative L2 error of the conserved variables <= 1e-6."""
    case = oc.mixing_layer_3d(mx=96, my=64, mz=48)
    d = oc.write_case(case, tmp_path / "mixed")
    a = ostc.Solver(str(d))
    a.set_state(case.bv)
    b = ostc.Solver(str(d))
    b.set_precision(ostc.PREC_MIXED)
    b.set_state(case.bv)
    a.step(100)
    b.step(100)
    ca, _ = a.get_state()
    cb, _ = b.get_state()
    err = oc.relative_errors(cb, ca)
    assert b.error_flags() == 0
    assert all(l2 <= 1e-6 for _, l2 in err), err


def test_device_flags_clean_and_residual(built, tmp_path):
    case = oc.mixing_layer_2d(mx=65, my=33)
    d = oc.write_case(case, tmp_path / "res")
    s = ostc.Solver(str(d))
    s.set_state(case.bv)
    s.store_residual_reference()
    _, b0 = s.get_state()
    s.step(3)
    _, b1 = s.get_state()
    res = s.residual()
    v0 = np.sqrt(b0[1] ** 2 + b0[2] ** 2 + b0[3] ** 2)
    v1 = np.sqrt(b1[1] ** 2 + b1[2] ** 2 + b1[3] ** 2)
    ref = np.sqrt([np.mean((b1[0] - b0[0]) ** 2), np.mean((v1 - v0) ** 2), np.mean((b1[4] - b0[4]) ** 2),
                   np.mean((b1[5] - b0[5]) ** 2)])
    assert np.allclose(res, ref, rtol=1e-10, atol=0)
    assert s.error_flags() == 0


@pytest.mark.parametrize("what", ["nan_temperature", "negative_pressure"])
def test_bad_state_raises_device_flag(built, tmp_path, what):
    """Fault detection without a GPU fault: a state seeded with a NaN temperature (or a negative
    pressure) at one interior node is stepped; the update kernel raises its device flag, the step
    returns OSTC_ENUMERIC, and ostc_error_flags reports and clears the flag."""
    import ostc

    case = oc.mixing_layer_3d(mx=24, my=16, mz=8)
    if what == "nan_temperature":
        case.bv[5, 4, 8, 12] = np.nan
    else:
        case.bv[4, 4, 8, 12] = -case.bv[4, 4, 8, 12]
    d = oc.write_case(case, tmp_path / "case")
    s = ostc.Solver(str(d))
    s.set_state(case.bv)
    with pytest.raises(ostc.OstcError) as e:
        s.step(1)
    assert e.value.code == -6  # OSTC_ENUMERIC
    flags = s.error_flags()
    assert flags & (ostc.FLAG_NAN | ostc.FLAG_NONPOSITIVE)
    assert s.error_flags() == 0  # read and cleared


@pytest.mark.parametrize("mixture", [False, True], ids=["air", "mixture"])
def test_run_states_matches_one_at_a_time(built, tmp_path, mixture):
    """ostc_run_states (independent states, copies overlapped with the steps) gives bitwise the
    states that set_state + step + get_state give one at a time."""
    case = (oc.reacting_mixing_layer_3d(mx=24, my=18, mz=12) if mixture else oc.mixing_layer_3d(mx=32, my=24, mz=16))
    d = oc.write_case(case, tmp_path / "case")
    s = ostc.Solver(str(d))
    rng = np.random.default_rng(5)
    states = []
    for m in range(3):
        bv = case.bv.copy()
        bv[2] *= 1 + 0.1 * m
        bv[1] += 0.01 * rng.standard_normal(bv[1].shape)
        states.append((bv, None if case.sv is None else case.sv.copy()))
    got = s.run_states([b for b, _ in states], 2, None if not mixture else [x for _, x in states])
    for (bv, sv), (gb, gs) in zip(states, got):
        s.set_state(bv, sv=sv)
        s.step(2)
        _, rb = s.get_state()
        assert np.array_equal(gb, rb)
        if mixture:
            assert np.array_equal(gs, s.get_species())
