"""Wall and inflow faces on the GPU against the oracle, through the C ABI: no-slip walls (apply_wall,
BoundCond.cuh:1024-1270: isothermal or adiabatic, no blowing or fluctuation) on both y faces, a
constant supersonic inflow (apply_inflow, BoundCond.cuh:483-613) at i = 0 with an outflow at
i = mx - 1, and (air) a subsonic inflow with a back-pressure outflow (BoundCond.cuh:1272-1441).  RK3 trajectories of air (3-D and 2-D) and of the 9-species mixture, 1e-12 relative per
conserved variable as the other trajectory tests.
"""
import math

import numpy as np
import pytest

import ostc
import ostc_cases as oc
from oracle import Oracle

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _run(case, tmp_path, steps, mixture=False):
    d = oc.write_case(case, tmp_path / case.name)
    s = ostc.Solver(str(d))
    o = Oracle(case)
    if mixture:
        s.set_state(case.bv, sv=case.sv)
        o.set_state(case.bv, case.sv)
    else:
        s.set_state(case.bv)
        o.set_state(case.bv)
    s.step(steps)
    o.step(steps)
    cg, bg = s.get_state()
    co, bo, _ = o.get_state()
    err = oc.relative_errors(cg, co)
    assert all(m < TOL and l2 < TOL for m, l2 in err), err
    assert s.error_flags() == 0
    return bg


@pytest.mark.parametrize("thermal", ["isothermal", "adiabatic"])
def test_wall_air_3d(built, tmp_path, thermal):
    case = oc.mixing_layer_3d(mx=32, my=24, mz=16, ybc="wall", wall_thermal=thermal)
    bg = _run(case, tmp_path, 10)
    assert np.all(bg[1:4, :, 0, :] == 0) and np.all(bg[1:4, :, -1, :] == 0)
    if thermal == "isothermal":
        assert np.all(bg[5, :, 0, :] == 300.0)


@pytest.mark.parametrize("thermal,recon,rs", [("isothermal", 4, 3), ("adiabatic", 5, 4)])
def test_wall_air_2d(built, tmp_path, thermal, recon, rs):
    case = oc.mixing_layer_2d(mx=65, my=33, reconstruction=recon, inviscid_scheme=rs, ybc="wall",
                              wall_thermal=thermal)
    _run(case, tmp_path, 20)


def test_wall_mixture(built, tmp_path):
    case = oc.reacting_mixing_layer_3d(mx=20, my=16, mz=10, ybc="wall")
    bg = _run(case, tmp_path, 3, mixture=True)
    assert np.all(bg[5, :, 0, :] == 300.0)


def test_wall_rejections(built, tmp_path):
    """The radiative wall and the fluctuating walls are refused with the reason."""
    case = oc.mixing_layer_3d(mx=16, my=12, mz=8, ybc="wall")
    case.bc_structs["wall"]["thermal_type"] = ("string", "equilibrium_radiation")
    d = oc.write_case(case, tmp_path / "rad")
    with pytest.raises(ostc.OstcError, match="equilibrium_radiation"):
        ostc.Solver(str(d))
    case.bc_structs["wall"]["thermal_type"] = ("string", "isothermal")
    case.bc_structs["wall"]["fluctuation_type"] = ("int", 1)
    d = oc.write_case(case, tmp_path / "fluct")
    with pytest.raises(ostc.OstcError, match="fluctuation"):
        ostc.Solver(str(d))


@pytest.mark.parametrize("ybc", ["farfield", "wall"])
def test_inflow_air_3d(built, tmp_path, ybc):
    case = oc.mixing_layer_3d(mx=32, my=24, mz=16, xbc="inflow", ybc=ybc)
    bg = _run(case, tmp_path, 10)
    st = case.inflow_states()[5]
    # the inflow face nodes hold the inflow state; with walls, the wall (applied later, higher
    # priority) owns the corner nodes j = 0 and j = my - 1
    js = slice(1, -1) if ybc == "wall" else slice(None)
    assert np.all(bg[1, :, js, 0] == st["u"]) and np.all(bg[4, :, js, 0] == st["pressure"])
    if ybc == "wall":
        assert np.all(bg[1, :, 0, 0] == 0)


def test_inflow_mixture(built, tmp_path):
    case = oc.reacting_mixing_layer_3d(mx=20, my=16, mz=10, xbc="inflow")
    _run(case, tmp_path, 3, mixture=True)


def test_inflow_rejections(built, tmp_path):
    """Profile-file inflows and the stability-mode / receptivity fluctuations are refused with the
    reason (white noise, fluctuation_type 1, is built: tests/test_gpu_inflow.py)."""
    for key, val in (("fluctuation_type", 2), ("fluctuation_type", 3), ("inflow_type", 1)):
        case = oc.mixing_layer_3d(mx=16, my=12, mz=8, xbc="inflow")
        case.bc_structs["inflow"][key] = ("int", val)
        d = oc.write_case(case, tmp_path / f"fl_{key}_{val}")
        with pytest.raises(ostc.OstcError, match=key):
            ostc.Solver(str(d))


@pytest.mark.parametrize("ybc", ["outflow", "wall"])
def test_subsonic_inflow_back_pressure_air(built, tmp_path, ybc):
    case = oc.mixing_layer_3d(mx=32, my=24, mz=16, xbc="subsonic", ybc=ybc)
    c0 = math.sqrt(1.4 * oc.R_AIR * 300.0)
    case.bv[1] = np.abs(case.bv[1]) + 0.3 * c0  # streamwise flow into the domain everywhere, subsonic
    _run(case, tmp_path, 10)


def test_characteristic_faces_refuse_mixtures(built, tmp_path):
    case = oc.reacting_mixing_layer_3d(mx=16, my=12, mz=8)
    case.faces[1] = oc.Face(case.faces[1].raw, 9)
    case.bc_structs["back_pressure"] = {"type": ("string", "back_pressure"), "label": ("int", 9),
                                        "pressure": ("real", 101325.0)}
    d = oc.write_case(case, tmp_path / "bp")
    with pytest.raises(ostc.OstcError, match="multi-species"):
        ostc.Solver(str(d))


# ---- the same faces against the reference's own FP64 build (fixtures from tests/golden/make_golden.py:
# the reference's Driver + RK3 with its apply_wall / apply_inflow / apply_subsonic_inflow /
# apply_back_pressure, BoundCond.cuh:235-613,1024-1441), and far-field faces of mixtures (apply_farfield,
# BoundCond.cuh:755-1022)

REFERENCE_FACE_CASES = ["ml3d_wall_isothermal", "ml3d_wall_adiabatic", "ml2d_wall_isothermal_weno5",
                        "ml2d_wall_adiabatic_weno7", "ml3d_inflow_outflow", "ml3d_subsonic_backpressure", "rml3d_wall",
                        "rml3d_inflow", "rml3d_farfield_fr72", "rml3d_farfield_mix71"]


@pytest.mark.parametrize("name", REFERENCE_FACE_CASES)
def test_faces_match_reference_build(built, tmp_path, name):
    import golden_util as gu

    case, steps, z, t_ref = gu.load(gu.fixture_path(name))
    gu.check_library(case, steps, z, t_ref, tmp_path / name, name=name).close()
