"""The steady driver (ostc_steady_step: the reference's steady_simulation, SteadySim.cuh:15-140) and dual time
stepping (ostc_dual_time_step: dual_time_stepping, DualTimeStepping.cuh:32-252) on the GPU.

* Against the reference's own FP64 build: fixtures golden_st_*.npz (tests/golden/make_golden.py) hold
  the state the reference reached after its steady iterations - air 3-D explicit and DPLUR, air 2-D
  DPLUR, the 9-species H2/air layer with the chemical source point-implicit (EPI), diagonal (DA),
  DPLUR + EPI and DPLUR with explicit chemistry, and the non-reacting mixture with DPLUR - compared
  at 1e-12 relative per conserved variable.
* Against the oracle's restatement (oracle/ostc_oracle.c orc_steady): DPLUR with no-slip walls (whose
  dq is zeroed on the wall nodes; the reference's own wall zeroing writes outside its array and defines
  no result to match) and DPLUR + DA.
* Dual time stepping against the reference build (fixtures golden_dt_*.npz: air 3-D and 2-D, the
  9-species layer with EPI chemistry; BDF2 physical steps, DPLUR pseudo-time iterations whose count
  adapts every second step) and the adapted inner-iteration count against the oracle's.
* The convergence stop of the reference (residual scaled by that of the first iteration, checked after
  iteration 1 and every output_screen-th) and the mixed-precision steady iteration against FP64.
"""
import numpy as np
import pytest

import golden_util as gu
import ostc
import ostc_cases as oc
from oracle import Oracle

pytestmark = pytest.mark.gpu

STEADY = dict(steady=1, implicit_method=0, dplur_inner_step=3, chem_src_method=0, convergence_criteria=1e-300)
DUAL = dict(steady=0, temporal_scheme=2, implicit_method=1, dplur_inner_step=2, inner_iteration=4,
            max_inner_iteration=8, iteration_adjust_step=2)
REFERENCE_STEADY = ["st_ml3d_explicit", "st_ml3d_dplur", "st_ml2d_dplur", "st_rml3d_epi", "st_rml3d_da",
                    "st_rml3d_dplur_epi", "st_rml3d_dplur_explicit", "st_rml3d_mix_dplur"]


@pytest.mark.parametrize("name", REFERENCE_STEADY)
def test_steady_matches_reference_build(built, tmp_path, name):
    case, steps, z, t_ref = gu.load(gu.fixture_path(name))
    s = gu.check_library(case, steps, z, t_ref, tmp_path / name)
    assert s.time() == 0.0  # the steady driver does not advance the physical time
    s.close()


@pytest.mark.parametrize("kind", ["air_wall_dplur", "mixture_dplur_da"])
def test_steady_matches_oracle(built, tmp_path, kind):
    if kind == "air_wall_dplur":
        case = oc.mixing_layer_3d(mx=24, my=20, mz=12, ybc="wall",
                                  steady=dict(STEADY, implicit_method=1, dplur_inner_step=2))
        n = 8
    else:
        case = oc.reacting_mixing_layer_3d(mx=16, my=12, mz=8, steady=dict(STEADY, implicit_method=1, chem_src_method=2))
        n = 4
    s = gu.run_library(case, n, tmp_path / kind)
    o = Oracle(case)
    o.set_state(case.bv)
    o.steady(n)
    err = oc.relative_errors(s.get_state()[0], o.get_state()[0])
    assert all(m < gu.TOL and l2 < gu.TOL for m, l2 in err), err
    assert s.error_flags() == 0
    s.close()


def test_steady_convergence_stop(built, tmp_path):
    # the scaled residual of iteration 1 is 1 by definition: a criterion above it stops there
    case = oc.mixing_layer_3d(mx=24, my=20, mz=12, ybc="outflow", steady=dict(STEADY, convergence_criteria=2.0))
    d = oc.write_case(case, tmp_path / "stop")
    s = ostc.Solver(str(d))
    s.set_state(case.bv)
    done, err = s.steady(10)
    assert (done, err) == (1, 1.0)
    s.close()
    # with a tiny criterion every requested iteration runs; the residual falls below its first value
    case = oc.mixing_layer_3d(mx=24, my=20, mz=12, ybc="outflow", steady=STEADY)
    d = oc.write_case(case, tmp_path / "run")
    (d / "setup.txt").write_text((d / "setup.txt").read_text() + "int output_screen = 5\n")
    s = ostc.Solver(str(d))
    s.set_state(case.bv)
    done, err = s.steady(10)
    assert done == 10 and 0 < err < 1.0, (done, err)
    s.close()


def test_steady_mixed_precision(built, tmp_path):
    case = oc.mixing_layer_3d(mx=40, my=24, mz=16, steady=dict(STEADY, implicit_method=1))
    d = oc.write_case(case, tmp_path / "mix")
    out = []
    for prec in (ostc.PREC_FP64, ostc.PREC_MIXED):
        s = ostc.Solver(str(d))
        s.set_precision(prec)
        s.set_state(case.bv)
        s.steady(10)
        out.append(s.get_state()[0])
        assert s.error_flags() == 0
        s.close()
    err = oc.relative_errors(out[1], out[0])
    assert all(l2 < 1e-6 for _, l2 in err), err


@pytest.mark.parametrize("name", ["dt_ml3d", "dt_ml2d", "dt_rml3d_epi"])
def test_dual_time_matches_reference_build(built, tmp_path, name):
    case, steps, z, t_ref = gu.load(gu.fixture_path(name))
    gu.check_library(case, steps, z, t_ref, tmp_path / name).close()


def test_dual_time_inner_adaptation_matches_oracle(built, tmp_path):
    dual = dict(steady=0, temporal_scheme=2, implicit_method=1, dplur_inner_step=2, inner_iteration=3,
                max_inner_iteration=9, iteration_adjust_step=1, dt=3e-7)
    case = oc.mixing_layer_3d(mx=24, my=20, mz=12, ybc="outflow", steady=dual)
    d = oc.write_case(case, tmp_path / "adapt")
    s = ostc.Solver(str(d))
    s.set_state(case.bv)
    o = Oracle(case)
    o.set_state(case.bv)
    for _ in range(4):
        assert s.dual(1) == o.dual(1)
    err = oc.relative_errors(s.get_state()[0], o.get_state()[0])
    assert all(m < gu.TOL and l2 < gu.TOL for m, l2 in err), err
    assert abs(s.time() - o.time()) <= 1e-14 * o.time()
    s.close()


@pytest.mark.parametrize("kind", ["steady_mixture_dplur_epi", "dual_air"])
def test_iteration_graph_equals_kernel_loop(built, tmp_path, kind):
    """A steady or dual-time iteration replayed from its captured graph gives the state the same
    iteration launched kernel by kernel gives (OSTC_LAUNCH_BLOCK_LOOP), bit for bit."""
    if kind == "dual_air":
        case = oc.mixing_layer_3d(mx=24, my=20, mz=12, ybc="outflow", steady=dict(DUAL, dt=2e-7))
    else:
        case = oc.reacting_mixing_layer_3d(mx=16, my=12, mz=8,
                                           steady=dict(STEADY, implicit_method=1, chem_src_method=1))
    out = []
    for mode in (ostc.LAUNCH_GRAPH, ostc.LAUNCH_BLOCK_LOOP):
        s = ostc.Solver(str(oc.write_case(case, tmp_path / f"m{mode}")))
        s.set_launch_mode(mode)
        s.set_state(case.bv, sv=case.sv)
        if kind == "dual_air":
            s.dual(4)
        else:
            s.steady(6)
        out.append(s.get_state()[0])
        s.close()
    assert np.array_equal(out[0], out[1])
