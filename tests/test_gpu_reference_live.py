"""The 3-D air benchmark layer at its full size (512 x 256 x 128 nodes, WENO7-Z + HLLC, viscous,
far-field y) advanced 3 SSP-RK3 steps by the reference's own FP64 CUDA build and by the library, and
compared on every node: 1e-12 relative per conserved variable (max norm and L2), physical time 1e-13.

The reference build (oracle/_ref/ref_harness, compiled from the reference's sources by
oracle/ref/build_ref.sh; its Driver + RK3, RK.cuh:19-228) runs in its own process first; its state file
is read back and the library then runs the same seeded case through the C ABI.  The committed fixture
golden_c2_ml3d_512x256x128_weno7_hllc.npz pins the same run on a node sample where the reference build
is absent.
"""
import tempfile
from pathlib import Path

import pytest

import ostc
import ostc_cases as oc
import refcase

pytestmark = pytest.mark.gpu

STEPS = 3
TOL = 1e-12


@pytest.mark.skipif(not refcase.HARNESS.exists(), reason="the reference build (oracle/_ref/ref_harness) is not here")
def test_full_size_air_layer_matches_reference_build(built, tmp_path):
    case = oc.mixing_layer_3d()
    assert (case.mx, case.my, case.mz) == (512, 256, 128)
    with tempfile.TemporaryDirectory(prefix="ostc_ref_", dir=tmp_path) as wd:
        cv_ref, _, t_ref = refcase.run_reference(case, STEPS, Path(wd), timeout=900)[:3]
    d = oc.write_case(case, tmp_path / "case")
    s = ostc.Solver(str(d))
    s.set_state(case.bv)
    s.step(STEPS)
    cv, _ = s.get_state()
    err = oc.relative_errors(cv, cv_ref)
    assert all(m < TOL and l2 < TOL for m, l2 in err), err
    assert abs(s.time() - t_ref) <= 1e-13 * t_ref
    assert s.error_flags() == 0
    s.close()
