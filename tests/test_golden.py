"""Parity against the reference solver's own FP64 CUDA build.

tests/golden/golden_*.npz were produced by tests/golden/make_golden.py: the reference's Driver and
RK3 (compiled from its sources by oracle/ref/build_ref.sh) advanced each seeded case on a B200.  The
CPU oracle is checked against them here without a GPU; the CUDA path is checked against them on
the GPU.  Bar: 1e-12 relative per conserved variable, max norm and L2 (ostc_cases.relative_errors),
and the physical time to 1e-13.
"""
import glob
import json
from pathlib import Path

import numpy as np
import pytest

import ostc_cases as oc
from oracle import MultiOracle, Oracle

HERE = Path(__file__).resolve().parent
FIXTURES = sorted(glob.glob(str(HERE / "golden" / "golden_*.npz")))
TOL = 1e-12


def _load(path):
    z = np.load(path)
    meta = json.loads(str(z["case"]))
    case = getattr(oc, meta["generator"])(**meta["kwargs"])
    if "n_block" in z:
        total = sum(np.sum(b.bv) for b in case.blocks)
        cv = [z[f"cv_{b}"] for b in range(int(z["n_block"]))]
    else:
        total = np.sum(case.bv)
        cv = z["cv"]
    assert abs(total - float(z["bv0_sum"])) <= 1e-12 * abs(float(z["bv0_sum"])), "case generator drifted"
    return case, int(z["steps"]), cv, float(z["t"])


def test_fixtures_present():
    assert len(FIXTURES) >= 4


@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: Path(p).stem)
def test_oracle_matches_reference(built, path):
    case, steps, cv_ref, t_ref = _load(path)
    if hasattr(case, "blocks"):
        m = MultiOracle(case)
        m.set_state()
        m.step(steps)
        for b, ref in enumerate(cv_ref):
            cv, _, _ = m.blocks[b].get_state()
            err = oc.relative_errors(cv, ref)
            assert all(mx < TOL and l2 < TOL for mx, l2 in err), (b, err)
        assert abs(m.time() - t_ref) <= 1e-13 * t_ref
        return
    o = Oracle(case)
    o.set_state(case.bv)
    o.step(steps)
    cv, _, _ = o.get_state()
    err = oc.relative_errors(cv, cv_ref)
    assert all(m < TOL and l2 < TOL for m, l2 in err), err
    assert abs(o.time() - t_ref) <= 1e-13 * t_ref


@pytest.mark.gpu
@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: Path(p).stem)
def test_gpu_matches_reference(built, tmp_path, path):
    import ostc

    case, steps, cv_ref, t_ref = _load(path)
    d = oc.write_case(case, tmp_path / "case")
    s = ostc.Solver(str(d))
    if hasattr(case, "blocks"):
        for b, blk in enumerate(case.blocks):
            s.set_state(blk.bv, block=b)
        s.step(steps)
        for b, ref in enumerate(cv_ref):
            cv, _ = s.get_state(block=b)
            err = oc.relative_errors(cv, ref)
            assert all(mx < TOL and l2 < TOL for mx, l2 in err), (b, err)
        assert abs(s.time() - t_ref) <= 1e-13 * t_ref
        assert s.error_flags() == 0
        return
    s.set_state(case.bv, sv=case.sv)
    s.step(steps)
    cv, _ = s.get_state()
    err = oc.relative_errors(cv, cv_ref)
    assert all(m < TOL and l2 < TOL for m, l2 in err), err
    assert abs(s.time() - t_ref) <= 1e-13 * t_ref
    assert s.error_flags() == 0
