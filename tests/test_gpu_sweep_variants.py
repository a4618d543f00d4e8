"""Every kernel shape of the AWENO sweeps computes the same face fluxes: pinned through
ostc_set_sweep_variant, each y / z variant (column march; three shared-memory tiles) advances the case
to the same state as the default shapes - FP64 and mixed precision, WENO7-Z + HLLC and WENO5-Z + AUSM+,
3-D - within 1e-13 relative (the expressions are the same; the compiler may fuse a multiply-add
differently in another kernel body), and the FP64 one matches the oracle to 1e-12."""
import numpy as np
import pytest

import ostc
import ostc_cases as oc
from oracle import Oracle

pytestmark = pytest.mark.gpu

STEPS = 3


def _run(d, case, prec, pins):
    s = ostc.Solver(str(d))
    s.set_precision(prec)
    for dir_, v in pins.items():
        s.set_sweep_variant(dir_, v, precision=prec)
    s.set_state(case.bv)
    s.step(STEPS)
    cv, _ = s.get_state()
    assert s.error_flags() == 0
    s.close()
    return cv


@pytest.mark.parametrize("recon,rs", [(5, 4), (4, 3)], ids=["weno7_hllc", "weno5_ausm"])
@pytest.mark.parametrize("prec", [ostc.PREC_FP64, ostc.PREC_MIXED], ids=["fp64", "mixed"])
def test_sweep_variants_agree(built, tmp_path, recon, rs, prec):
    # extents that leave partial row tiles in x (mx not a multiple of 63 or 127) and partial tiles in y/z
    case = oc.mixing_layer_3d(mx=140, my=36, mz=20, reconstruction=recon, inviscid_scheme=rs)
    d = oc.write_case(case, tmp_path / "c")
    base = _run(d, case, prec, {0: 0, 1: 0, 2: 0})
    for dir_, n in ((1, 4), (2, 4)):
        for v in range(1, n):
            cv = _run(d, case, prec, {dir_: v})
            err = oc.relative_errors(cv, base)
            assert all(m < 1e-13 and l2 < 1e-13 for m, l2 in err), (dir_, v, err)
    if prec == ostc.PREC_FP64:
        o = Oracle(case)
        o.set_state(case.bv)
        o.step(STEPS)
        err = oc.relative_errors(base, o.get_state()[0])
        assert all(m < 1e-12 and l2 < 1e-12 for m, l2 in err), err


def test_sweep_variant_refusals_and_report(built, tmp_path):
    case = oc.mixing_layer_3d(mx=40, my=24, mz=16)
    d = oc.write_case(case, tmp_path / "c")
    s = ostc.Solver(str(d))
    with pytest.raises(ostc.OstcError, match="outside"):
        s.set_sweep_variant(0, 9)
    with pytest.raises(ostc.OstcError, match="precision"):
        s.set_sweep_variant(3, 0)
    for dir_ in range(3):
        s.set_sweep_variant(dir_, -1)  # back to the autotuner, forgetting results cached for this shape
    s.set_state(case.bv)
    s.step(1)
    for dir_ in range(3):
        chosen, ms = s.tune_report(dir_)
        assert 0 <= chosen < len(ms) and len(ms) == (1 if dir_ == 0 else 4)
        assert all(t > 0 for t in ms), (dir_, ms)  # every variant was timed in this fresh context
