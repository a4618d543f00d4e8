"""Parity against the reference solver's own FP64 CUDA build.

tests/golden/golden_*.npz were produced by tests/golden/make_golden.py: the reference's Driver and
RK3 (compiled from its sources by oracle/ref/build_ref.sh) advanced each seeded case on a B200.  The
CPU oracle is checked against them here without a GPU (the fixtures it finishes within seconds); the
CUDA path is checked against every one of them on the GPU (the boundary-face fixtures in
test_gpu_faces.py, the flow-field and statistics files in test_gpu_plt.py / test_gpu_stat.py).
Bar: 1e-12 relative per conserved variable, max norm and L2 (ostc_cases.relative_errors), and the
physical time to 1e-13; the benchmark-size fixtures are compared on a seeded node sample and on every
k- and j-plane sum (golden_util).
"""
from pathlib import Path

import numpy as np
import pytest

import golden_util as gu
from oracle import MultiOracle, Oracle

FIXTURES = gu.all_fixtures()
# fixtures whose library check lives beside the feature it pins
FACE_FIXTURES = {"ml3d_wall_isothermal", "ml3d_wall_adiabatic", "ml2d_wall_isothermal_weno5",
                 "ml2d_wall_adiabatic_weno7", "ml3d_inflow_outflow", "ml3d_subsonic_backpressure", "rml3d_wall",
                 "rml3d_inflow", "rml3d_farfield_fr72", "rml3d_farfield_mix71"}
FILE_FIXTURES = {"ml3d_stat_plt", "rml3d_stat_plt", "ml2d_plt", "ml3d_stat_extra", "ml2d_stat_extra",
                 "rml3d_stat_extra"}
# node-steps the serial oracle finishes in a few seconds (mixtures cost about ten times air)
ORACLE_BUDGET = 4e6


def _oracle_affordable(path):
    m, steps, sampled, multi = gu.meta(path)
    if sampled or gu.noisy(m["kwargs"]):
        # white-noise inflows draw from curand states the oracle does not restate; the library is
        # checked against the reference build directly
        return False
    kw = m["kwargs"]
    if multi and kw.get("uneven_axes"):
        nodes = kw.get("nb", 12) * kw.get("hi", 256) ** 3
    elif multi:
        nodes = sum(kw.get("dims") or [kw.get("hi", 256)] * kw.get("nb", 12)) * kw.get("my", 256) * kw.get("mz", 256)
    else:
        nodes = kw.get("mx", 0) * kw.get("my", 0) * kw.get("mz", 1)
    cost = nodes * steps * (10 if m["generator"].startswith("reacting") else 1)
    return 0 < cost <= ORACLE_BUDGET


CPU_FIXTURES = [p for p in FIXTURES if _oracle_affordable(p)]
GPU_FIXTURES = [p for p in FIXTURES if gu.name_of(p) not in FACE_FIXTURES | FILE_FIXTURES]


def test_fixtures_present():
    names = {gu.name_of(p) for p in FIXTURES}
    assert len(FIXTURES) >= 15
    # the benchmark configurations at their stated sizes
    assert {"c1_ml2d_256x128_weno5_ausm", "c2_ml3d_512x256x128_weno7_hllc", "c3_rml3d_96x48x24_fr72"} <= names


@pytest.mark.parametrize("path", CPU_FIXTURES, ids=gu.name_of)
def test_oracle_matches_reference(built, path):
    case, steps, z, t_ref = gu.load(path)
    if hasattr(case, "blocks"):
        m = MultiOracle(case)
        m.set_state()
        m.step(steps)
        for b in range(int(z["n_block"])):
            gu.assert_state(m.blocks[b].get_state()[0], z, block=b)
        assert abs(m.time() - t_ref) <= gu.TOL_T * t_ref
        return
    tm, tl, tt = gu.tolerances(gu.name_of(path))
    o = Oracle(case)
    o.set_state(case.bv)
    o.advance(steps)
    gu.assert_state(o.get_state()[0], z, tol=(tm, tl))
    if o.dual_case:
        t_ref = steps * case.scheme["dt"]  # not stored by the reference's dual-time driver
    assert abs(o.time() - t_ref) <= tt * t_ref


@pytest.mark.gpu
@pytest.mark.parametrize("path", GPU_FIXTURES, ids=gu.name_of)
def test_gpu_matches_reference(built, tmp_path, path):
    case, steps, z, t_ref = gu.load(path)
    s = gu.check_library(case, steps, z, t_ref, tmp_path / "case", name=gu.name_of(path))
    s.close()


@pytest.mark.parametrize("name", sorted(n for n in FILE_FIXTURES if "stat" in n and gu.fixture_path(n).exists()))
def test_oracle_statistics_match_reference_files(built, name):
    """The oracle's restatement of the basic statistics collector (SinglePointStat.cu:641-706) summed over
    the same trajectory as the reference's exported coll_*.bin files: rho, p and the stat_rey_1st extras
    T, u in the listed order, rho*p, after every step past step 2."""
    from ref_files import read_stat_file

    case, steps, z, _ = gu.load(gu.fixture_path(name))
    o = Oracle(case)
    o.set_state(case.bv)
    files = ["coll_rey_1st.bin", "coll_fav_1st.bin", "coll_rey_2nd.bin", "coll_fav_2nd.bin"]
    ref = [read_stat_file(z["file_" + f].tobytes()) for f in files]
    n_var = [r[2].__len__() for r in ref]
    shape = (case.mz + 2, case.my + 2, case.mx + 2)
    acc = np.zeros(sum(n_var) * int(np.prod(shape)))
    for st in range(1, steps + 1):
        o.step(1)
        if st > 2:
            o.stat_collect(acc, [5, 1], True)
    off = 0
    for g, (nb, ngg, names, counters, blocks) in enumerate(ref):
        assert (nb, ngg) == (1, 1) and counters == [steps - 2] * len(names)
        n = n_var[g] * int(np.prod(shape))
        got = acc[off:off + n].reshape((n_var[g],) + shape)
        off += n
        gu.assert_fields(names, got, blocks[0][1])


@pytest.mark.parametrize("name", sorted(n for n in FILE_FIXTURES
                                        if n.endswith("stat_extra") and gu.fixture_path(n).exists()))
def test_oracle_additional_statistics_match_reference_files(built, name):
    """The oracle's restatement of the additional collectors (SinglePointStat.cu:707-722; TkeBudget.cu,
    SpeciesStat.cu) summed over the same trajectory as the reference's tke_budget.bin and species
    files: the viscous stresses and their work, and for H2, OH, O2 rho u_i Y and the dissipation terms."""
    from ref_files import read_stat_file

    case, steps, z, _ = gu.load(gu.fixture_path(name))
    o = Oracle(case)
    o.set_state(case.bv)
    shape = (case.mz, case.my, case.mx)
    mix = case.mixture is not None
    ss = [case.mixture["tables"].names.index(n) for n in ("H2", "OH", "O2")] if mix else []
    tke = np.zeros((7,) + shape)
    svc = np.zeros((3 * len(ss),) + shape) if mix else None
    sdr = np.zeros((5 * len(ss),) + shape) if mix else None
    for st in range(1, steps + 1):
        o.step(1)
        if st > 2:
            o.stat_extra(tke, svc, sdr, ss)
    pairs = [("tke_budget.bin", tke)] + ([("species_velocity_correlation.bin", svc),
                                          ("species_dissipation_rate.bin", sdr)] if mix else [])
    for fname, got in pairs:
        nb, ngg, names, counters, blocks = read_stat_file(z["file_" + fname].tobytes())
        assert (nb, ngg) == (1, 0) and counters == [steps - 2] * len(names), fname
        gu.assert_fields(names, got, blocks[0][1], tol=gu.TOL_GRAD)
