"""Single-point statistics (SinglePointStat: collect_single_point_basic_statistics after every step past
start_collect_statistics_iter, export_statistical_data) through the C ABI, against the oracle's
restatement accumulated over the same steps.

The accumulators are sums of the state (one ghost layer included), so they carry the state's own
difference from the oracle: 1e-12 relative per variable in the max norm, the trajectory tolerance.
"""
import numpy as np
import pytest

import ostc
import ostc_cases as oc
from oracle import MultiOracle, Oracle
from ref_files import read_stat_file

pytestmark = pytest.mark.gpu

TOL = 1e-12
# statistics of gradients (central differences of the state): the state's 1e-13 difference from the
# oracle grows by the ratio of a value to its local difference
GRAD_TOL = 1e-10
ALL = ostc.STAT_REY_U | ostc.STAT_REY_V | ostc.STAT_REY_W | ostc.STAT_REY_T | ostc.STAT_RHO_P
IDX = {ostc.STAT_REY_U: 1, ostc.STAT_REY_V: 2, ostc.STAT_REY_W: 3, ostc.STAT_REY_T: 5}


def _split(acc, n_var, shape):
    out, off = [], 0
    n = int(np.prod(shape))
    for nv in n_var:
        out.append(acc[off:off + nv * n].reshape((nv,) + shape))
        off += nv * n
    return out


def _check(s, oracle_blocks, flags, n_steps, start):
    """Step both sides one step at a time, the oracle collecting past `start`, and compare."""
    rey = [IDX[f] for f in (ostc.STAT_REY_U, ostc.STAT_REY_V, ostc.STAT_REY_W, ostc.STAT_REY_T) if flags & f]
    rho_p = bool(flags & ostc.STAT_RHO_P)
    s.stat_enable(start, flags)
    n_var, _, _ = s.stat_info()
    accs = []
    for b, o in enumerate(oracle_blocks):
        mz, my, mx = s.shape(b)
        accs.append(np.zeros(sum(n_var) * (mx + 2) * (my + 2) * (mz + 2)))
    return n_var, rey, rho_p, accs


def _run_and_compare(s, step_oracle, oracle_blocks, flags, n_steps, start):
    n_var, rey, rho_p, accs = _check(s, oracle_blocks, flags, n_steps, start)
    for st in range(1, n_steps + 1):
        s.step(1)
        step_oracle()
        if st > start:
            for o, acc in zip(oracle_blocks, accs):
                o.stat_collect(acc, rey, rho_p)
    nv, nc, steps = s.stat_info()
    assert (nc, steps) == (n_steps - start, n_steps)
    for b, acc in enumerate(accs):
        mz, my, mx = s.shape(b)
        want = _split(acc, n_var, (mz + 2, my + 2, mx + 2))
        for g in range(4):
            got = s.stat_get(g, block=b)
            assert got.shape == want[g].shape
            for l in range(got.shape[0]):
                scale = np.max(np.abs(want[g][l]))
                if scale == 0:  # w = 0 in 2-D: the sums stay exactly zero
                    assert np.all(got[l] == 0), (b, ostc.STAT_GROUPS[g], l)
                    continue
                err = np.max(np.abs(got[l] - want[g][l])) / scale
                assert err < TOL, (b, ostc.STAT_GROUPS[g], l, err)
    assert s.error_flags() == 0
    return n_var


@pytest.mark.parametrize("dims,flags", [((40, 24, 20), ALL), ((65, 33, 1), ostc.STAT_REY_T), ((36, 20, 16), 0)],
                         ids=["3d_all", "2d_T", "3d_basic"])
def test_stat_air_matches_oracle(built, tmp_path, dims, flags):
    mx, my, mz = dims
    case = oc.mixing_layer_2d(mx=mx, my=my) if mz == 1 else oc.mixing_layer_3d(mx=mx, my=my, mz=mz)
    d = oc.write_case(case, tmp_path / "c")
    s = ostc.Solver(str(d))
    s.set_state(case.bv)
    o = Oracle(case)
    o.set_state(case.bv)
    n_var = _run_and_compare(s, lambda: o.step(1), [o], flags, 6, 2)
    assert n_var == [2 + bin(flags & 15).count("1"), 4, 2 + (1 if flags & ostc.STAT_RHO_P else 0), 7]


def test_stat_mixture_matches_oracle(built, tmp_path):
    case = oc.reacting_mixing_layer_3d(mx=24, my=18, mz=12)
    d = oc.write_case(case, tmp_path / "c")
    s = ostc.Solver(str(d))
    s.set_state(case.bv, sv=case.sv)
    o = Oracle(case)
    o.set_state(case.bv, case.sv)
    n_var = _run_and_compare(s, lambda: o.step(1), [o], ostc.STAT_RHO_P | ostc.STAT_REY_U, 4, 1)
    assert n_var == [3, 4 + 9, 3, 7 + 9]


def test_stat_multiblock_matches_oracle(built, tmp_path):
    mc = oc.multiblock_mixing_layer_3d(dims=[20, 17, 23], my=16, mz=10)
    d = oc.write_case(mc, tmp_path / "mb")
    s = ostc.Solver(str(d))
    for b, blk in enumerate(mc.blocks):
        s.set_state(blk.bv, block=b)
    m = MultiOracle(mc)
    m.set_state()
    _run_and_compare(s, lambda: m.step(1), m.blocks, ALL, 4, 0)


def test_stat_export_import_and_setup(built, tmp_path):
    """Setup-driven collection (if_collect_statistics, start_collect_statistics_iter, stat_rey_1st in the
    listed order, rho_p_correlation), the exported files, and a continued collection from them."""
    case = oc.reacting_mixing_layer_3d(mx=16, my=12, mz=8)
    d = oc.write_case(case, tmp_path / "c")
    setup = d / "setup.txt"
    setup.write_text(setup.read_text() + "bool if_collect_statistics = 1\nint start_collect_statistics_iter = 1\n"
                     "array string stat_rey_1st {\n    T u\n}\nbool rho_p_correlation = 1\n")
    s = ostc.Solver(str(d))
    s.set_state(case.bv, sv=case.sv)
    s.step(3)
    n_var, nc, steps = s.stat_info()
    assert n_var == [4, 13, 3, 16] and (nc, steps) == (2, 3)
    out = tmp_path / "stat"
    out.mkdir()
    s.stat_export(out)
    names = case.mixture["tables"].names
    expect_names = [["rho", "p", "T", "u"], ["rhoU", "rhoV", "rhoW", "rhoT"] + ["rho" + n for n in names],
                    ["RhoRho", "pp", "rhoP"],
                    ["rhoUU", "rhoVV", "rhoWW", "rhoUV", "rhoUW", "rhoVW", "rhoTT"] + ["rho" + n + n for n in names]]
    for g, fname in enumerate(["coll_rey_1st.bin", "coll_fav_1st.bin", "coll_rey_2nd.bin", "coll_fav_2nd.bin"]):
        nb, ngg, fnames, counters, blocks = read_stat_file(out / fname)
        assert (nb, ngg) == (1, 1) and fnames == expect_names[g] and counters == [2] * n_var[g]
        assert blocks[0][0] == (16, 12, 8)
        assert np.array_equal(blocks[0][1], s.stat_get(g))
    rey1 = s.stat_get(0)
    assert np.all(rey1[0] > 0)  # sums of a positive density, ghost layer included
    s2 = ostc.Solver(str(d))
    s2.set_state(case.bv, sv=case.sv)
    s2.stat_import(out)
    assert s2.stat_info()[1] == 2
    for g in range(4):
        assert np.array_equal(s2.stat_get(g), s.stat_get(g))
    # a selection that differs from the files is refused with the reason
    s3 = ostc.Solver(str(d))
    s3.set_state(case.bv, sv=case.sv)
    s3.stat_enable(0, ostc.STAT_REY_U)
    with pytest.raises(ostc.OstcError, match="coll_rey_1st.bin"):
        s3.stat_import(out)


def test_stat_continued_collection(built, tmp_path):
    """if_continue_collect_statistics: a second context that imports the files and restarts from the
    same state collects on its next step and ends with the sums of the uninterrupted run.  Outflow y
    faces: a restart re-applies the boundary faces to the stored state, and the far-field face
    rewrites its boundary node from that node's own value, so a far-field case would restart from a
    slightly different state (in the reference as here)."""
    case = oc.mixing_layer_3d(mx=24, my=16, mz=12, ybc="outflow")
    d = oc.write_case(case, tmp_path / "c")
    s = ostc.Solver(str(d))
    s.set_state(case.bv)
    s.stat_enable(1, ALL)
    s.step(3)
    out = tmp_path / "stat"
    out.mkdir()
    s.stat_export(out)
    s2 = ostc.Solver(str(d))
    s2.set_state(s.get_state()[1])
    s2.stat_enable(1, ALL)
    s2.stat_import(out)
    s.step(2)
    s2.step(2)
    assert s.stat_info()[1] == 4 and s2.stat_info()[1] == 4
    for g in range(4):
        a, b = s.stat_get(g), s2.stat_get(g)
        for l in range(a.shape[0]):
            assert np.max(np.abs(a[l] - b[l])) <= TOL * np.max(np.abs(a[l])), (g, l)


def test_stat_off_and_bad_flags(built, tmp_path):
    case = oc.mixing_layer_3d(mx=16, my=12, mz=8)
    d = oc.write_case(case, tmp_path / "c")
    s = ostc.Solver(str(d))
    s.set_state(case.bv)
    with pytest.raises(ostc.OstcError, match="statistics collection is off"):
        s.stat_info()
    with pytest.raises(ostc.OstcError, match="unknown flag"):
        s.stat_enable(0, 256)
    s.stat_enable(5, 0)
    s.step(2)
    assert s.stat_info()[1:] == (0, 2)
    assert np.all(s.stat_get(1) == 0)
    s.stat_disable()
    with pytest.raises(ostc.OstcError):
        s.stat_get(0)


# ---- against the coll_*.bin files the reference itself exported at the end of the same run
# (SinglePointStat.cu:515-706, RK.cuh:200-207); fixtures from tests/golden/make_golden.py

@pytest.mark.parametrize("name", ["ml3d_stat_plt", "rml3d_stat_plt", "ml3d_stat_extra", "ml2d_stat_extra",
                                  "rml3d_stat_extra"])
def test_stat_matches_reference_files(built, tmp_path, name):
    import golden_util as gu

    case, steps, z, t_ref = gu.load(gu.fixture_path(name))
    extra = name.endswith("stat_extra")
    s = gu.check_library(case, steps, z, t_ref, tmp_path / name, gu.STAT_SETUP_EXTRA if extra else gu.STAT_SETUP)
    out = tmp_path / "stat"
    out.mkdir()
    s.stat_export(out)
    files = sorted(k[len("file_"):] for k in z.files if k.startswith("file_") and k.endswith(".bin"))
    assert len(files) >= 4
    for fname in files:
        nb, ngg, names, counters, blocks = read_stat_file(out / fname)
        rnb, rngg, rnames, rcounters, rblocks = read_stat_file(z["file_" + fname].tobytes())
        assert (nb, ngg, names, counters) == (rnb, rngg, rnames, rcounters), fname
        for (ext, got), (rext, ref) in zip(blocks, rblocks):
            assert ext == rext
            gu.assert_fields(names, got, ref, tol=gu.TOL if fname.startswith("coll_") else gu.TOL_GRAD)
    s.close()


EXTRA = ostc.STAT_TKE_BUDGET | ostc.STAT_SPECIES_VELOCITY | ostc.STAT_SPECIES_DISSIPATION


@pytest.mark.parametrize("kind", ["air_3d", "air_2d", "mixture_3d"])
def test_additional_collectors_match_oracle(built, tmp_path, kind):
    """The TKE budget and (mixtures, every species) the species velocity correlation and dissipation
    rate through ostc_stat_enable, against the oracle's orc_stat_extra over the same steps."""
    if kind == "air_3d":
        case = oc.mixing_layer_3d(mx=32, my=24, mz=16)
    elif kind == "air_2d":
        case = oc.mixing_layer_2d(mx=49, my=33)
    else:
        case = oc.reacting_mixing_layer_3d(mx=24, my=18, mz=12)
    d = oc.write_case(case, tmp_path / "c")
    s = ostc.Solver(str(d))
    s.set_state(case.bv, sv=case.sv)
    o = Oracle(case)
    o.set_state(case.bv)
    s.stat_enable(1, EXTRA)
    shape = s.shape(0)
    ns = case.sv.shape[0] if case.sv is not None else 0
    tke = np.zeros((7,) + shape)
    svc = np.zeros((3 * ns,) + shape) if ns else None
    sdr = np.zeros((5 * ns,) + shape) if ns else None
    for st in range(1, 5):
        s.step(1)
        o.step(1)
        if st > 1:
            o.stat_extra(tke, svc, sdr, list(range(ns)))
    assert [s.stat_group_vars(g) for g in (4, 5, 6)] == [7, 3 * ns, 5 * ns]
    for g, want in ((4, tke), (5, svc), (6, sdr)):
        if want is None:
            continue
        got = s.stat_get(g)
        assert got.shape == want.shape
        for l in range(got.shape[0]):
            scale = np.max(np.abs(want[l]))
            if scale == 0:
                assert np.all(got[l] == 0), (g, l)
                continue
            assert np.max(np.abs(got[l] - want[l])) <= GRAD_TOL * scale, (ostc.STAT_GROUPS[g], l)
    # the exported files carry them with their names and no ghost layer
    out = tmp_path / "stat"
    out.mkdir()
    s.stat_export(out)
    nb, ngg, names, counters, blocks = read_stat_file(out / "tke_budget.bin")
    assert (nb, ngg, names[0], names[-1], counters) == (1, 0, "Tau11", "TauIjDUiDXj", [3] * 7)
    assert blocks[0][1].shape == (7,) + shape
    assert (out / "species_dissipation_rate.bin").exists() == bool(ns)
