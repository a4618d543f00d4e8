"""Tecplot flow-field file (FieldIO: flowfield.plt, binary V112; read_flowfield restarts from it)
through the C ABI: the layout parsed field by field against the state, and write -> read round trips
(air, 2-D air, 9-species mixture, two blocks).  A restart holds the primitive state bit for bit and
recomputes the conservative state from it, as read_flowfield does.  The continued trajectory matches
the uninterrupted one to 1e-12 relative for air; for mixtures to 1e-6, because the stored temperature
is the Newton iterate of the last stage (relative tolerance 1e-3), not the root the restart's energy
is computed from.  The restart cases use faces that leave their face nodes consistent (outflow,
periodic, walls): symmetry and far-field faces rewrite a face node's primitive state without its
conservative state, so a restart from primitive variables departs from the uninterrupted run there,
in the reference as here.
"""
import numpy as np
import pytest

import ostc
import ostc_cases as oc
from ref_files import read_plt

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", ["air3d", "air2d", "mixture"])
def test_plt_layout_and_restart(built, tmp_path, kind):
    if kind == "air3d":
        case = oc.mixing_layer_3d(mx=24, my=16, mz=12, ybc="outflow")
    elif kind == "air2d":
        case = oc.mixing_layer_2d(mx=33, my=17, ybc="wall")
    else:
        case = oc.reacting_mixing_layer_3d(mx=16, my=12, mz=8)
    mix = kind == "mixture"
    d = oc.write_case(case, tmp_path / "c")
    s = ostc.Solver(str(d))
    s.set_state(case.bv, sv=case.sv) if mix else s.set_state(case.bv)
    s.step(3)
    t3 = s.time()
    cv3, bv3 = s.get_state()
    g = 2
    s.write_plt(tmp_path / "flowfield.plt", ngg_out=g)
    names, zones, data = read_plt(tmp_path / "flowfield.plt")
    expect = ["x", "y", "z", "density", "u", "v", "w", "pressure", "temperature", "mach"]
    if mix:
        expect += case.mixture["tables"].names
    assert names == expect
    mz, my, mx = s.shape()
    assert zones[0][2] == (mx + 2 * g, my + 2 * g, mz + 2 * g) and zones[0][1] == t3
    arr = data[0]
    inner = (slice(g, -g),) * 3
    for l in range(6):
        assert np.array_equal(arr[3 + l][inner], bv3[l]), expect[3 + l]
    # coordinates: the interior nodes of the grid file (scaled to metres)
    assert np.allclose(arr[0][inner], case.x * case.grid_scale, rtol=1e-15, atol=0)
    vel = np.sqrt(bv3[1] ** 2 + bv3[2] ** 2 + bv3[3] ** 2)
    if not mix:
        assert np.allclose(arr[9][inner], vel / np.sqrt(1.4 * oc.R_AIR * bv3[5]), rtol=1e-14)
    else:
        assert np.array_equal(arr[10:][(slice(None),) + inner], s.get_species())
    if mz == 1:
        # 2-D: the flow variables of the k ghost layers repeat k = 0
        assert np.array_equal(arr[3:, 0], arr[3:, g])
    # restart: a new context from the file
    s2 = ostc.Solver(str(d))
    assert s2.read_plt(tmp_path / "flowfield.plt") == t3
    cv_r, bv_r = s2.get_state()
    assert np.array_equal(bv_r, bv3)
    s.step(2)
    s2.step(2)
    err = oc.relative_errors(s2.get_state()[0], s.get_state()[0])
    tol = 1e-6 if mix else 1e-12
    assert all(m < tol and l2 < tol for m, l2 in err), err
    assert abs(s2.time() - s.time()) <= (tol if mix else 1e-14) * s.time()  # CFL dt follows the state


def test_plt_two_blocks_and_rejections(built, tmp_path):
    mc = oc.multiblock_mixing_layer_3d(dims=[20, 17], my=14, mz=9)
    d = oc.write_case(mc, tmp_path / "mb")
    s = ostc.Solver(str(d))
    for b, blk in enumerate(mc.blocks):
        s.set_state(blk.bv, block=b)
    s.step(2)
    s.write_plt(tmp_path / "f.plt", ngg_out=1)
    names, zones, data = read_plt(tmp_path / "f.plt")
    assert [z[0] for z in zones] == ["zone 0", "zone 1"]
    s2 = ostc.Solver(str(d))
    s2.read_plt(tmp_path / "f.plt")
    for b in range(2):
        # every node but the far-field face rows (the far-field face rewrites its node from that
        # node's own value each time it is applied) holds the written state exactly
        assert np.array_equal(s2.get_state(block=b)[1][:, :, 1:-1], s.get_state(block=b)[1][:, :, 1:-1])
    # a file whose zones do not match the case is refused with the reason
    single = oc.mixing_layer_3d(mx=20, my=14, mz=9)
    d1 = oc.write_case(single, tmp_path / "one")
    s1 = ostc.Solver(str(d1))
    with pytest.raises(ostc.OstcError, match="zone count"):
        s1.read_plt(tmp_path / "f.plt")
    (tmp_path / "junk.plt").write_bytes(b"not a plot file")
    with pytest.raises(ostc.OstcError, match="not a Tecplot"):
        s1.read_plt(tmp_path / "junk.plt")


# ---- against the flowfield.plt the reference itself wrote at the end of the same run (FieldIO.h:73-450,
# ngg_out 0 as RK3 uses, RK.cuh:57,204); fixtures from tests/golden/make_golden.py

@pytest.mark.parametrize("name", ["ml3d_stat_plt", "rml3d_stat_plt", "ml2d_plt"])
def test_plt_matches_reference_file(built, tmp_path, name):
    import golden_util as gu

    case, steps, z, t_ref = gu.load(gu.fixture_path(name))
    s = gu.check_library(case, steps, z, t_ref, tmp_path / name, gu.STAT_SETUP if "stat" in name else "")
    s.write_plt(tmp_path / "flowfield.plt", ngg_out=0)
    names, zones, data = read_plt(tmp_path / "flowfield.plt")
    rnames, rzones, rdata = read_plt(z["file_flowfield.plt"].tobytes())
    assert names == rnames
    assert [(zn, dims) for zn, _, dims in zones] == [(zn, dims) for zn, _, dims in rzones]
    for (_, t, _), (_, rt, _) in zip(zones, rzones):
        assert abs(t - rt) <= gu.TOL_T * rt
    for got, ref in zip(data, rdata):
        gu.assert_fields(names, got, ref)
    s.close()
