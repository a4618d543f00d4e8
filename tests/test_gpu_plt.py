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

pytestmark = pytest.mark.gpu


def read_plt(path):
    """Minimal reader of the V112 layout that ostc_write_plt and the reference's FieldIO write."""
    raw = path.read_bytes()
    pos = 8
    assert raw[:8] == b"#!TDV112"

    def take(fmt, n=1):
        nonlocal pos
        v = np.frombuffer(raw, dtype=fmt, count=n, offset=pos)
        pos += v.nbytes
        return v

    def s():
        out = ""
        while True:
            c = int(take(np.int32)[0])
            if c == 0:
                return out
            out += chr(c)

    byte_order, file_type = (int(x) for x in take(np.int32, 2))
    assert (byte_order, file_type) == (1, 0)
    assert s() == "Solution file"
    nvar = int(take(np.int32)[0])
    names = [s() for _ in range(nvar)]
    zones = []
    marker = float(take(np.float32)[0])
    while marker == 299.0:
        name = s()
        parent, strand = (int(x) for x in take(np.int32, 2))
        t = float(take(np.float64)[0])
        color, ztype, loc, raw_nb, misc = (int(x) for x in take(np.int32, 5))
        dims = tuple(int(x) for x in take(np.int32, 3))
        aux = int(take(np.int32)[0])
        assert (parent, strand, color, ztype, loc, raw_nb, misc, aux) == (-1, -2, -1, 0, 0, 0, 0, 0)
        zones.append((name, t, dims))
        marker = float(take(np.float32)[0])
    assert marker == 357.0
    data = []
    for _, _, (nx, ny, nz) in zones:
        assert float(take(np.float32)[0]) == 299.0
        assert list(take(np.int32, nvar)) == [2] * nvar
        assert [int(x) for x in take(np.int32, 3)] == [0, 0, -1]
        mm = take(np.float64, 2 * nvar).reshape(nvar, 2)
        arr = take(np.float64, nvar * nx * ny * nz).reshape(nvar, nz, ny, nx)
        assert np.array_equal(mm[:, 0], arr.min(axis=(1, 2, 3))) and np.array_equal(mm[:, 1], arr.max(axis=(1, 2, 3)))
        data.append(arr)
    assert pos == len(raw)
    return names, zones, data


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
