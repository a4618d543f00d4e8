"""Multi-block grids joined by 1:1 interfaces (the reference's inner-face file and
inner_communication): the CPU oracle's multi-block driver on the host, the CUDA path against it on
the GPU.

Tolerance as in test_gpu_parity: 1e-12 relative per conserved variable (momentum against the momentum
magnitude), max norm and L2, per block.
"""
import numpy as np
import pytest

import ostc_cases as oc
from oracle import MultiOracle, Oracle

TOL = 1e-12


def test_single_block_multi_driver_matches_oracle(built):
    """A one-block multi-block case through the multi-block driver equals the single-block oracle."""
    mc = oc.multiblock_mixing_layer_3d(dims=[24], my=16, mz=10)
    b = mc.blocks[0]
    sc = oc.Case("one", b.mx, b.my, b.mz, b.x, b.y, b.z, mc.grid_scale, b.faces, mc.bc_structs, mc.scheme, b.bv,
                 freestream=mc.freestream)
    m = MultiOracle(mc)
    m.set_state()
    o = Oracle(sc)
    o.set_state(sc.bv)
    m.step(3)
    o.step(3)
    cm, _, _ = m.blocks[0].get_state()
    co, _, _ = o.get_state()
    assert np.array_equal(cm, co)


def test_interface_registration_chain(built):
    """Host parsing: every block of a 4-block chain reports its interfaces through probe_case."""
    import ostc

    mc = oc.multiblock_mixing_layer_3d(dims=[20, 17, 23, 19], my=14, mz=9)
    import tempfile
    from pathlib import Path
    d = oc.write_case(mc, Path(tempfile.mkdtemp()) / "mb")
    info = ostc.probe_case(str(d))
    assert info["n_block"] == 4


@pytest.mark.gpu
@pytest.mark.parametrize("dims,my,mz,recon,rs,steps", [([20, 17, 23], 16, 10, 5, 4, 10),
                                                         ([30, 21, 26, 18], 24, 1, 4, 3, 20),
                                                         ([22, 19], 14, 9, 2, 2, 10)],
                         ids=["3d_awe7_hllc", "2d_awe5_ausm", "3d_muscl_roe"])
def test_gpu_multiblock_matches_oracle(built, tmp_path, dims, my, mz, recon, rs, steps):
    import ostc

    mc = oc.multiblock_mixing_layer_3d(dims=dims, my=my, mz=mz, reconstruction=recon, inviscid_scheme=rs)
    d = oc.write_case(mc, tmp_path / "mb")
    s = ostc.Solver(str(d))
    assert s.n_block == len(dims)
    for b, blk in enumerate(mc.blocks):
        s.set_state(blk.bv, block=b)
    m = MultiOracle(mc)
    m.set_state()
    s.step(steps)
    m.step(steps)
    assert abs(s.time() - m.time()) <= 1e-13 * m.time()
    for b in range(len(dims)):
        cg, _ = s.get_state(block=b)
        co, _, _ = m.blocks[b].get_state()
        err = oc.relative_errors(cg, co)
        assert all(mx < TOL and l2 < TOL for mx, l2 in err), (b, err)
    assert s.error_flags() == 0


def _solver(mc, path):
    import ostc

    s = ostc.Solver(str(oc.write_case(mc, path)))
    for b, blk in enumerate(mc.blocks):
        s.set_state(blk.bv, block=b)
    return s


@pytest.mark.gpu
def test_gpu_uneven_axes_matches_oracle(built, tmp_path):
    """Every block's three extents differ: interfaces cover the overlap of neighbouring x faces and the
    rest of each x face is an outflow patch (faces and interfaces on sub-ranges of a side)."""
    mc = oc.multiblock_mixing_layer_3d(nb=5, lo=10, hi=24, seed=11, uneven_axes=True)
    assert len({(b.my, b.mz) for b in mc.blocks}) > 1
    s = _solver(mc, tmp_path / "mb")
    m = MultiOracle(mc)
    m.set_state()
    s.step(8)
    m.step(8)
    assert abs(s.time() - m.time()) <= 1e-13 * m.time()
    for b in range(len(mc.blocks)):
        err = oc.relative_errors(s.get_state(block=b)[0], m.blocks[b].get_state()[0])
        assert all(mx < TOL and l2 < TOL for mx, l2 in err), (b, err)


@pytest.mark.gpu
@pytest.mark.parametrize("uneven", [False, True], ids=["chain", "uneven_axes"])
def test_block_loop_equals_graph(built, tmp_path, uneven):
    """The per-block launch loop (kernels launched from the host, block after block) and the captured
    step graph (blocks forked onto side streams) give the same state bit for bit."""
    import ostc

    mc = (oc.multiblock_mixing_layer_3d(nb=4, lo=10, hi=22, seed=5, uneven_axes=True) if uneven else
          oc.multiblock_mixing_layer_3d(dims=[20, 17, 23, 19], my=14, mz=9))
    out = []
    for mode in (ostc.LAUNCH_GRAPH, ostc.LAUNCH_BLOCK_LOOP):
        s = _solver(mc, tmp_path / f"m{mode}")
        s.set_launch_mode(mode)
        s.step(6)
        out.append([s.get_state(block=b)[0] for b in range(len(mc.blocks))] + [s.time()])
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)
