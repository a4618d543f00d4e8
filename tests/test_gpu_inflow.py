"""Mixing-layer and white-noise inflows on the GPU, through the C ABI.

A problem_type 1 case (the reference's shipped spatial mixing layer) takes the two-stream profile at
its inflow face (apply_inflow, inflow_type 2, BoundCond.cuh:384-430) and starts every node, ghosts
included, from that profile (initialize_mixing_layer_with_info, Initialize.cu:259-326).  Without
fluctuation the trajectory is checked against the oracle at 1e-12 relative per conserved variable,
air 3-D / 2-D and the 9-species mixture.

With fluctuation_type 1 the face adds curand normal draws times intensity times the local speed to u
(and v in the mixing-layer profile, within |y| < 4 delta_omega), one generator state per node of the
ghost-padded face plane seeded as curand_init(seed + i, i, 0) (BoundCond.cu:1384-1391).  The noise is
pinned against the reference build's own fixtures (tests/golden, seed = the clock the harness fixed);
here: the face values minus the profile, scaled by intensity times speed, are standard normal (mean and
spread), zero outside the band, repeatable for one seed and different for another.

With fluctuation_type 11 the digital filter (DigitalFilter.cu) replaces the noise: per application a new
normal field over the face plane, made zero-mean and unit-rms along z, filtered in y and z, correlated
in time with the previous field and scaled by the Cholesky factor of a Gaussian Reynolds-stress profile;
the face velocity carries it times the streams' velocity difference.  Also pinned by reference-build
fixtures; here: its spread at the layer centre and its seed behaviour.
"""
import numpy as np
import pytest

import ostc
import ostc_cases as oc
from oracle import Oracle

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _solver(case, tmp_path, name):
    s = ostc.Solver(str(oc.write_case(case, tmp_path / name)))
    s.set_state(case.bv, sv=case.sv)
    return s


@pytest.mark.parametrize("kw,steps", [(dict(mx=40, my=32, mz=8), 10), (dict(mx=48, my=40, mz=1), 15),
                                      (dict(mx=32, my=24, mz=6, species=True), 6)],
                         ids=["air_3d", "air_2d", "species_3d"])
def test_mixing_layer_inflow_matches_oracle(built, tmp_path, kw, steps):
    case = oc.spatial_mixing_layer_3d(**kw)
    s = _solver(case, tmp_path, "ml")
    o = Oracle(case)
    o.set_state(case.bv, case.sv) if case.sv is not None else o.set_state(case.bv)
    s.step(steps)
    o.step(steps)
    err = oc.relative_errors(s.get_state()[0], o.get_state()[0])
    assert all(m < TOL and l2 < TOL for m, l2 in err), err
    assert abs(s.time() - o.time()) <= 1e-13 * o.time()
    assert s.error_flags() == 0


def _face_noise(case, s):
    """(u, v) of the inflow face nodes minus the profile, over intensity times the profile speed, and the
    band mask |y| < 4 delta_omega."""
    st = case.mixing_layer_streams()
    up, lo, dw = st["upper"], st["lower"], st["delta_omega"]
    y = case.y[:, :, 0] * case.grid_scale
    u0 = 0.5 * (up[1] + lo[1]) + 0.5 * (up[1] - lo[1]) * np.tanh(2 * y / dw)
    _, bv = s.get_state()
    rms = case.bc_structs["freestream"]["fluctuation_intensity"][1]
    scale = rms * np.abs(u0)
    return (bv[1, :, :, 0] - u0) / scale, bv[2, :, :, 0] / scale, np.abs(y) < 4 * dw


def test_white_noise_is_standard_normal(built, tmp_path):
    case = oc.spatial_mixing_layer_3d(mx=24, my=80, mz=32, fluctuation_type=1, intensity=0.01)
    s = _solver(case, tmp_path, "noise")
    s.set_inflow_seed(12345)
    s.step(1)
    zu, zv, band = _face_noise(case, s)
    n = int(band.sum())
    assert n > 1000
    for z in (zu[band], zv[band]):
        assert abs(float(np.mean(z))) < 5 / np.sqrt(n)
        assert abs(float(np.std(z)) - 1) < 0.1
    # outside the band the face keeps the profile (tanh rounding aside)
    assert np.max(np.abs(zu[~band])) < 1e-9 and np.max(np.abs(zv[~band])) < 1e-9


def test_white_noise_repeats_for_a_seed(built, tmp_path):
    case = oc.spatial_mixing_layer_3d(mx=24, my=32, mz=8, fluctuation_type=1)
    out = []
    for n, seed in enumerate((7, 7, 8)):
        s = _solver(case, tmp_path, f"s{n}")
        s.set_inflow_seed(seed)
        s.step(3)
        out.append(s.get_state()[0])
        s.close()
    assert np.array_equal(out[0], out[1])
    assert not np.array_equal(out[0], out[2])


def test_constant_inflow_noise(built, tmp_path):
    """A constant inflow with fluctuation_type 1: u of every face node (ghost-padded range included)
    moves by intensity times the inflow speed times a normal draw; v, w, p, T keep the inflow state."""
    case = oc.mixing_layer_3d(mx=16, my=48, mz=32, ybc="outflow", xbc="inflow", inflow_noise=0.01)
    s = _solver(case, tmp_path, "const")
    s.set_inflow_seed(99)
    s.step(1)
    st = case.inflow_states()[5]
    _, bv = s.get_state()
    speed = float(np.sqrt(st["u"] ** 2 + st["v"] ** 2 + st["w"] ** 2))
    z = (bv[1, :, :, 0] - st["u"]) / (0.01 * speed)
    assert abs(float(np.mean(z))) < 5 / np.sqrt(z.size)
    assert abs(float(np.std(z)) - 1) < 0.1
    assert np.all(bv[2, :, :, 0] == st["v"]) and np.all(bv[4, :, :, 0] == st["pressure"])


def test_more_than_one_noisy_face_refused(built, tmp_path):
    case = oc.mixing_layer_3d(mx=16, my=12, mz=8, ybc="outflow", xbc="inflow", inflow_noise=0.01)
    case.faces[1] = oc.Face(case.faces[1].raw, 5)  # the x-max face becomes a second noisy inflow
    with pytest.raises(ostc.OstcError, match="more than one inflow face"):
        _solver(case, tmp_path, "two")


def test_digital_filter_spread_and_seed(built, tmp_path):
    """v on the inflow plane over the velocity difference has the rms sqrt(R22 exp(-2 (y / delta_omega)^2))
    of the Lund transform (R22 = 0.12) near the layer centre; one seed repeats, another does not."""
    case = oc.spatial_mixing_layer_3d(mx=16, my=40, mz=64, fluctuation_type=11)
    st = case.mixing_layer_streams()
    du = abs(st["upper"][1] - st["lower"][1])
    out = []
    for n, seed in enumerate((21, 21, 22)):
        s = _solver(case, tmp_path, f"df{n}")
        s.set_inflow_seed(seed)
        s.step(2)
        out.append(s.get_state()[1])
        s.close()
    assert np.array_equal(out[0], out[1])
    assert not np.array_equal(out[0], out[2])
    ys = case.y[0, :, 0] * case.grid_scale / st["delta_omega"]
    rows = np.abs(ys) < 0.5
    v = out[0][2, :, :, 0][:, rows] / du
    want = np.sqrt(0.12 * np.exp(-2 * ys[rows] ** 2))
    ratio = float(np.sqrt(np.mean(v ** 2)) / np.sqrt(np.mean(want ** 2)))
    assert 0.6 < ratio < 1.4, ratio
    assert abs(float(np.mean(v))) < 0.2 * float(np.sqrt(np.mean(want ** 2)))
