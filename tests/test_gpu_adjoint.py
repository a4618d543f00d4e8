"""Adjoint of the multi-component right-hand side (ostc_rhs_vjp, no reference counterpart) against
central finite differences of ostc_rhs on the GPU, through the C ABI.

The product is pinned by the dot-product identity <w, J v> = <J^T w, v>: J v is taken as the central
difference (R(cv + eps v) - R(cv - eps v)) / (2 eps) with the perturbed states set through
ostc_set_conservative (equation of state, ghost faces and properties follow cv), J^T w from
ostc_rhs_vjp at cv.  v is seeded N(0,1) times |cv| per node and variable (a relative perturbation
everywhere), w seeded N(0,1); the differences at 2 eps and eps (eps = 1e-8) are combined by
Richardson extrapolation.  Tolerance, as numpy's isclose: |<w, J v> - <J^T w, v>| <= 1e-6 |<w, J v>|
+ 1e-9 sum |w * J v| (the second term covers directions whose inner product cancels to a small
fraction of its terms, where the difference's own error is set by the terms).

The WENO-Z weights of the flux-split path use eps ~ 1e-40 (scaled): where a characteristic field is
locally constant (a field that does not vary along a sweep, e.g. the species fields of a layer that
is uniform in x) the weights jump with any perturbation, the flux is only directionally
differentiable there, and no linear adjoint can match a finite difference.  The seeded states
therefore carry 5 % multiplicative noise on T, p and every Y besides the layer's velocity noise; on
them a plain central difference converges to the adjoint as O(eps^2) down to ~1e-7 (eps = 1e-8).
"""
import numpy as np
import pytest

import ostc_cases as oc

pytestmark = pytest.mark.gpu
EPS = 1e-8
RTOL = 1e-6
ATOL = 1e-9  # times sum |w * J v|
NOISE = 5e-2


def _noisy(case, seed=5, rough=False):
    """5 % seeded noise on T, p and the mass fractions (renormalised), rho from the equation of state.
    rough: also 1e-3 |N(0,1)| on every mass fraction and 5 % of the velocity difference on u, v, w
    everywhere.  On grids that reach far from the layer (|y| of several thicknesses) the seeded case is
    otherwise uniform to rounding there (the envelope of its velocity noise and the tanh blend of its
    streams vanish) and a species absent from one stream stays zero: constant fields in which the WENO-Z
    weights are only directionally differentiable, so finite differences of the whole right-hand side
    stop converging (192 x 96 x 48: 2-5 % off at every step size from 1e-6 to 1e-8; roughened: 1e-7)."""
    rng = np.random.default_rng(seed)
    case.bv[5] *= 1 + NOISE * rng.standard_normal(case.bv[5].shape)
    case.bv[4] *= 1 + NOISE * rng.standard_normal(case.bv[4].shape)
    sv = case.sv * (1 + NOISE * rng.standard_normal(case.sv.shape))
    if rough:
        du = case.extra["du"]
        for l in (1, 2, 3) if case.mz > 1 else (1, 2):
            case.bv[l] += NOISE * du * rng.standard_normal(case.bv[l].shape)
        sv += 1e-3 * np.abs(rng.standard_normal(case.sv.shape))
    case.sv[:] = sv / sv.sum(axis=0)
    mw = 1 / np.einsum("l...,l->...", case.sv, 1 / case.mixture["tables"].mw)
    case.bv[0] = case.bv[4] * mw / (oc.R_U * case.bv[5])
    return case


def _solver(case, tmp_path, rough=False):
    import ostc

    case = _noisy(case, rough=rough)
    d = oc.write_case(case, tmp_path / "case")
    s = ostc.Solver(str(d))
    s.set_state(case.bv, sv=case.sv)
    cv0, _ = s.get_state()
    return s, cv0


def _directions(cv0, rng, n):
    return [rng.standard_normal(cv0.shape) * np.abs(cv0) for _ in range(n)]


def _fd(s, cv0, v, mask, eps=EPS):
    """Central differences at 2 eps and eps combined by Richardson extrapolation (error O(eps^4))."""
    d = []
    for h in (2 * eps, eps):
        s.set_conservative(cv0 + h * v)
        rp = s.rhs(mask)
        s.set_conservative(cv0 - h * v)
        rm = s.rhs(mask)
        d.append((rp - rm) / (2 * h))
    s.set_conservative(cv0)
    return (4 * d[1] - d[0]) / 3


def _check(s, cv0, mask, rng, n_dir):
    w = rng.standard_normal(cv0.shape)
    s.set_conservative(cv0)
    g = s.rhs_vjp(w, mask)
    errs = []
    for v in _directions(cv0, rng, n_dir):
        jv = _fd(s, cv0, v, mask)
        lhs, rhs = float(np.sum(w * jv)), float(np.sum(g * v))
        # error in units of the tolerance (<= 1 passes)
        errs.append(abs(lhs - rhs) / (RTOL * abs(lhs) + ATOL * float(np.sum(np.abs(w * jv)))))
    return errs


@pytest.mark.parametrize("kw", [dict(inviscid_scheme=72), dict(inviscid_scheme=71, finite_rate=False)],
                         ids=["fr72", "mix71"])
@pytest.mark.parametrize("mask,name", [(1, "inviscid"), (2, "viscous"), (4, "source"), (7, "all")])
def test_vjp_matches_finite_differences(built, tmp_path, kw, mask, name):
    case = oc.reacting_mixing_layer_3d(mx=24, my=18, mz=12, **kw)
    s, cv0 = _solver(case, tmp_path)
    if mask == 4 and not kw.get("finite_rate", True):
        # no chemistry: the source term and its adjoint are zero
        w = np.random.default_rng(1).standard_normal(cv0.shape)
        assert not np.any(s.rhs_vjp(w, 4))
        return
    errs = _check(s, cv0, mask, np.random.default_rng(7 + mask), 4)
    assert max(errs) <= 1.0, (name, errs)


def test_vjp_64_directions_2d(built, tmp_path):
    """64 seeded directions on a 2-D reacting layer (all terms)."""
    case = oc.reacting_mixing_layer_3d(mx=40, my=24, mz=1)
    s, cv0 = _solver(case, tmp_path)
    errs = _check(s, cv0, 7, np.random.default_rng(64), 64)
    assert max(errs) <= 1.0, sorted(errs)[-5:]


def test_vjp_64_directions_192x96x48(built, tmp_path):
    """The adjoint workload's size: the 9-species reacting layer on 192 x 96 x 48 (roughened, see
    _noisy), FP64, a seeded Gaussian cotangent on every conserved variable, 64 seeded directions (all
    terms), each within the 1e-6 relative bar."""
    case = oc.reacting_mixing_layer_3d(mx=192, my=96, mz=48)
    s, cv0 = _solver(case, tmp_path, rough=True)
    errs = _check(s, cv0, 7, np.random.default_rng(192), 64)
    assert max(errs) <= 1.0, sorted(errs)[-5:]


def test_vjp_is_linear_and_additive(built, tmp_path):
    case = oc.reacting_mixing_layer_3d(mx=20, my=16, mz=10)
    s, cv0 = _solver(case, tmp_path)
    rng = np.random.default_rng(3)
    w1, w2 = rng.standard_normal(cv0.shape), rng.standard_normal(cv0.shape)
    g = s.rhs_vjp(2.0 * w1 - w2)
    g_lin = 2.0 * s.rhs_vjp(w1) - s.rhs_vjp(w2)
    assert np.max(np.abs(g - g_lin)) <= 1e-10 * np.max(np.abs(g))
    parts = s.rhs_vjp(w1, 1) + s.rhs_vjp(w1, 2) + s.rhs_vjp(w1, 4)
    g1 = s.rhs_vjp(w1, 7)
    assert np.max(np.abs(parts - g1)) <= 1e-10 * np.max(np.abs(g1))


def test_torch_autograd_wrapper(built, tmp_path):
    """ostc_rhs / ostc_rhs_vjp as a torch.autograd.Function (test harness only): the gradient of
    L(cv) = <w, rhs(cv)> by backward() against a central difference along a seeded direction."""
    torch = pytest.importorskip("torch")
    case = oc.reacting_mixing_layer_3d(mx=20, my=16, mz=10)
    s, cv0 = _solver(case, tmp_path)

    class Rhs(torch.autograd.Function):
        @staticmethod
        def forward(ctx, cv):
            s.set_conservative(cv.detach().numpy())
            return torch.from_numpy(s.rhs())

        @staticmethod
        def backward(ctx, g):
            return torch.from_numpy(s.rhs_vjp(g.detach().numpy()))

    rng = np.random.default_rng(11)
    w = torch.from_numpy(rng.standard_normal(cv0.shape))
    x = torch.from_numpy(cv0.copy()).requires_grad_(True)
    loss = (w * Rhs.apply(x)).sum()
    loss.backward()
    v = _directions(cv0, rng, 1)[0]
    jv = _fd(s, cv0, v, 7)
    fd = float(np.sum(w.numpy() * jv))
    ad = float(np.sum(x.grad.numpy() * v))
    assert abs(fd - ad) <= RTOL * abs(fd) + ATOL * float(np.sum(np.abs(w.numpy() * jv)))


AIR = {"weno7_hllc_3d": lambda: oc.mixing_layer_3d(mx=24, my=20, mz=12, ybc="outflow"),
       "weno5_ausm_3d": lambda: oc.mixing_layer_3d(mx=20, my=16, mz=12, ybc="outflow", reconstruction=4,
                                                   inviscid_scheme=3),
       # Lax-Friedrichs: |U| and the larger spectral radius put two kinks in every face flux, so a
       # smaller grid keeps the differences off them
       "weno7_lf_3d": lambda: oc.mixing_layer_3d(mx=14, my=12, mz=10, ybc="outflow", inviscid_scheme=1),
       "weno5_ausm_2d": lambda: oc.mixing_layer_2d(mx=40, my=28, ybc="outflow")}


def _check_air(s, cv0, mask, rng, n_dir):
    """_check with the differences at steps 1e-7 and 1e-8, each direction judged by the better one.
    The air right-hand side is only piecewise smooth: the HLLC contact switch (sign of the star speed),
    AUSM+'s upwind switch (sign of the mass flux), the Lax-Friedrichs flux's |U| and larger spectral
    radius have kinks, and a direction's difference crosses one at some face with a probability that grows
    with the step and the number of faces (the crossing face's term then carries an O(1) error).  At
    1e-8 the difference of nearly cancelling fluxes carries ~1e-6 of rounding, at 1e-7 ~1e-8, and at
    1e-5 the WENO weights' curvature ~1e-3.  A wrong adjoint disagrees at both steps; a kink crossed
    at one step leaves the other."""
    w = rng.standard_normal(cv0.shape)
    s.set_conservative(cv0)
    g = s.rhs_vjp(w, mask)
    errs = []
    for v in _directions(cv0, rng, n_dir):
        rhs = float(np.sum(g * v))
        e = []
        for eps in (1e-7, 1e-8):
            jv = _fd(s, cv0, v, mask, eps)
            lhs = float(np.sum(w * jv))
            e.append(abs(lhs - rhs) / (RTOL * abs(lhs) + ATOL * float(np.sum(np.abs(w * jv)))))
        errs.append(min(e))
    return errs


def _air_solver(case, tmp_path, seed=3):
    """An air layer with 2 % seeded noise on T and p (rho from the equation of state), so that no
    sweep sees a field that is constant along it."""
    import ostc

    rng = np.random.default_rng(seed)
    case.bv[5] *= 1 + 2e-2 * rng.standard_normal(case.bv[5].shape)
    case.bv[4] *= 1 + 2e-2 * rng.standard_normal(case.bv[4].shape)
    case.bv[0] = case.bv[4] / (oc.R_AIR * case.bv[5])
    s = ostc.Solver(str(oc.write_case(case, tmp_path / "air")))
    s.set_state(case.bv)
    return s, s.get_state()[0]


@pytest.mark.parametrize("name", list(AIR))
@pytest.mark.parametrize("mask,term", [(1, "inviscid"), (2, "viscous"), (3, "all")])
def test_air_vjp_matches_finite_differences(built, tmp_path, name, mask, term):
    """The air path (AWENO5/7-Z with AUSM+, HLLC or Lax-Friedrichs, Sutherland viscous terms, periodic and
    outflow faces): ostc_rhs_vjp against Richardson central differences of ostc_rhs, 6 directions."""
    s, cv0 = _air_solver(AIR[name](), tmp_path)
    errs = _check_air(s, cv0, mask, np.random.default_rng(11 + mask), 6)
    assert max(errs) <= 1.0, (name, term, errs)


@pytest.mark.parametrize("name", ["weno7_hllc_3d", "weno5_ausm_2d"])
def test_air_vjp_64_directions(built, tmp_path, name):
    """64 seeded directions (all terms)."""
    s, cv0 = _air_solver(AIR[name](), tmp_path)
    errs = _check_air(s, cv0, 3, np.random.default_rng(64), 64)
    assert max(errs) <= 1.0, sorted(errs)[-5:]


def test_vjp_rejects_uncovered_cases(built, tmp_path):
    import ostc

    air = oc.mixing_layer_3d(mx=24, my=16, mz=8)  # far-field y faces
    d = oc.write_case(air, tmp_path / "air")
    s = ostc.Solver(str(d))
    s.set_state(air.bv)
    with pytest.raises(ostc.OstcError, match="periodic and outflow"):
        s.rhs_vjp(np.zeros((5,) + s.shape(0)))
    air_out = oc.mixing_layer_3d(mx=24, my=16, mz=8, ybc="outflow")
    s1 = ostc.Solver(str(oc.write_case(air_out, tmp_path / "air_out")))
    s1.set_state(air_out.bv)
    s1.set_precision(ostc.PREC_MIXED)
    with pytest.raises(ostc.OstcError, match="FP64 step"):
        s1.step_vjp(np.zeros((5,) + s1.shape(0)))
    pv_air = oc.mixing_layer_3d(mx=24, my=16, mz=8, ybc="outflow", reconstruction=2)
    s4 = ostc.Solver(str(oc.write_case(pv_air, tmp_path / "pv_air")))
    s4.set_state(pv_air.bv)
    with pytest.raises(ostc.OstcError, match="AWENO"):
        s4.rhs_vjp(np.zeros((5,) + s4.shape(0)))
    case = oc.reacting_mixing_layer_3d(mx=20, my=16, mz=10)
    s2, cv0 = _solver(case, tmp_path)
    s2.set_chem_mode(ostc.CHEM_POINT_IMPLICIT)
    with pytest.raises(ostc.OstcError, match="point-implicit"):
        s2.rhs_vjp(np.zeros_like(cv0))
    pv = oc.reacting_mixing_layer_3d(mx=20, my=16, mz=10, inviscid_scheme=3)
    d3 = oc.write_case(pv, tmp_path / "pv")
    s3 = ostc.Solver(str(d3))
    s3.set_state(pv.bv, sv=pv.sv)
    with pytest.raises(ostc.OstcError, match="flux-split"):
        s3.rhs_vjp(np.zeros((14,) + s3.shape(0)))


def _fixed_dt_solver(tmp_path, dims, steps_dt_from=None):
    """Noisy reacting layer with a fixed dt (the CFL dt of its initial state): finite differences of
    whole steps then see the same dt the adjoint holds fixed."""
    import ostc

    mx, my, mz = dims
    case = _noisy(oc.reacting_mixing_layer_3d(mx=mx, my=my, mz=mz))
    d = oc.write_case(case, tmp_path / "cfl")
    s = ostc.Solver(str(d))
    s.set_state(case.bv, sv=case.sv)
    dt = s.step(1)
    s.close()
    case.scheme["fixed_time_step"] = 1
    case.scheme["dt"] = dt
    d = oc.write_case(case, tmp_path / "fixed")
    s = ostc.Solver(str(d))
    s.set_state(case.bv, sv=case.sv)
    cv0, _ = s.get_state()
    return s, cv0, case


def _fd_steps(s, case, cv0, v, n, eps=EPS):
    """Richardson-extrapolated central difference of q_n(q_0) along v.  Every perturbed start is set
    from the exact base state (set_state), so that its temperature Newton iteration starts from the
    base T and ends O(eps^2) from the root."""
    d = []
    for h in (2 * eps, eps):
        out = []
        for sg in (1, -1):
            s.set_state(case.bv, sv=case.sv)
            s.set_conservative(cv0 + sg * h * v)
            s.step(n)
            out.append(s.get_state()[0])
        d.append((out[0] - out[1]) / (2 * h))
    s.set_state(case.bv, sv=case.sv)
    return (4 * d[1] - d[0]) / 3


@pytest.mark.parametrize("dims", [(24, 18, 12), (40, 24, 1)], ids=["3d", "2d"])
def test_step_vjp_matches_finite_differences(built, tmp_path, dims):
    """Adjoint of one SSP-RK3 step (dt fixed) against differences of whole steps."""
    s, cv0, case = _fixed_dt_solver(tmp_path, dims)
    rng = np.random.default_rng(21)
    w = rng.standard_normal(cv0.shape)
    g = s.step_vjp(w)
    cv_after, _ = s.get_state()
    assert np.array_equal(cv_after, cv0)  # the state is left as it was
    for v in _directions(cv0, rng, 3):
        jv = _fd_steps(s, case, cv0, v, 1)
        lhs, rhs = float(np.sum(w * jv)), float(np.sum(g * v))
        assert abs(lhs - rhs) <= RTOL * abs(lhs) + ATOL * float(np.sum(np.abs(w * jv))), (lhs, rhs)


def test_checkpointed_trajectory_adjoint(built, tmp_path):
    """ostc_adjoint_steps over 7 steps with a checkpoint every 3 (segments of 3, 3, 1 steps): the
    gradient of <w, q_7> w.r.t. q_0 against differences of 7-step runs, and the context ends at q_7."""
    s, cv0, case = _fixed_dt_solver(tmp_path, (24, 18, 12))
    rng = np.random.default_rng(22)
    w = rng.standard_normal(cv0.shape)
    lam0 = s.adjoint_steps(7, w, every=3)
    q7, _ = s.get_state()
    t7 = s.time()
    s.set_state(case.bv, sv=case.sv)
    s.step(7)
    q7_ref, _ = s.get_state()
    assert np.array_equal(q7, q7_ref)
    assert t7 == s.time()
    for v in _directions(cv0, rng, 2):
        jv = _fd_steps(s, case, cv0, v, 7)
        lhs, rhs = float(np.sum(w * jv)), float(np.sum(lam0 * v))
        assert abs(lhs - rhs) <= RTOL * abs(lhs) + ATOL * float(np.sum(np.abs(w * jv))), (lhs, rhs)
    # the checkpoint spacing does not change the result
    s.set_state(case.bv, sv=case.sv)
    lam1 = s.adjoint_steps(7, w, every=7)
    assert np.max(np.abs(lam1 - lam0)) <= 1e-10 * np.max(np.abs(lam0))


def test_momentum_thickness_gradient_wrt_mode_amplitudes(built, tmp_path):
    """The sensitivity problem of the adjoint: d theta(q_N) / d a_m for the momentum thickness after
    N = 10 steps and the amplitudes a_m of 8 seeded v' modes (a_m = 1/8 at the base), by one
    checkpointed trajectory adjoint (every 4 steps), against Richardson differences of 10-step runs
    in each a_m.  Noisy reacting layer (T, p, Y), fixed dt.

    theta moves by only ~1e-11 per 1e-5 of an amplitude, and the 10-step runs are piecewise smooth
    in a_m at that scale (a stage's temperature Newton iteration count, the |U| kink of the split
    fluxes), so these difference quotients scatter by ~1e-5 of the gradient whatever the step; the
    tolerance here is 1e-4 of the largest component.  The 1e-6 pin of the trajectory adjoint is
    test_checkpointed_trajectory_adjoint."""
    import ostc

    base = _noisy(oc.reacting_mixing_layer_3d(mx=24, my=18, mz=12))
    shapes = oc.mode_shapes(base)
    a0 = np.full(8, 1.0 / 8)
    c0 = oc.add_modes(base, a0, shapes)
    d = oc.write_case(c0, tmp_path / "cfl")
    s = ostc.Solver(str(d))
    s.set_state(c0.bv, sv=c0.sv)
    dt = s.step(1)
    s.close()
    c0.scheme["fixed_time_step"], c0.scheme["dt"] = 1, dt
    d = oc.write_case(c0, tmp_path / "fixed")
    s = ostc.Solver(str(d))
    n, du, dy = 10, c0.extra["du"], c0.extra["h"]
    s.set_state(c0.bv, sv=c0.sv)
    cv0, _ = s.get_state()
    rho0 = float(cv0[0].mean())

    def theta(a):
        c = oc.add_modes(base, a, shapes)
        s.set_state(c.bv, sv=c.sv)
        s.step(n)
        return oc.momentum_thickness(s.get_state()[0], du, rho0, dy)

    _, g_n = theta(a0)
    s.set_state(c0.bv, sv=c0.sv)
    lam0 = s.adjoint_steps(n, g_n, every=4)
    grad_ad = np.array([np.sum(lam0 * dm) for dm in oc.dcv_dmodes(cv0, shapes)])
    h = 1e-5
    grad_fd = np.empty(8)
    for m in range(8):
        e = np.zeros(8)
        e[m] = 1.0
        d1 = (theta(a0 + h * e)[0] - theta(a0 - h * e)[0]) / (2 * h)
        d2 = (theta(a0 + 2 * h * e)[0] - theta(a0 - 2 * h * e)[0]) / (4 * h)
        grad_fd[m] = (4 * d1 - d2) / 3
    assert np.max(np.abs(grad_ad - grad_fd)) <= 1e-4 * np.max(np.abs(grad_fd)), (grad_ad, grad_fd)


def _fixed_dt_air(tmp_path, make):
    """A noisy air layer (see _air_solver) with a fixed dt, the CFL dt of its initial state."""
    import ostc

    case = make()
    s, _ = _air_solver(case, tmp_path)
    dt = s.step(1)
    s.close()
    case.scheme["fixed_time_step"] = 1
    case.scheme["dt"] = dt
    s = ostc.Solver(str(oc.write_case(case, tmp_path / "air_fixed")))
    s.set_state(case.bv)
    return s, s.get_state()[0], case


def _air_steps_err(s, case, cv0, w, lam, v, n):
    """Error of <lam, v> against differences of n-step runs along v, in units of the tolerance, judged
    by the better of steps 1e-7 and 1e-8 (see _check_air)."""
    rhs = float(np.sum(lam * v))
    e = []
    for eps in (1e-7, 1e-8):
        jv = _fd_steps(s, case, cv0, v, n, eps)
        lhs = float(np.sum(w * jv))
        e.append(abs(lhs - rhs) / (RTOL * abs(lhs) + ATOL * float(np.sum(np.abs(w * jv)))))
    return min(e)


@pytest.mark.parametrize("name", ["weno7_hllc_3d", "weno5_ausm_2d"])
def test_air_step_vjp_matches_finite_differences(built, tmp_path, name):
    """Adjoint of one air SSP-RK3 step (dt fixed) against differences of whole steps."""
    s, cv0, case = _fixed_dt_air(tmp_path, AIR[name])
    rng = np.random.default_rng(23)
    w = rng.standard_normal(cv0.shape)
    g = s.step_vjp(w)
    assert np.array_equal(s.get_state()[0], cv0)  # the state is left as it was
    errs = [_air_steps_err(s, case, cv0, w, g, v, 1) for v in _directions(cv0, rng, 3)]
    assert max(errs) <= 1.0, errs


def test_air_checkpointed_trajectory_adjoint(built, tmp_path):
    """ostc_adjoint_steps on the air layer: 5 steps with a checkpoint every 2, against differences of
    5-step runs; the context ends at q_5; the checkpoint spacing does not change the result."""
    s, cv0, case = _fixed_dt_air(tmp_path, AIR["weno7_hllc_3d"])
    rng = np.random.default_rng(24)
    w = rng.standard_normal(cv0.shape)
    lam0 = s.adjoint_steps(5, w, every=2)
    q5, _ = s.get_state()
    s.set_state(case.bv)
    s.step(5)
    assert np.array_equal(q5, s.get_state()[0])
    errs = [_air_steps_err(s, case, cv0, w, lam0, v, 5) for v in _directions(cv0, rng, 2)]
    assert max(errs) <= 1.0, errs
    s.set_state(case.bv)
    lam1 = s.adjoint_steps(5, w, every=5)
    assert np.max(np.abs(lam1 - lam0)) <= 1e-10 * np.max(np.abs(lam0))
