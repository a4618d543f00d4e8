"""ctypes binding of the CPU oracle (oracle/ostc_oracle.c).

TEST INFRASTRUCTURE: used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg only, as the
checker or the timed CPU baseline.  The oracle restates the reference OpenSTC RHS + SSP-RK3 path for
calorically perfect air in serial FP64 C; each routine cites the reference file:line it follows.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "libostc_oracle.so"


class OrcFace(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int), ("raw", ctypes.c_int * 6)] + [
        (n, ctypes.c_double) for n in ("density", "u", "v", "w", "pressure", "temperature", "acoustic_speed",
                                       "gamma", "entropy", "mw")] + [("wall_adiabatic", ctypes.c_int), ("y", ctypes.c_double * 16),
                                                                     ("inflow_type", ctypes.c_int),
                                                                     ("delta_omega", ctypes.c_double),
                                                                     ("lower", ctypes.c_double * 6),
                                                                     ("y_lower", ctypes.c_double * 16)]


MAXS, MAXR = 16, 64


class OrcChem(ctypes.Structure):
    D, I = ctypes.c_double, ctypes.c_int
    _fields_ = [("n_spec", I), ("n_reac", I), ("mw", D * MAXS), ("t_low", D * MAXS), ("t_mid", D * MAXS),
                ("low", D * (MAXS * 7)), ("high", D * (MAXS * 7)), ("lj_potent_inv", D * MAXS),
                ("vis_coeff", D * MAXS), ("wj_div_wi_1_4", D * (MAXS * MAXS)), ("sqrt_wiwj_8", D * (MAXS * MAXS)),
                ("binary_diff", D * (MAXS * MAXS)), ("kb_over_eps_jk", D * (MAXS * MAXS)), ("label", I * MAXR),
                ("rev_type", I * MAXR), ("order", I * MAXR), ("stoi_f", I * (MAXR * MAXS)),
                ("stoi_b", I * (MAXR * MAXS)), ("A", D * MAXR), ("b", D * MAXR), ("Ea", D * MAXR), ("A2", D * MAXR),
                ("b2", D * MAXR), ("Ea2", D * MAXR), ("third_body", D * (MAXR * MAXS)), ("troe_alpha", D * MAXR),
                ("troe_t3", D * MAXR), ("troe_t1", D * MAXR), ("troe_t2", D * MAXR)]


class OrcInner(ctypes.Structure):
    _fields_ = [("raw", ctypes.c_int * 7), ("traw", ctypes.c_int * 7)]


def chem_struct(t) -> OrcChem:
    """ctypes copy of oracle/chem.py tables (row-major, first n_spec / n_reac entries used)."""
    c = OrcChem()
    c.n_spec, c.n_reac = t.n_spec, t.n_reac
    for name, _ in OrcChem._fields_[2:]:
        v = getattr(t, name, None)
        if v is None:
            continue
        flat = np.asarray(v).ravel()
        arr = getattr(c, name)
        for i, x in enumerate(flat):
            arr[i] = x
    return c


class OrcCase(ctypes.Structure):
    _fields_ = [("mx", ctypes.c_int), ("my", ctypes.c_int), ("mz", ctypes.c_int), ("reconstruction", ctypes.c_int),
                ("inviscid_scheme", ctypes.c_int), ("riemann", ctypes.c_int), ("entropy_fix_factor", ctypes.c_double),
                ("viscous_order", ctypes.c_int), ("cfl", ctypes.c_double),
                ("prandtl", ctypes.c_double), ("fixed_time_step", ctypes.c_int), ("dt", ctypes.c_double),
                ("n_face", ctypes.c_int), ("face", OrcFace * 16), ("n_spec", ctypes.c_int),
                ("finite_rate", ctypes.c_int), ("chem", ctypes.POINTER(OrcChem)), ("weno_eps_scale", ctypes.c_double),
                ("v_ref", ctypes.c_double), ("has_init", ctypes.c_int), ("init_bv", ctypes.c_double * 6),
                ("init_sv", ctypes.c_double * MAXS), ("chem_mode", ctypes.c_int), ("implicit_method", ctypes.c_int),
                ("dplur_inner", ctypes.c_int), ("chem_src_method", ctypes.c_int), ("inner_iteration", ctypes.c_int),
                ("max_inner_iteration", ctypes.c_int), ("iteration_adjust_step", ctypes.c_int),
                ("problem_type", ctypes.c_int), ("ml_upper", ctypes.c_double * 6), ("ml_lower", ctypes.c_double * 6),
                ("ml_y_upper", ctypes.c_double * MAXS), ("ml_y_lower", ctypes.c_double * MAXS),
                ("ml_delta_omega", ctypes.c_double)]


def riemann_of(reconstruction: int, inviscid_scheme: int) -> int:
    """Riemann solver the reference's switches select: 1 LF, 2 Roe, 3 AUSM+, 4 HLLC.  Roe only with a
    primitive reconstruction (inviscid_type 2, Parameter.cpp:264-278); every unlisted scheme falls to
    AUSM+ (InviscidScheme.cu:145-159, 345-359)."""
    if inviscid_scheme == 2 and reconstruction in (1, 2, 3):
        return 2
    return inviscid_scheme if inviscid_scheme in (1, 4) else 3


def _set_init(c, case):
    ml = case.mixing_layer_streams() if getattr(case, "mixing_layer", None) else None
    if ml is not None:
        # problem_type 1: every node starts from the two-stream profile
        c.problem_type = 1
        for q in range(6):
            c.ml_upper[q], c.ml_lower[q] = ml["upper"][q], ml["lower"][q]
        for q, (a, b) in enumerate(zip(ml["y_upper"], ml["y_lower"])):
            c.ml_y_upper[q], c.ml_y_lower[q] = a, b
        c.ml_delta_omega = ml["delta_omega"]
    st = case.default_state() if hasattr(case, "default_state") else None
    if st is not None:
        bv, y = st
        c.has_init = 1
        for q in range(6):
            c.init_bv[q] = bv[q]
        for q, v in enumerate(y):
            c.init_sv[q] = v


def build() -> Path:
    subprocess.run(["make", "-C", str(HERE)], check=True, capture_output=True)
    return LIB


_lib = None


def load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        lib = ctypes.CDLL(str(LIB))
        vp, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)
        lib.orc_create.argtypes = [ctypes.POINTER(OrcCase), dp, dp, dp]
        lib.orc_create.restype = vp
        lib.orc_destroy.argtypes = [vp]
        lib.orc_ngg.argtypes = [vp]
        lib.orc_set_state.argtypes = [vp, dp]
        lib.orc_set_state_sv.argtypes = [vp, dp, dp]
        lib.orc_get_mixture.argtypes = [vp, dp, dp, dp, dp, dp]
        lib.orc_get_state.argtypes = [vp, dp, dp, dp]
        lib.orc_get_metric.argtypes = [vp, dp, dp]
        lib.orc_rhs.argtypes = [vp, ctypes.c_uint, dp]
        lib.orc_step.argtypes = [vp, ctypes.c_int]
        lib.orc_step.restype = ctypes.c_double
        lib.orc_steady.argtypes = [vp, ctypes.c_int]
        lib.orc_steady.restype = None
        lib.orc_dual.argtypes = [vp, ctypes.c_int]
        lib.orc_dual.restype = ctypes.c_int
        lib.orc_stat_collect.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.c_int, dp]
        lib.orc_stat_extra.argtypes = [vp, vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int), vp, vp]
        lib.orc_time.argtypes = [vp]
        lib.orc_time.restype = ctypes.c_double
        lib.orc_dt.argtypes = [vp]
        lib.orc_dt.restype = ctypes.c_double
        lib.orc_multi_create.argtypes = [ctypes.c_int, ctypes.POINTER(OrcCase), ctypes.POINTER(dp),
                                         ctypes.POINTER(dp), ctypes.POINTER(dp), ctypes.POINTER(ctypes.c_int),
                                         ctypes.POINTER(OrcInner)]
        lib.orc_multi_create.restype = vp
        lib.orc_multi_destroy.argtypes = [vp]
        lib.orc_multi_block.argtypes = [vp, ctypes.c_int]
        lib.orc_multi_block.restype = vp
        lib.orc_multi_set_state.argtypes = [vp, ctypes.POINTER(dp), ctypes.POINTER(dp)]
        lib.orc_multi_step.argtypes = [vp, ctypes.c_int]
        lib.orc_multi_step.restype = ctypes.c_double
        _lib = lib
    return _lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


dp_arr = ctypes.POINTER(ctypes.c_double)


class Oracle:
    """CPU restatement of one single-block case (see ostc_cases.Case)."""

    def __init__(self, case, chem_mode: int = 0):
        self.lib = load()
        c = OrcCase()
        c.chem_mode = chem_mode
        c.mx, c.my, c.mz = case.mx, case.my, case.mz
        s = case.scheme
        c.reconstruction, c.inviscid_scheme, c.viscous_order = s["reconstruction"], s["inviscid_scheme"], s["viscous_order"]
        c.riemann = riemann_of(s["reconstruction"], s["inviscid_scheme"])
        c.entropy_fix_factor = s.get("entropy_fix_factor", 0.125)
        c.cfl, c.prandtl = s["cfl"], s["prandtl_number"]
        c.fixed_time_step, c.dt = 0, 1e-8
        c.implicit_method, c.dplur_inner = s.get("implicit_method", 0), s.get("dplur_inner_step", 3)
        c.chem_src_method = s.get("chem_src_method", 0)
        c.inner_iteration, c.max_inner_iteration = s.get("inner_iteration", 20), s.get("max_inner_iteration", 30)
        c.iteration_adjust_step = s.get("iteration_adjust_step", 20)
        self.steady_case = bool(s.get("steady", 0))
        self.dual_case = not self.steady_case and s.get("temporal_scheme", 3) == 2
        if self.dual_case:
            c.fixed_time_step, c.dt = 1, s.get("dt", 1e-8)
        types = case.label_types()
        ff = {**case.farfield_states(), **case.wall_states(), **case.inflow_states(),
              **case.characteristic_states()}
        c.n_face = len(case.faces)
        for n, f in enumerate(case.faces):
            c.face[n].type = types[f.label]
            for q in range(6):
                c.face[n].raw[q] = f.raw[q]
            if f.label in ff:
                for k, v in ff[f.label].items():
                    if k in ("y", "y_lower"):
                        v = (ctypes.c_double * 16)(*v)
                    elif k == "lower":
                        v = (ctypes.c_double * 6)(*v)
                    setattr(c.face[n], k, v)
        self.n_spec = 0
        mix = getattr(case, "mixture", None)
        if mix is not None:
            import chem  # the full restated tables (thermo, transport, reactions) of the same files
            tables = chem.read(mix["chem_dir"], mix["mechanism"], mix["therm"], mix["tran"],
                               reactions=mix["finite_rate"])
            self.tables = tables
            self._chem = chem_struct(tables)
            c.chem = ctypes.pointer(self._chem)
            c.n_spec = self.n_spec = tables.n_spec
            c.finite_rate = 1 if mix["finite_rate"] else 0
        c.weno_eps_scale, c.v_ref = case.reference_scales()
        _set_init(c, case)
        self.case = case
        self.shape = (case.mz, case.my, case.mx)
        x = np.ascontiguousarray(case.x * case.grid_scale, dtype=np.float64)
        y = np.ascontiguousarray(case.y * case.grid_scale, dtype=np.float64)
        z = np.ascontiguousarray(case.z * case.grid_scale, dtype=np.float64)
        if case.mz == 1:
            # 2-D: the reference scales z too, but builds k ghosts at unit spacing after scaling
            z = np.ascontiguousarray(case.z * case.grid_scale, dtype=np.float64)
        self._c = c
        self.h = self.lib.orc_create(ctypes.byref(c), _dp(x), _dp(y), _dp(z))

    def close(self):
        if self.h:
            self.lib.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, bv: np.ndarray, sv: np.ndarray | None = None):
        bv = np.ascontiguousarray(bv, dtype=np.float64)
        if sv is None and getattr(self.case, "sv", None) is not None and self.n_spec:
            sv = self.case.sv
        if self.n_spec:
            sv = np.ascontiguousarray(sv, dtype=np.float64)
            self.lib.orc_set_state_sv(self.h, _dp(bv), _dp(sv))
        else:
            self.lib.orc_set_state(self.h, _dp(bv))

    def mixture(self):
        """Interior Y_k, conductivity, rho D_k, acoustic speed, gamma."""
        sv = np.empty((self.n_spec,) + self.shape)
        rd = np.empty((self.n_spec,) + self.shape)
        cond, ac, ga = np.empty(self.shape), np.empty(self.shape), np.empty(self.shape)
        self.lib.orc_get_mixture(self.h, _dp(sv), _dp(cond), _dp(rd), _dp(ac), _dp(ga))
        return dict(sv=sv, cond=cond, rho_d=rd, acoustic=ac, gamma=ga)

    def get_state(self):
        cv = np.empty((5 + self.n_spec,) + self.shape)
        bv = np.empty((6,) + self.shape)
        mul = np.empty(self.shape)
        self.lib.orc_get_state(self.h, _dp(cv), _dp(bv), _dp(mul))
        return cv, bv, mul

    def metric(self):
        m = np.empty((9,) + self.shape)
        j = np.empty(self.shape)
        self.lib.orc_get_metric(self.h, _dp(m), _dp(j))
        return m, j

    def rhs(self, mask: int = 3) -> np.ndarray:
        dq = np.empty((5 + self.n_spec,) + self.shape)
        self.lib.orc_rhs(self.h, mask, _dp(dq))
        return dq

    def step(self, n: int = 1) -> float:
        return self.lib.orc_step(self.h, n)

    def steady(self, n: int = 1):
        """n iterations of the steady driver (local time steps, explicit / EPI / DA / DPLUR)."""
        self.lib.orc_steady(self.h, n)

    def dual(self, n: int = 1) -> int:
        """n physical steps of dual time stepping; the inner-iteration count in force afterwards."""
        return self.lib.orc_dual(self.h, n)

    def advance(self, n: int):
        """n steps of the case's own time-advance driver: steady iterations, dual-time or SSP-RK3 steps."""
        if self.steady_case:
            return self.steady(n)
        return self.dual(n) if self.dual_case else self.step(n)

    def stat_collect(self, acc: np.ndarray, rey_idx=(), rho_p: bool = False):
        """Add one single-point statistics collection of the current state to acc (float64,
        C-contiguous, the four groups [n_var][mz+2][my+2][mx+2] back to back; orc_stat_collect)."""
        assert acc.dtype == np.float64 and acc.flags.c_contiguous
        idx = (ctypes.c_int * max(1, len(rey_idx)))(*rey_idx)
        self.lib.orc_stat_collect(self.h, len(rey_idx), idx, int(rho_p), _dp(acc))

    def stat_extra(self, tke=None, svc=None, sdr=None, ss_idx=()):
        """Add one collection of the additional statistics of the current state (orc_stat_extra): tke
        [7, mz, my, mx], and for the species ss_idx svc [3 nss, ...] and sdr [5 nss, ...]; None skips."""
        def ptr(a):
            if a is None:
                return None
            assert a.dtype == np.float64 and a.flags.c_contiguous
            return a.ctypes.data
        idx = (ctypes.c_int * max(1, len(ss_idx)))(*ss_idx)
        self.lib.orc_stat_extra(self.h, ptr(tke), len(ss_idx), idx, ptr(svc), ptr(sdr))

    def time(self) -> float:
        return self.lib.orc_time(self.h)

    def dt(self) -> float:
        return self.lib.orc_dt(self.h)


class _BlockView:
    """Per-block accessor of a multi-block oracle (state, metric) sharing the Oracle methods."""

    def __init__(self, lib, h, shape, n_spec):
        self.lib, self.h, self.shape, self.n_spec = lib, h, shape, n_spec

    get_state = Oracle.get_state
    stat_collect = Oracle.stat_collect
    stat_extra = Oracle.stat_extra
    metric = Oracle.metric
    mixture = Oracle.mixture
    time = Oracle.time


class MultiOracle:
    """CPU restatement of a multi-block case (ostc_cases.MultiCase): per-block contexts joined by the
    interface exchange of the reference (orc_multi_*)."""

    def __init__(self, case):
        self.lib = load()
        nb = len(case.blocks)
        cases = (OrcCase * nb)()
        types = case.label_types()
        ff = {**case.farfield_states(), **case.wall_states(), **case.inflow_states(),
              **case.characteristic_states()}
        self._keep = []
        xs, ys, zs = (dp_arr * nb)(), (dp_arr * nb)(), (dp_arr * nb)()
        for b, blk in enumerate(case.blocks):
            c = cases[b]
            c.mx, c.my, c.mz = blk.mx, blk.my, blk.mz
            sch = case.scheme
            c.reconstruction, c.inviscid_scheme, c.viscous_order = sch["reconstruction"], sch["inviscid_scheme"], sch["viscous_order"]
            c.riemann = riemann_of(sch["reconstruction"], sch["inviscid_scheme"])
            c.entropy_fix_factor = sch.get("entropy_fix_factor", 0.125)
            c.cfl, c.prandtl = sch["cfl"], sch["prandtl_number"]
            c.fixed_time_step, c.dt = 0, 1e-8
            c.n_face = len(blk.faces)
            for n, f in enumerate(blk.faces):
                c.face[n].type = types[f.label]
                for q in range(6):
                    c.face[n].raw[q] = f.raw[q]
                if f.label in ff:
                    for k, v in ff[f.label].items():
                        setattr(c.face[n], k, (ctypes.c_double * 16)(*v) if k == "y" else v)
            c.weno_eps_scale, c.v_ref = case.reference_scales()
            _set_init(c, case)
            for arr, src in ((xs, blk.x), (ys, blk.y), (zs, blk.z)):
                a = np.ascontiguousarray(src * case.grid_scale, dtype=np.float64)
                self._keep.append(a)
                arr[b] = _dp(a)
        nin = (ctypes.c_int * nb)(*[len(b.inner) for b in case.blocks])
        allf = [f for b in case.blocks for f in b.inner]
        inner = (OrcInner * max(1, len(allf)))()
        for i, (src, tar) in enumerate(allf):
            for q in range(7):
                inner[i].raw[q], inner[i].traw[q] = src[q], tar[q]
        self.h = self.lib.orc_multi_create(nb, cases, xs, ys, zs, nin, inner)
        self.case = case
        self.blocks = [_BlockView(self.lib, self.lib.orc_multi_block(self.h, b), (blk.mz, blk.my, blk.mx), 0)
                       for b, blk in enumerate(case.blocks)]

    def close(self):
        if self.h:
            self.lib.orc_multi_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self):
        nb = len(self.case.blocks)
        bvs = [np.ascontiguousarray(b.bv, dtype=np.float64) for b in self.case.blocks]
        self._state = bvs
        arr = (dp_arr * nb)(*[_dp(a) for a in bvs])
        self.lib.orc_multi_set_state(self.h, arr, None)

    def step(self, n: int = 1) -> float:
        return self.lib.orc_multi_step(self.h, n)

    def time(self) -> float:
        return self.blocks[0].time()
