"""ctypes binding of libostc_b200.so (include/ostc.h).

This is the Python face of the C ABI for test harnesses and benchmarks; the library itself is C++ and
CUDA.  Loading fails loudly when the shared library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

PKG_DIR = Path(__file__).resolve().parent.parent
LIB_PATH = PKG_DIR / "libostc_b200.so"

OSTC_HOST, OSTC_DEVICE = 0, 1
PREC_FP64, PREC_MIXED = 0, 1
TERM_INVISCID, TERM_VISCOUS, TERM_SOURCE, TERM_ALL = 1, 2, 4, 7
FLAG_NONPOSITIVE, FLAG_NAN = 1, 2
CHEM_EXPLICIT, CHEM_POINT_IMPLICIT = 0, 1
LAUNCH_GRAPH, LAUNCH_BLOCK_LOOP = 0, 1
STAT_REY_U, STAT_REY_V, STAT_REY_W, STAT_REY_T, STAT_RHO_P = 1, 2, 4, 8, 16
STAT_TKE_BUDGET, STAT_SPECIES_VELOCITY, STAT_SPECIES_DISSIPATION = 32, 64, 128
STAT_GROUPS = ("reynolds_1st", "favre_1st", "reynolds_2nd", "favre_2nd", "tke_budget", "species_velocity_correlation",
               "species_dissipation_rate")

EXPORTS = [
    "ostc_create", "ostc_destroy", "ostc_last_error", "ostc_n_blocks", "ostc_block_dims", "ostc_n_var",
    "ostc_set_precision", "ostc_set_state", "ostc_get_state", "ostc_rhs", "ostc_rk3_step",
    "ostc_physical_time", "ostc_store_residual_reference", "ostc_residual", "ostc_error_flags",
    "ostc_device_view", "ostc_profile_steps", "ostc_total_nodes", "ostc_probe_case", "ostc_timed_steps",
    "ostc_step_kernel_count", "ostc_residual_noalloc", "ostc_set_chem_mode", "ostc_set_conservative",
    "ostc_rhs_vjp", "ostc_rk3_step_vjp", "ostc_adjoint_steps", "ostc_run_states", "ostc_bounds_flags",
    "ostc_bounds_checked", "ostc_stat_enable", "ostc_stat_disable", "ostc_stat_info", "ostc_stat_get",
    "ostc_stat_export", "ostc_stat_import", "ostc_write_plt", "ostc_read_plt", "ostc_tune_report",
    "ostc_set_sweep_variant", "ostc_steady_step", "ostc_dual_time_step", "ostc_set_launch_mode",
    "ostc_set_inflow_seed", "ostc_stat_group_vars",
]


class OstcError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"ostc error {code}: {msg}")
        self.code = code


class ZoneView(ctypes.Structure):
    _fields_ = [("mx", ctypes.c_int), ("my", ctypes.c_int), ("mz", ctypes.c_int), ("ngg", ctypes.c_int),
                ("gz", ctypes.c_int), ("pitch", ctypes.c_int), ("sy", ctypes.c_int), ("sz", ctypes.c_int),
                ("plane", ctypes.c_longlong), ("cv", ctypes.c_void_p), ("bv", ctypes.c_void_p),
                ("mul", ctypes.c_void_p), ("metric", ctypes.c_void_p), ("jac", ctypes.c_void_p)]


_lib = None


def load_library(path: os.PathLike | None = None) -> ctypes.CDLL:
    """Load libostc_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    # OSTC_LIBRARY selects another build of the same ABI (the bounds-checked one in tests)
    p = Path(path) if path else Path(os.environ.get("OSTC_LIBRARY", LIB_PATH))
    if not p.exists():
        raise OstcError(-100, f"{p} not built: run __graft_entry__.build() (nvcc for sm_100a)")
    lib = ctypes.CDLL(str(p))
    vp, ip, dp = ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double)
    lib.ostc_create.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ip, ctypes.POINTER(vp)]
    lib.ostc_destroy.argtypes = [vp]
    lib.ostc_destroy.restype = None
    lib.ostc_last_error.argtypes = [vp]
    lib.ostc_last_error.restype = ctypes.c_char_p
    lib.ostc_n_blocks.argtypes = [vp, ctypes.POINTER(ip)]
    lib.ostc_block_dims.argtypes = [vp, ip, ctypes.POINTER(ip)]
    lib.ostc_n_var.argtypes = [vp, ctypes.POINTER(ip), ctypes.POINTER(ip)]
    lib.ostc_set_precision.argtypes = [vp, ip]
    lib.ostc_set_chem_mode.argtypes = [vp, ip]
    lib.ostc_set_state.argtypes = [vp, ip, vp, vp, ip]
    lib.ostc_get_state.argtypes = [vp, ip, vp, vp, vp, ip]
    lib.ostc_rhs.argtypes = [vp, ip, ctypes.c_uint, vp, ip]
    lib.ostc_set_conservative.argtypes = [vp, ip, vp, ip]
    lib.ostc_rhs_vjp.argtypes = [vp, ip, ctypes.c_uint, vp, vp, ip]
    lib.ostc_rk3_step_vjp.argtypes = [vp, vp, vp, ip]
    lib.ostc_adjoint_steps.argtypes = [vp, ip, ip, vp, vp, ip]
    lib.ostc_run_states.argtypes = [vp, ip, vp, vp, vp, vp, ip]
    lib.ostc_bounds_flags.argtypes = [vp, ctypes.POINTER(ctypes.c_uint)]
    lib.ostc_bounds_checked.argtypes = []
    lib.ostc_stat_enable.argtypes = [vp, ip, ctypes.c_uint]
    lib.ostc_stat_disable.argtypes = [vp]
    lib.ostc_stat_info.argtypes = [vp, ctypes.POINTER(ip), ctypes.POINTER(ip), ctypes.POINTER(ctypes.c_longlong)]
    lib.ostc_stat_get.argtypes = [vp, ip, ip, vp, ip]
    lib.ostc_stat_export.argtypes = [vp, ctypes.c_char_p]
    lib.ostc_stat_import.argtypes = [vp, ctypes.c_char_p]
    lib.ostc_write_plt.argtypes = [vp, ctypes.c_char_p, ip, ctypes.c_double]
    lib.ostc_read_plt.argtypes = [vp, ctypes.c_char_p, dp]
    lib.ostc_rk3_step.argtypes = [vp, ip, dp]
    lib.ostc_physical_time.argtypes = [vp, dp]
    lib.ostc_store_residual_reference.argtypes = [vp]
    lib.ostc_residual.argtypes = [vp, dp]
    lib.ostc_error_flags.argtypes = [vp, ctypes.POINTER(ctypes.c_uint)]
    lib.ostc_device_view.argtypes = [vp, ip, ctypes.POINTER(ZoneView)]
    lib.ostc_profile_steps.argtypes = [vp, ip, ip, ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ip), dp]
    lib.ostc_total_nodes.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
    lib.ostc_tune_report.argtypes = [vp, ip, ip, ip, ctypes.POINTER(ip), ctypes.POINTER(ctypes.c_float), ip]
    lib.ostc_set_sweep_variant.argtypes = [vp, ip, ip, ip]
    lib.ostc_set_launch_mode.argtypes = [vp, ip]
    lib.ostc_set_inflow_seed.argtypes = [vp, ctypes.c_longlong]
    lib.ostc_stat_group_vars.argtypes = [vp, ip, ctypes.POINTER(ctypes.c_int)]
    lib.ostc_steady_step.argtypes = [vp, ip, ctypes.POINTER(ip), dp]
    lib.ostc_dual_time_step.argtypes = [vp, ip, ctypes.POINTER(ip)]
    lib.ostc_timed_steps.argtypes = [vp, ip, dp]
    lib.ostc_step_kernel_count.argtypes = [vp, ctypes.POINTER(ip)]
    lib.ostc_residual_noalloc.argtypes = [vp, vp, ctypes.c_longlong, dp, vp]
    lib.ostc_probe_case.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(ip), ctypes.c_char_p, ip]
    if path is None:
        _lib = lib
    return lib


def probe_case(input_dir: str, setup: str | None = None) -> dict:
    """Parse a case directory on the host only (no GPU): derived values the reference computes."""
    lib = load_library()
    out = (ctypes.c_int * 16)()
    msg = ctypes.create_string_buffer(512)
    rc = lib.ostc_probe_case((setup or "").encode(), str(input_dir).encode(), out, msg, 512)
    if rc != 0:
        raise OstcError(rc, msg.value.decode())
    keys = ["ngg", "inviscid_type", "n_var", "n_scalar", "n_block", "dimension", "mx", "my", "mz",
            "n_faces", "reconstruction", "inviscid_scheme", "viscous_order", "n_bc_launches"]
    return {k: out[i] for i, k in enumerate(keys)}


def residual_noalloc(bv_new_ptr: int, bv_old_ptr: int, n_nodes: int, stream: int = 0) -> np.ndarray:
    """RMS changes of rho, |V|, p, T between two device states [6][n_nodes] without any device
    allocation (ostc_residual_noalloc)."""
    lib = load_library()
    r = (ctypes.c_double * 4)()
    rc = lib.ostc_residual_noalloc(ctypes.c_void_p(bv_new_ptr), ctypes.c_void_p(bv_old_ptr), n_nodes, r,
                                   ctypes.c_void_p(stream) if stream else None)
    if rc != 0:
        raise OstcError(rc, lib.ostc_last_error(None).decode())
    return np.array(r[:])


def _ptr(a: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data)


class Solver:
    """One library context on one GPU (RHS + SSP-RK3 for a reference-format case directory)."""

    def __init__(self, input_dir: str, setup: str | None = None, device: int = 0):
        self.lib = load_library()
        h = ctypes.c_void_p()
        rc = self.lib.ostc_create((setup or "").encode(), str(input_dir).encode(), device, ctypes.byref(h))
        if rc != 0:
            raise OstcError(rc, self.lib.ostc_last_error(None).decode())
        self.h = h
        n = ctypes.c_int()
        self._check(self.lib.ostc_n_blocks(self.h, ctypes.byref(n)))
        self.n_block = n.value
        self.dims = []
        for b in range(self.n_block):
            d = (ctypes.c_int * 4)()
            self._check(self.lib.ostc_block_dims(self.h, b, d))
            self.dims.append(tuple(d))
        nv, ns = ctypes.c_int(), ctypes.c_int()
        self._check(self.lib.ostc_n_var(self.h, ctypes.byref(nv), ctypes.byref(ns)))
        self.n_var, self.n_scalar = nv.value, ns.value

    def _check(self, rc: int):
        if rc < 0:
            raise OstcError(rc, self.lib.ostc_last_error(self.h).decode())
        return rc

    def close(self):
        if getattr(self, "h", None):
            self.lib.ostc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def shape(self, block: int = 0):
        mx, my, mz, _ = self.dims[block]
        return (mz, my, mx)

    def set_precision(self, mode: int):
        self._check(self.lib.ostc_set_precision(self.h, mode))

    def set_chem_mode(self, mode: int):
        self._check(self.lib.ostc_set_chem_mode(self.h, mode))

    def set_state(self, bv: np.ndarray, block: int = 0, sv: np.ndarray | None = None):
        """bv [6][mz][my][mx] (rho, u, v, w, p, T); sv [n_spec][mz][my][mx] mass fractions for mixtures."""
        bv = np.ascontiguousarray(bv, dtype=np.float64)
        assert bv.shape == (6,) + self.shape(block), bv.shape
        if sv is not None:
            sv = np.ascontiguousarray(sv, dtype=np.float64)
            assert sv.shape == (self.n_scalar,) + self.shape(block), sv.shape
        self._check(self.lib.ostc_set_state(self.h, block, _ptr(bv), None if sv is None else _ptr(sv), OSTC_HOST))

    def set_state_ptr(self, bv_ptr: int, block: int = 0, kind: int = OSTC_HOST):
        self._check(self.lib.ostc_set_state(self.h, block, ctypes.c_void_p(bv_ptr), None, kind))

    def get_state(self, block: int = 0):
        sh = self.shape(block)
        cv = np.empty((self.n_var,) + sh)
        bv = np.empty((6,) + sh)
        self._check(self.lib.ostc_get_state(self.h, block, _ptr(cv), _ptr(bv), None, OSTC_HOST))
        return cv, bv

    def get_species(self, block: int = 0) -> np.ndarray:
        """Mass fractions sv [n_spec][mz][my][mx] of a mixture case."""
        sv = np.empty((self.n_scalar,) + self.shape(block))
        self._check(self.lib.ostc_get_state(self.h, block, None, None, _ptr(sv), OSTC_HOST))
        return sv

    def get_state_ptr(self, cv_ptr: int, bv_ptr: int, block: int = 0, kind: int = OSTC_HOST):
        self._check(self.lib.ostc_get_state(self.h, block, ctypes.c_void_p(cv_ptr) if cv_ptr else None,
                                            ctypes.c_void_p(bv_ptr) if bv_ptr else None, None, kind))

    def rhs(self, mask: int = TERM_ALL, block: int = 0) -> np.ndarray:
        dq = np.empty((self.n_var,) + self.shape(block))
        self._check(self.lib.ostc_rhs(self.h, block, mask, _ptr(dq), OSTC_HOST))
        return dq

    def set_conservative(self, cv: np.ndarray, block: int = 0):
        """Interior conservative state [n_var][k][j][i]; primitive state, ghosts and properties follow."""
        cv = np.ascontiguousarray(cv, dtype=np.float64)
        self._check(self.lib.ostc_set_conservative(self.h, block, _ptr(cv), OSTC_HOST))

    def rhs_vjp(self, dq_bar: np.ndarray, mask: int = TERM_ALL, block: int = 0) -> np.ndarray:
        """(d rhs / d cv)^T dq_bar at the current state, same layout as rhs()."""
        dq_bar = np.ascontiguousarray(dq_bar, dtype=np.float64)
        cv_bar = np.empty((self.n_var,) + self.shape(block))
        self._check(self.lib.ostc_rhs_vjp(self.h, block, mask, _ptr(dq_bar), _ptr(cv_bar), OSTC_HOST))
        return cv_bar

    def run_states_ptr(self, bv_in: list, bv_out: list, n_steps: int = 1, sv_in=None, sv_out=None):
        """ostc_run_states over host pointers (ints, ideally pinned memory): state i from bv_in[i]
        (sv_in[i]), advanced n_steps steps, written to bv_out[i] (sv_out[i])."""
        n = len(bv_in)
        arr = lambda ps: (ctypes.c_void_p * n)(*[ctypes.c_void_p(p) for p in ps]) if ps is not None else None
        self._check(self.lib.ostc_run_states(self.h, n, arr(bv_in), arr(sv_in), arr(bv_out), arr(sv_out), n_steps))

    def run_states(self, bv_in: list, n_steps: int = 1, sv_in=None):
        """Advance each of the (bv, sv) host states n_steps steps; returns the list of (bv, sv) results."""
        bvi = [np.ascontiguousarray(b, dtype=np.float64) for b in bv_in]
        svi = None if sv_in is None else [np.ascontiguousarray(x, dtype=np.float64) for x in sv_in]
        bvo = [np.empty_like(b) for b in bvi]
        svo = None if svi is None else [np.empty_like(x) for x in svi]
        self.run_states_ptr([b.ctypes.data for b in bvi], [b.ctypes.data for b in bvo], n_steps,
                            None if svi is None else [x.ctypes.data for x in svi],
                            None if svo is None else [x.ctypes.data for x in svo])
        return list(zip(bvo, svo if svo is not None else [None] * len(bvo)))

    # ---- Tecplot flow-field file (FieldIO / read_flowfield)
    def write_plt(self, path: str, ngg_out: int = 0, solution_time: float | None = None):
        """Write the current state as the reference's flowfield.plt (binary Tecplot V112)."""
        t = self.time() if solution_time is None else solution_time
        self._check(self.lib.ostc_write_plt(self.h, str(path).encode(), ngg_out, t))

    def read_plt(self, path: str) -> float:
        """Restart every block from a flowfield.plt; returns the file's solution time."""
        t = ctypes.c_double()
        self._check(self.lib.ostc_read_plt(self.h, str(path).encode(), ctypes.byref(t)))
        return t.value

    # ---- single-point statistics (SinglePointStat)
    def stat_enable(self, start_step: int = 0, flags: int = 0):
        """Zero the accumulators and collect after every later step whose index (from this call,
        1-based) exceeds start_step; flags: STAT_REY_* extras and STAT_RHO_P."""
        self._check(self.lib.ostc_stat_enable(self.h, start_step, flags))

    def stat_disable(self):
        self._check(self.lib.ostc_stat_disable(self.h))

    def stat_info(self):
        """(variables per group, collections, steps since enabling)."""
        nv = (ctypes.c_int * 4)()
        nc = ctypes.c_int()
        st = ctypes.c_longlong()
        self._check(self.lib.ostc_stat_info(self.h, nv, ctypes.byref(nc), ctypes.byref(st)))
        return list(nv), nc.value, st.value

    def stat_group_vars(self, group: int) -> int:
        n = ctypes.c_int()
        self._check(self.lib.ostc_stat_group_vars(self.h, group, ctypes.byref(n)))
        return n.value

    def stat_get(self, group: int, block: int = 0) -> np.ndarray:
        """Sums of group (0 Reynolds 1st, 1 Favre 1st, 2 Reynolds 2nd, 3 Favre 2nd: [n_var, mz + 2, my + 2,
        mx + 2], one ghost layer on every side; 4 TKE budget, 5 species velocity correlation, 6 species
        dissipation rate: [n_var, mz, my, mx]) of block."""
        nv = self.stat_group_vars(group)
        mz, my, mx = self.shape(block)
        g = 1 if group < 4 else 0
        out = np.empty((nv, mz + 2 * g, my + 2 * g, mx + 2 * g))
        self._check(self.lib.ostc_stat_get(self.h, block, group, out.ctypes.data, OSTC_HOST))
        return out

    def stat_export(self, directory: str):
        self._check(self.lib.ostc_stat_export(self.h, str(directory).encode()))

    def stat_import(self, directory: str):
        self._check(self.lib.ostc_stat_import(self.h, str(directory).encode()))

    def bounds_flags(self) -> int:
        """Index-bounds flags of the bounds-checked build (read and cleared; 0 in the regular build)."""
        f = ctypes.c_uint()
        self._check(self.lib.ostc_bounds_flags(self.h, ctypes.byref(f)))
        return f.value

    def step_vjp(self, lam_out: np.ndarray) -> np.ndarray:
        """(d q' / d q)^T lam_out for one RK3 step from the current state (dt held fixed)."""
        lam_out = np.ascontiguousarray(lam_out, dtype=np.float64)
        lam_in = np.empty_like(lam_out)
        self._check(self.lib.ostc_rk3_step_vjp(self.h, _ptr(lam_out), _ptr(lam_in), OSTC_HOST))
        return lam_in

    def adjoint_steps(self, n_steps: int, lam_final: np.ndarray, every: int = 20) -> np.ndarray:
        """Advance n_steps and return (d q_N / d q_0)^T lam_final (checkpoint every `every` steps)."""
        lam_final = np.ascontiguousarray(lam_final, dtype=np.float64)
        lam0 = np.empty_like(lam_final)
        self._check(self.lib.ostc_adjoint_steps(self.h, n_steps, every, _ptr(lam_final), _ptr(lam0), OSTC_HOST))
        return lam0

    def step(self, n: int = 1) -> float:
        dt = ctypes.c_double()
        self._check(self.lib.ostc_rk3_step(self.h, n, ctypes.byref(dt)))
        return dt.value

    def step_async(self, n: int = 1):
        self._check(self.lib.ostc_rk3_step(self.h, n, None))

    def timed_steps(self, n: int) -> float:
        """Advance n steps; device milliseconds between events on the library's stream."""
        ms = ctypes.c_double()
        self._check(self.lib.ostc_timed_steps(self.h, n, ctypes.byref(ms)))
        return ms.value

    def step_kernel_count(self) -> int:
        k = ctypes.c_int()
        self._check(self.lib.ostc_step_kernel_count(self.h, ctypes.byref(k)))
        return k.value

    def time(self) -> float:
        t = ctypes.c_double()
        self._check(self.lib.ostc_physical_time(self.h, ctypes.byref(t)))
        return t.value

    def store_residual_reference(self):
        self._check(self.lib.ostc_store_residual_reference(self.h))

    def residual(self) -> np.ndarray:
        r = (ctypes.c_double * 4)()
        self._check(self.lib.ostc_residual(self.h, r))
        return np.array(r[:])

    def error_flags(self) -> int:
        f = ctypes.c_uint()
        self._check(self.lib.ostc_error_flags(self.h, ctypes.byref(f)))
        return f.value

    def device_view(self, block: int = 0) -> ZoneView:
        v = ZoneView()
        self._check(self.lib.ostc_device_view(self.h, block, ctypes.byref(v)))
        return v

    def total_nodes(self) -> int:
        n = ctypes.c_longlong()
        self._check(self.lib.ostc_total_nodes(self.h, ctypes.byref(n)))
        return n.value

    def steady(self, n: int = 1):
        """Up to n iterations of the steady driver (ostc_steady_step): (iterations run, last scaled
        residual or -1)."""
        done = ctypes.c_int()
        err = ctypes.c_double()
        self._check(self.lib.ostc_steady_step(self.h, n, ctypes.byref(done), ctypes.byref(err)))
        return done.value, err.value

    def dual(self, n: int = 1) -> int:
        """n physical steps of dual time stepping (ostc_dual_time_step); the inner-iteration count in
        force afterwards."""
        inner = ctypes.c_int()
        self._check(self.lib.ostc_dual_time_step(self.h, n, ctypes.byref(inner)))
        return inner.value

    def set_inflow_seed(self, seed: int):
        """Reseed the white-noise inflow generators (curand_init(seed + i, i, 0) per face-plane node)."""
        self._check(self.lib.ostc_set_inflow_seed(self.h, seed))

    def set_launch_mode(self, mode: int):
        """LAUNCH_GRAPH (one CUDA graph per step) or LAUNCH_BLOCK_LOOP (every kernel launched from the host,
        block after block, as the reference's per-block loop does)."""
        self._check(self.lib.ostc_set_launch_mode(self.h, mode))

    def set_sweep_variant(self, dir: int, variant: int, precision: int = 0):
        """Pin sweep `dir` (0/1/2 = x/y/z) to kernel variant `variant` (-1: back to the autotuner)."""
        self._check(self.lib.ostc_set_sweep_variant(self.h, precision, dir, variant))

    def tune_report(self, dir: int, precision: int = 0, block: int = 0):
        """(chosen variant, [ms per launch of each variant]) from the sweep autotuner (dir 0/1/2 = x/y/z)."""
        chosen = ctypes.c_int()
        ms = (ctypes.c_float * 8)()
        n = self._check(self.lib.ostc_tune_report(self.h, block, precision, dir, ctypes.byref(chosen), ms, 8))
        return chosen.value, list(ms[:n])

    def profile(self, n_steps: int) -> dict:
        mx = 32
        names = (ctypes.c_char_p * mx)()
        launches = (ctypes.c_int * mx)()
        ms = (ctypes.c_double * mx)()
        k = self._check(self.lib.ostc_profile_steps(self.h, n_steps, mx, names, launches, ms))
        return {names[i].decode(): (launches[i], ms[i]) for i in range(k)}
