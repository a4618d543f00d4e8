"""Runs the reference solver's own RK3 path (oracle/_ref/ref_harness, built by oracle/ref/build_ref.sh
from the reference sources) on a synthetic case.  TEST INFRASTRUCTURE: used only to generate the
golden fixtures under tests/golden/ that pin the CPU oracle and the CUDA path to the reference.

The case directory gets the same setup.txt, grid and boundary files the library reads, plus the
keys the reference's Driver needs for a plain (non-mixing-layer) start: a `freestream` inflow struct
for its default initialisation and reference state, and neutral values for statistics / sponge /
digital-filter keys it reads without defaults.  The harness then overwrites the interior primitive
state with the case's seeded state and runs Driver::initialize_computation() + RK3() for `steps`
steps on GPU 0.
"""
from __future__ import annotations

import os
import subprocess
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
HARNESS = HERE / "_ref" / "ref_harness"
# the clock value the harness reports to the reference (its inflow noise seed, BoundCond.cu:1731-1734);
# a library run reproduces the noise with ostc_set_inflow_seed(REF_TIME)
REF_TIME = 1700000000

EXTRA = """
// keys the reference reads without defaults (parity runs only)
int initial = 0
string default_init = freestream
int output_file = 100000000
int output_screen = 100000000
int slice_frequency = 100000000
real cfl_steady = 1
bool rho_p_correlation = 0
bool stat_tke_budget = 0
bool stat_species_velocity_correlation = 0
bool stat_species_dissipation_rate = 0
real spongeCoefficient = 1e-8
string mesh_prefix = grid
string result_file = none
int reynolds_stress_supplier = 0
real delta_omega = 1e-3
real total_simulation_time = 1e30
bool use_df = 0
array real sc_passive_scalar {
    0.5
}
array real sct_passive_scalar {
    1.0
}
array string stat_rey_1st {
    u
}
array string stat_species {
    all
}
"""

FREESTREAM = """struct freestream = {
    string type = inflow
    int label = 5
    real mach = @MACH@
    real pressure = @P@
    real temperature = @T@
    real u = 1.0
    real v = 0.0
    real w = 0.0
}
"""


def write_reference_case(case, steps: int, directory: os.PathLike, setup_extra: str = "") -> Path:
    """setup_extra: setup.txt lines appended last (the reference keeps the last value of a key)."""
    import ostc_cases as oc

    d = Path(directory)
    inp = d / "input"
    oc.write_case(case, inp)
    setup = (inp / "setup.txt").read_text()
    setup = setup.replace(f"int total_step = {case.steps}", f"int total_step = {steps}")
    setup = setup.replace("int initial = 1\n", "")
    bv0 = case.blocks[0].bv if hasattr(case, "blocks") else case.bv
    p0 = float(bv0[4].flat[0])
    t0 = float(bv0[5].flat[0])
    ml = getattr(case, "mixing_layer", None)
    # a mixing-layer case names its own delta_omega and its inflow struct `freestream` is the reference
    # state (problem_type 1)
    extra = EXTRA.replace("real delta_omega = 1e-3\n", "") if ml else EXTRA
    if ml and "df_rij" in ml:
        extra = extra.replace("int reynolds_stress_supplier = 0\n", "")
    setup += extra
    own_fs = "freestream" in getattr(case, "bc_structs", {})
    if not case.freestream and not own_fs:
        setup += FREESTREAM.replace("@MACH@", "0.5").replace("@P@", repr(p0)).replace("@T@", repr(t0))
    (inp / "setup.txt").write_text(setup)
    if not case.freestream and not own_fs:
        setup += "string reference_state = freestream\n"
    setup += setup_extra
    (inp / "setup.txt").write_text(setup)
    with open(d / "state_in.bin", "wb") as f:
        for blk in (case.blocks if hasattr(case, "blocks") else [case]):
            np.ascontiguousarray(blk.bv, dtype=np.float64).tofile(f)
            if blk.sv is not None:
                np.ascontiguousarray(blk.sv, dtype=np.float64).tofile(f)
    (d / "output" / "message").mkdir(parents=True, exist_ok=True)
    return d


def run_reference(case, steps: int, workdir: os.PathLike | None = None, timeout: int = 1800,
                  with_seconds: bool = False, setup_extra: str = ""):
    """Returns (cv[n_var,mz,my,mx], bv[6,mz,my,mx], physical time[, sv[n_spec,...] for mixtures]) after
    `steps` reference RK3 steps, and with_seconds the wall time of the reference's RK3 call.  The files
    the reference writes at the end of its run (output/flowfield.plt, output/stat/coll_*.bin when the
    setup collects statistics) stay in `workdir`."""
    if not HARNESS.exists():
        raise FileNotFoundError(f"{HARNESS} not built (oracle/ref/build_ref.sh)")
    d = Path(workdir) if workdir else Path(tempfile.mkdtemp(prefix="ostc_ref_"))
    write_reference_case(case, steps, d, setup_extra)
    r = subprocess.run([str(HARNESS), "state_in.bin", "state_out.bin"], cwd=d, capture_output=True, text=True,
                       timeout=timeout, env=dict(os.environ, OSTC_REF_TIME=str(REF_TIME)))
    if r.returncode != 0:
        raise RuntimeError(f"reference harness failed ({r.returncode}):\n{r.stdout[-4000:]}\n{r.stderr[-3000:]}")
    raw = np.fromfile(d / "state_out.bin", dtype=np.float64)
    if hasattr(case, "blocks"):
        # multi-block: per block [cv(5), bv(6)] interior, then the time
        out, off = [], 0
        for blk in case.blocks:
            nn = blk.nodes
            a = raw[off: off + 11 * nn].reshape((11,) + blk.bv.shape[1:])
            out.append((a[:5].copy(), a[5:].copy()))
            off += 11 * nn
        res = ([o[0] for o in out], [o[1] for o in out], float(raw[off]))
        if with_seconds:
            sec = [float(l.split("=")[1]) for l in r.stdout.splitlines() if "rk3_seconds" in l]
            return res + (sec[0] if sec else float("nan"),)
        return res
    n = case.nodes
    ns = 0 if case.sv is None else case.sv.shape[0]
    nv = 5 + ns
    out = raw[: (nv + 6 + ns) * n].reshape((nv + 6 + ns,) + case.bv.shape[1:])
    res = (out[:nv].copy(), out[nv:nv + 6].copy(), float(raw[(nv + 6 + ns) * n]))
    if ns:
        res = res + (out[nv + 6:].copy(),)
    if with_seconds:
        sec = [float(l.split("=")[1]) for l in r.stdout.splitlines() if "rk3_seconds" in l]
        return res + (sec[0] if sec else float("nan"),)
    return res
