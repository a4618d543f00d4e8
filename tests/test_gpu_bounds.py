"""Index-bounds checks without a memory checker: the bounds-checked build of the library
(libostc_b200_checked.so, -DOSTC_BOUNDS_CHECK) checks every padded-plane and interior index its
kernels form through the block accessors, clamps any index outside the block and raises a flag.
Tiny grids of every path (air AWENO / primitive schemes with each face type, walls, inflows and
back pressure, mixtures with the flux-split schemes, multi-block interfaces with the statistics
collector, the adjoint) run through it in a child process; the
flags must stay 0 and the results must match the oracle as the regular build's do."""
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]
CHECKED = ROOT / "openstc-mixinglayer_b200" / "libostc_b200_checked.so"

CHILD = r'''
import json, sys, tempfile
import numpy as np
sys.path.insert(0, "openstc-mixinglayer_b200/python"); sys.path.insert(0, "oracle")
import ostc, ostc_cases as oc
from oracle import Oracle, MultiOracle
assert ostc.load_library().ostc_bounds_checked() == 1
out = {}
def run(name, case, steps, mixture=False):
    d = oc.write_case(case, tempfile.mkdtemp())
    s = ostc.Solver(str(d)); s.set_state(case.bv, sv=case.sv) if mixture else s.set_state(case.bv)
    s.rhs(7); s.step(steps)
    cg, _ = s.get_state()
    o = Oracle(case); o.set_state(case.bv); o.step(steps)
    co, _, _ = o.get_state()
    err = max(max(m, l) for m, l in oc.relative_errors(cg, co))
    out[name] = {"flags": s.bounds_flags(), "err": err}
    if mixture:
        w = np.random.default_rng(0).standard_normal(cg.shape)
        s.rhs_vjp(w); s.step_vjp(w)
        out[name]["adjoint_flags"] = s.bounds_flags()
    s.close()
run("awe7_hllc_farfield_3d", oc.mixing_layer_3d(mx=12, my=10, mz=8), 2)
run("muscl_roe_2d", oc.mixing_layer_2d(mx=33, my=17, reconstruction=2, inviscid_scheme=2), 2)
run("awe5_ausm_outflow_3d", oc.mixing_layer_3d(mx=12, my=10, mz=8, ybc="outflow", reconstruction=4, inviscid_scheme=3), 2)
run("fr72_3d", oc.reacting_mixing_layer_3d(mx=12, my=10, mz=8), 2, mixture=True)
run("mix71_3d", oc.reacting_mixing_layer_3d(mx=12, my=10, mz=8, inviscid_scheme=71, finite_rate=False), 2, mixture=True)
run("wall_iso_3d", oc.mixing_layer_3d(mx=12, my=10, mz=8, ybc="wall"), 2)
run("wall_adi_2d", oc.mixing_layer_2d(mx=33, my=17, ybc="wall", wall_thermal="adiabatic"), 2)
run("inflow_3d", oc.mixing_layer_3d(mx=12, my=10, mz=8, xbc="inflow"), 2)
sub = oc.mixing_layer_3d(mx=12, my=10, mz=8, xbc="subsonic", ybc="outflow")
sub.bv[1] = np.abs(sub.bv[1]) + 100.0
run("subsonic_back_pressure_3d", sub, 2)
mc = oc.multiblock_mixing_layer_3d(nb=3, lo=10, hi=16, my=10, mz=8, seed=1)
d = oc.write_case(mc, tempfile.mkdtemp())
s = ostc.Solver(str(d))
for b, blk in enumerate(mc.blocks): s.set_state(blk.bv, block=b)
s.stat_enable(0, 31)  # the statistics collector reads every block's ghost layer
s.step(2)
out["multiblock_3"] = {"flags": s.bounds_flags(), "err": 0.0}
print(json.dumps(out))
'''


def test_bounds_checked_build(built):
    sys.path.insert(0, str(ROOT / "openstc-mixinglayer_b200"))
    import build as libbuild

    libbuild.build(checked=True)  # no-op when up to date
    env = dict(os.environ, OSTC_LIBRARY=str(CHECKED))
    r = subprocess.run([sys.executable, "-c", CHILD], cwd=ROOT, env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-3000:]
    res = json.loads(r.stdout.strip().splitlines()[-1])
    for name, v in res.items():
        assert v["flags"] == 0, (name, v)
        assert v.get("adjoint_flags", 0) == 0, (name, v)
        assert v["err"] < 1e-12, (name, v)
