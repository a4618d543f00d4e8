"""Run one synthetic mixing-layer workload through the library and print its device time per step.

    python openstc-mixinglayer_b200/python/run_case.py --case reacting --dims 192 96 64 --steps 2

Cases: ``air`` (3-D temporal mixing layer, AWENO7 + HLLC, viscous), ``reacting`` (9-species H2/air
layer, flux-split characteristic WENO7, finite-rate chemistry) and ``multiblock`` (the uneven 12-block
chain).  Used as the short command under a profiler, where a full benchmark would launch too much.
"""
from __future__ import annotations

import argparse
import json
import tempfile

import ostc
import ostc_cases as oc


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--case", choices=["air", "reacting", "multiblock"], default="air")
    p.add_argument("--dims", type=int, nargs=3, default=None, help="nodes in x, y, z (air / reacting)")
    p.add_argument("--steps", type=int, default=2)
    p.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    p.add_argument("--chem", choices=["explicit", "point_implicit"], default="explicit")
    p.add_argument("--device", type=int, default=0)
    a = p.parse_args()

    tmp = tempfile.mkdtemp(prefix=f"ostc_{a.case}_")
    if a.case == "multiblock":
        case = oc.multiblock_mixing_layer_3d(seed=0)
    elif a.case == "reacting":
        case = oc.reacting_mixing_layer_3d(*(a.dims or (384, 192, 96)), seed=0)
    else:
        case = oc.mixing_layer_3d(*(a.dims or (512, 256, 128)), seed=0)
    oc.write_case(case, tmp)
    s = ostc.Solver(tmp, device=a.device)
    s.set_precision(ostc.PREC_MIXED if a.precision == "mixed" else ostc.PREC_FP64)
    if a.case == "reacting":
        s.set_chem_mode(ostc.CHEM_POINT_IMPLICIT if a.chem == "point_implicit" else ostc.CHEM_EXPLICIT)
    if a.case == "multiblock":
        for b, blk in enumerate(case.blocks):
            s.set_state(blk.bv, block=b)
    else:
        s.set_state(case.bv, sv=getattr(case, "sv", None))
    ms = s.timed_steps(a.steps)
    print(json.dumps({"case": a.case, "nodes": s.total_nodes(), "steps": a.steps,
                      "ms_per_step": ms / a.steps, "error_flags": s.error_flags()}))
    flags = s.error_flags()
    s.close()
    raise SystemExit(1 if flags else 0)


if __name__ == "__main__":
    main()
