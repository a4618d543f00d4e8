"""Times the reference's own FP64 CUDA build (oracle/_ref/ref_harness) on a mixing-layer workload.

TEST INFRASTRUCTURE: a measurement of the reference for comparison, never part of the product.  The
harness wall-clocks its RK3() call (cudaDeviceSynchronize on both sides), which includes the
reference's per-run fixed costs (its final flow-field write, first-launch overheads).  Two runs of
n1 and n2 steps are taken and the per-step time is the difference quotient, so those fixed costs
cancel:  ms/step = (t(n2) - t(n1)) / (n2 - n1).

Usage: python oracle/ref/time_reference.py [mx my mz] [--steps n1 n2] [--case reacting_mixing_layer_3d]
       python oracle/ref/time_reference.py --case multiblock_uneven   (the twelve-block chain whose extents
       are each drawn in [32, 256], seed 0: the reference's per-block launch loop, RK.cuh:112-174)
Prints one JSON line: grid, steps, per-run seconds, ms/step and cell-steps/s.
"""
from __future__ import annotations

import argparse
import json
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT / "openstc-mixinglayer_b200" / "python"))
sys.path.insert(0, str(ROOT / "oracle"))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("dims", nargs="*", type=int, default=[512, 256, 128])
    ap.add_argument("--steps", nargs=2, type=int, default=[4, 24])
    ap.add_argument("--case", default="mixing_layer_3d",
                    choices=["mixing_layer_3d", "reacting_mixing_layer_3d", "multiblock_uneven"])
    a = ap.parse_args()
    import ostc_cases as oc
    import refcase

    mx, my, mz = a.dims
    if a.case == "multiblock_uneven":
        case = oc.multiblock_mixing_layer_3d(nb=12, lo=32, hi=256, seed=0, uneven_axes=True)
        grid = [[b.mx, b.my, b.mz] for b in case.blocks]
    else:
        case = getattr(oc, a.case)(mx=mx, my=my, mz=mz)
        grid = [mx, my, mz]
    secs = []
    for n in a.steps:
        *_, s = refcase.run_reference(case, n, with_seconds=True)
        secs.append(s)
    n1, n2 = a.steps
    ms = (secs[1] - secs[0]) / (n2 - n1) * 1e3
    print(json.dumps({"impl": "reference FP64 CUDA build", "grid": grid, "steps": a.steps,
                      "rk3_seconds": secs, "ms_per_step": ms, "cell_steps_per_s": case.nodes / ms * 1e3,
                      "workload": a.case}))


if __name__ == "__main__":
    main()
