"""Generates the golden fixtures that pin the CPU oracle (and the CUDA path) to the reference solver.

Runs on a machine with a GPU: the reference (OpenSTC-MixingLayer) has no CPU implementation of this
path, so its own FP64 CUDA build - compiled from its sources by oracle/ref/build_ref.sh and driven by
oracle/ref/ref_harness.cu through the reference's Driver and RK3 - advances each seeded case, and the
interior conservative state it reaches is stored here with the case description.

    python tests/golden/make_golden.py [outdir]

Each fixture golden_<name>.npz holds cv (5 x mz x my x mx, float64, reference after `steps` steps),
t (physical time), steps, and the case-generator call; the initial state is regenerated from it
(ostc_cases, seeded) and its sum is stored as bv0_sum to detect drift of the generator.
"""
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "openstc-mixinglayer_b200" / "python"))
sys.path.insert(0, str(ROOT / "oracle"))

import ostc_cases as oc  # noqa: E402
import refcase  # noqa: E402

CASES = [
    # name, generator, kwargs, steps
    ("ml2d_weno5_ausm", "mixing_layer_2d", dict(mx=65, my=33, reconstruction=4, inviscid_scheme=3), 100),
    ("ml2d_weno7_hllc", "mixing_layer_2d", dict(mx=65, my=33, reconstruction=5, inviscid_scheme=4), 50),
    ("ml3d_weno7_hllc_farfield", "mixing_layer_3d",
     dict(mx=32, my=20, mz=16, reconstruction=5, inviscid_scheme=4), 20),
    ("ml3d_weno5_ausm_outflow", "mixing_layer_3d",
     dict(mx=32, my=20, mz=16, reconstruction=4, inviscid_scheme=3, ybc="outflow"), 20),
    # primitive reconstructions (inviscid_type 0 and 2) and AWENO with Lax-Friedrichs
    ("ml2d_muscl_roe", "mixing_layer_2d", dict(mx=65, my=33, reconstruction=2, inviscid_scheme=2), 100),
    ("ml2d_nnd_hllc", "mixing_layer_2d", dict(mx=65, my=33, reconstruction=3, inviscid_scheme=4), 100),
    ("ml2d_weno5_lf", "mixing_layer_2d", dict(mx=65, my=33, reconstruction=4, inviscid_scheme=1), 50),
    ("ml3d_first_ausm_outflow", "mixing_layer_3d",
     dict(mx=32, my=20, mz=16, reconstruction=1, inviscid_scheme=3, ybc="outflow"), 20),
    ("ml3d_muscl_lf_farfield", "mixing_layer_3d",
     dict(mx=32, my=20, mz=16, reconstruction=2, inviscid_scheme=1), 20),
    ("ml3d_nnd_roe_farfield", "mixing_layer_3d",
     dict(mx=32, my=20, mz=16, reconstruction=3, inviscid_scheme=2), 20),
    # 9-species H2/air mixtures: finite-rate (FR) and non-reacting (Mixture) models, flux-split WENO7
    ("rml3d_fr72", "reacting_mixing_layer_3d", dict(mx=32, my=20, mz=16, inviscid_scheme=72), 10),
    ("rml3d_mix71", "reacting_mixing_layer_3d", dict(mx=32, my=20, mz=16, inviscid_scheme=71, finite_rate=False), 10),
    ("rml2d_fr72", "reacting_mixing_layer_3d", dict(mx=48, my=24, mz=1, inviscid_scheme=72), 20),
    # multi-block chains joined by 1:1 interfaces (inner-face file)
    ("mb3d_awe7_hllc", "multiblock_mixing_layer_3d", dict(dims=[20, 17, 23], my=16, mz=10), 10),
    ("mb2d_awe5_ausm", "multiblock_mixing_layer_3d",
     dict(dims=[30, 21, 26, 18], my=24, mz=1, reconstruction=4, inviscid_scheme=3), 20),
]


def make_case(gen, kw):
    return getattr(oc, gen)(**kw)


def main(outdir: Path, only=None):
    outdir.mkdir(parents=True, exist_ok=True)
    for name, gen, kw, steps in CASES:
        if only and name not in only:
            continue
        case = make_case(gen, kw)
        cv, bv, t = refcase.run_reference(case, steps)[:3]
        meta = json.dumps({"generator": gen, "kwargs": kw})
        if hasattr(case, "blocks"):
            arrays = {f"cv_{b}": c for b, c in enumerate(cv)}
            np.savez_compressed(outdir / f"golden_{name}.npz", t=t, steps=steps, case=meta, n_block=len(cv),
                                bv0_sum=float(sum(np.sum(b.bv) for b in case.blocks)), **arrays)
            print(name, "t =", t, "blocks", len(cv), flush=True)
            continue
        np.savez_compressed(outdir / f"golden_{name}.npz", cv=cv, t=t, steps=steps, case=meta,
                            bv0_sum=float(np.sum(case.bv)))
        print(name, "t =", t, "rho range", float(bv[0].min()), float(bv[0].max()), flush=True)


if __name__ == "__main__":
    main(Path(sys.argv[1]) if len(sys.argv) > 1 else Path(__file__).resolve().parent, sys.argv[2:] or None)
