"""Generates the golden fixtures that pin the CPU oracle (and the CUDA path) to the reference solver.

Runs on a machine with a GPU: the reference (OpenSTC-MixingLayer) has no CPU implementation of this
path, so its own FP64 CUDA build - compiled from its sources by oracle/ref/build_ref.sh and driven by
oracle/ref/ref_harness.cu through the reference's Driver and RK3 - advances each seeded case, and the
interior conservative state it reaches is stored here with the case description.

    python tests/golden/make_golden.py [outdir] [case names...]

Each fixture golden_<name>.npz holds the case-generator call, steps, t (physical time) and the sum of
the regenerated initial state (bv0_sum, to detect drift of the generator), and either
  * cv (n_var x mz x my x mx, float64: the reference state after `steps` steps; cv_<b> per block), or,
    for the grids of the benchmark sizes (`sampled`), a summary that a test can compare node by node
    without storing the whole field: 16384 seeded node indices `idx` with the reference's cv there
    (`cv_s`), the per-variable error scales of the whole field (`smax`, `sl2`: max-abs and L2 norm,
    the momentum components sharing the momentum vector's, as ostc_cases.relative_errors scales them),
    and the k-plane and j-plane sums of cv and |cv| (`ksum`, `kabs`, `jsum`, `jabs`);
  * file_<name>: the bytes of files the reference wrote at the end of its run (its flowfield.plt,
    its statistics files coll_*.bin), for the cases that keep them.
"""
import json
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "openstc-mixinglayer_b200" / "python"))
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT / "tests"))

import ostc_cases as oc  # noqa: E402
import refcase  # noqa: E402
from golden_util import STAT_SETUP, STAT_SETUP_EXTRA  # noqa: E402

STAT_FILES = ["output/stat/coll_rey_1st.bin", "output/stat/coll_fav_1st.bin", "output/stat/coll_rey_2nd.bin",
              "output/stat/coll_fav_2nd.bin"]
PLT = ["output/flowfield.plt"]
EXTRA_FILES = ["output/stat/tke_budget.bin", "output/stat/species_velocity_correlation.bin",
               "output/stat/species_dissipation_rate.bin"]
# steady driver settings (no early stop on convergence: the fixture runs a fixed iteration count)
STEADY = dict(steady=1, implicit_method=0, dplur_inner_step=3, chem_src_method=0, convergence_criteria=1e-300)
# dual time stepping settings (its DPLUR needs implicit_method 1 for the reference to allocate the iterates,
# Field.cu:557-563)
DUAL = dict(steady=0, temporal_scheme=2, implicit_method=1, dplur_inner_step=2, inner_iteration=4,
            max_inner_iteration=8, iteration_adjust_step=2)

CASES = [
    # name, generator, kwargs, steps[, options: sampled / setup (extra setup.txt lines) / files (kept)]
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
    # the benchmark configurations at their stated sizes (or a 3-D grid of the same shape family):
    # the 2-D layer exactly (256 x 128 cells, node-coincident periodic x, 100 steps) ...
    ("c1_ml2d_256x128_weno5_ausm", "mixing_layer_2d", dict(mx=257, my=129), 100),
    # ... the 3-D air layer (WENO7-Z + HLLC, viscous, far-field y) at 1/64 of its nodes over 20 steps
    # and at its full 512 x 256 x 128 over 3 steps ...
    ("c2_ml3d_128x64x32_weno7_hllc", "mixing_layer_3d", dict(mx=128, my=64, mz=32), 20, dict(sampled=True)),
    ("c2_ml3d_512x256x128_weno7_hllc", "mixing_layer_3d", dict(), 3, dict(sampled=True)),
    # ... the reacting 9-species layer (flux-split WENO7, finite-rate chemistry) at 1/64 of its nodes
    ("c3_rml3d_96x48x24_fr72", "reacting_mixing_layer_3d", dict(mx=96, my=48, mz=24), 20, dict(sampled=True)),
    # ... and a twelve-block chain of uneven i extents
    ("c4_mb3d_12_blocks", "multiblock_mixing_layer_3d", dict(dims=None, my=18, mz=8), 10),
    # every block's three extents drawn; neighbours share the overlapping part of their x faces, the
    # rest of each x face is an outflow patch
    ("mb3d_uneven_axes", "multiblock_mixing_layer_3d", dict(nb=4, lo=8, hi=20, seed=3, uneven_axes=True), 10),
    # boundary faces beyond the mixing-layer set: no-slip walls, constant supersonic inflow, subsonic
    # inflow with back pressure (air), walls and inflow for the mixture
    ("ml3d_wall_isothermal", "mixing_layer_3d", dict(mx=32, my=24, mz=16, ybc="wall"), 10),
    ("ml3d_wall_adiabatic", "mixing_layer_3d", dict(mx=32, my=24, mz=16, ybc="wall", wall_thermal="adiabatic"), 10),
    ("ml2d_wall_isothermal_weno5", "mixing_layer_2d", dict(mx=65, my=33, ybc="wall"), 20),
    ("ml2d_wall_adiabatic_weno7", "mixing_layer_2d",
     dict(mx=65, my=33, reconstruction=5, inviscid_scheme=4, ybc="wall", wall_thermal="adiabatic"), 20),
    ("ml3d_inflow_outflow", "mixing_layer_3d", dict(mx=32, my=20, mz=12, ybc="outflow", xbc="inflow"), 10),
    # (the j = 0 face applies the reference state: the reference builds a subsonic inflow only after a
    # far-field or inflow face has set its reference values)
    ("ml3d_subsonic_backpressure", "mixing_layer_3d",
     dict(mx=32, my=20, mz=12, ybc="outflow", xbc="subsonic", ref_face=True), 10),
    ("rml3d_wall", "reacting_mixing_layer_3d", dict(mx=20, my=16, mz=10, ybc="wall"), 5),
    ("rml3d_inflow", "reacting_mixing_layer_3d", dict(mx=24, my=16, mz=10, xbc="inflow"), 5),
    # far-field (Riemann-invariant) faces of a mixture: fuel stream above, vitiated air below
    ("rml3d_farfield_fr72", "reacting_mixing_layer_3d", dict(mx=32, my=20, mz=16, ybc="farfield"), 10),
    ("rml3d_farfield_mix71", "reacting_mixing_layer_3d",
     dict(mx=32, my=20, mz=16, ybc="farfield", inviscid_scheme=71, finite_rate=False), 10),
    # mixtures on the primitive-reconstruction path (reconstruction<mixture> + AUSM+ / HLLC / Roe mixture
    # branches), reacting and frozen, 3-D and 2-D, one with far-field faces
    ("rml3d_muscl_ausm", "reacting_mixing_layer_3d", dict(mx=24, my=16, mz=10, inviscid_scheme=3), 5),
    ("rml3d_nnd_hllc", "reacting_mixing_layer_3d",
     dict(mx=24, my=16, mz=10, inviscid_scheme=4, reconstruction=3, finite_rate=False), 5),
    ("rml3d_first_roe", "reacting_mixing_layer_3d", dict(mx=24, my=16, mz=10, inviscid_scheme=2, reconstruction=1), 5),
    ("rml2d_muscl_roe", "reacting_mixing_layer_3d", dict(mx=40, my=26, mz=1, inviscid_scheme=2), 10),
    ("rml3d_farfield_nnd_ausm", "reacting_mixing_layer_3d",
     dict(mx=24, my=16, mz=10, ybc="farfield", inviscid_scheme=3, reconstruction=3), 5),
    # spatial mixing layers (problem_type 1, the reference's shipped layout): the two-stream inflow
    # profile, air and 9-species, 3-D and 2-D; with white noise on the inflow velocity (its generator
    # seeded from the clock the harness fixes), also on a constant inflow
    ("sml3d_air", "spatial_mixing_layer_3d", dict(mx=40, my=32, mz=8), 10),
    ("sml2d_air", "spatial_mixing_layer_3d", dict(mx=48, my=40, mz=1), 15),
    ("sml3d_species", "spatial_mixing_layer_3d", dict(mx=32, my=24, mz=6, species=True), 6),
    ("sml3d_air_noise", "spatial_mixing_layer_3d", dict(mx=40, my=32, mz=8, fluctuation_type=1), 10),
    ("sml2d_air_noise", "spatial_mixing_layer_3d", dict(mx=48, my=40, mz=1, fluctuation_type=1), 15),
    ("sml3d_species_noise", "spatial_mixing_layer_3d",
     dict(mx=32, my=24, mz=6, species=True, fluctuation_type=1, intensity=0.02), 6),
    # the digital filter's turbulent inflow (fluctuation_type 11), air and 9-species
    ("sml3d_air_df", "spatial_mixing_layer_3d", dict(mx=24, my=32, mz=56, fluctuation_type=11), 6),
    ("sml3d_species_df", "spatial_mixing_layer_3d", dict(mx=20, my=24, mz=56, species=True, fluctuation_type=11), 4),
    ("ml3d_inflow_noise", "mixing_layer_3d", dict(mx=32, my=20, mz=12, ybc="outflow", xbc="inflow", inflow_noise=0.01), 10),
    # the reference's steady driver (SteadySim.cuh): local time steps, explicit or DPLUR implicit
    # treatment (DPLUR.cuh), the chemical source explicit, point-implicit (EPI) or diagonal (DA).  No
    # wall case with DPLUR: the reference zeroes dq over the wall's ngg-padded range in an array with
    # one ghost layer (DPLUR.cu:22-40, Mesh.cpp:14-32, Field.cu:559-562), outside that array
    ("st_ml3d_explicit", "mixing_layer_3d", dict(mx=24, my=20, mz=12, ybc="outflow", steady=STEADY), 10),
    ("st_ml3d_dplur", "mixing_layer_3d", dict(mx=24, my=20, mz=12, steady=dict(STEADY, implicit_method=1)), 10),
    ("st_ml2d_dplur", "mixing_layer_2d", dict(mx=49, my=33, steady=dict(STEADY, implicit_method=1)), 15),
    ("st_rml3d_epi", "reacting_mixing_layer_3d", dict(mx=16, my=12, mz=8, steady=dict(STEADY, chem_src_method=1)), 5),
    ("st_rml3d_da", "reacting_mixing_layer_3d", dict(mx=16, my=12, mz=8, steady=dict(STEADY, chem_src_method=2)), 5),
    ("st_rml3d_dplur_epi", "reacting_mixing_layer_3d",
     dict(mx=16, my=12, mz=8, steady=dict(STEADY, implicit_method=1, chem_src_method=1)), 5),
    ("st_rml3d_dplur_explicit", "reacting_mixing_layer_3d",
     dict(mx=16, my=12, mz=8, steady=dict(STEADY, implicit_method=1, dplur_inner_step=2)), 5),
    ("st_rml3d_mix_dplur", "reacting_mixing_layer_3d",
     dict(mx=16, my=12, mz=8, finite_rate=False, steady=dict(STEADY, implicit_method=1)), 5),
    ("st_rml3d_muscl_ausm_dplur_epi", "reacting_mixing_layer_3d",
     dict(mx=16, my=12, mz=8, inviscid_scheme=3, steady=dict(STEADY, implicit_method=1, chem_src_method=1)), 5),
    # dual time stepping (DualTimeStepping.cuh, temporal_scheme 2): BDF2 physical steps of fixed dt, DPLUR
    # pseudo-time inner iterations whose count adapts every iteration_adjust_step-th step
    ("dt_ml3d", "mixing_layer_3d", dict(mx=24, my=20, mz=12, ybc="outflow", steady=dict(DUAL, dt=2e-7)), 6),
    ("dt_ml2d", "mixing_layer_2d", dict(mx=49, my=33, steady=dict(DUAL, dt=4e-7)), 6),
    ("dt_rml3d_epi", "reacting_mixing_layer_3d",
     dict(mx=16, my=12, mz=8, steady=dict(DUAL, dt=5e-8, chem_src_method=1)), 4),
    # the files the reference writes at the end of a run: flow field and statistics
    ("ml3d_stat_plt", "mixing_layer_3d", dict(mx=16, my=12, mz=8, ybc="outflow"), 6,
     dict(setup=STAT_SETUP, files=PLT + STAT_FILES)),
    ("rml3d_stat_plt", "reacting_mixing_layer_3d", dict(mx=12, my=10, mz=6), 5,
     dict(setup=STAT_SETUP, files=PLT + STAT_FILES)),
    ("ml2d_plt", "mixing_layer_2d", dict(mx=33, my=17, ybc="wall"), 5, dict(files=PLT)),
    # the additional collectors' files: the TKE budget (air 3-D and 2-D), and for three species of the
    # reacting layer their velocity correlation and dissipation rate
    ("ml3d_stat_extra", "mixing_layer_3d", dict(mx=16, my=12, mz=8, ybc="outflow"), 6,
     dict(setup=STAT_SETUP_EXTRA, files=STAT_FILES + EXTRA_FILES[:1])),
    ("ml2d_stat_extra", "mixing_layer_2d", dict(mx=33, my=17), 5,
     dict(setup=STAT_SETUP_EXTRA, files=STAT_FILES + EXTRA_FILES[:1])),
    ("rml3d_stat_extra", "reacting_mixing_layer_3d", dict(mx=12, my=10, mz=6), 5,
     dict(setup=STAT_SETUP_EXTRA, files=STAT_FILES + EXTRA_FILES)),
]

N_SAMPLE = 16384


def reference_dt_defined(nodes: int) -> bool:
    """Whether the reference's CFL minimum is defined for a block of this many nodes.  Its min_of_arr /
    block_reduce_min (TimeAdvanceFunc.cu:70-89, gxl_lib/MyAtomic.cuh:33-64) read the shared-memory slot
    of a warp that never wrote it when the last 128-thread block of a pass holds 32, 64 or 96 entries:
    the first pass over the nodes, and the second over the per-block minima (one per 128 nodes)."""
    first = nodes % 128
    second = -(-nodes // 128)
    return first not in (32, 64, 96) and second not in (32, 64, 96)


def c4_dims(nb=12, lo=12, hi=30, my=18, mz=8, seed=4):
    """Seeded uneven i extents of a twelve-block chain, each a block size the reference's dt is defined for."""
    rng = np.random.default_rng(seed)
    dims = []
    while len(dims) < nb:
        mx = int(rng.integers(lo, hi + 1))
        if reference_dt_defined(mx * my * mz):
            dims.append(mx)
    return dims


for _e in CASES:
    if _e[0] == "c4_mb3d_12_blocks":
        _e[2]["dims"] = c4_dims()


def make_case(gen, kw):
    return getattr(oc, gen)(**kw)


def scales(cv):
    """Per-variable (max-abs, L2) error scales as ostc_cases.relative_errors forms them."""
    mom = slice(1, 4)
    mom_max = float(np.max(np.sqrt(np.sum(cv[mom] ** 2, axis=0))))
    mom_l2 = float(np.linalg.norm(cv[mom]))
    smax, sl2 = [], []
    for l in range(cv.shape[0]):
        if 1 <= l <= 3:
            smax.append(mom_max)
            sl2.append(mom_l2)
        else:
            smax.append(float(np.max(np.abs(cv[l]))))
            sl2.append(float(np.linalg.norm(cv[l])))
    return np.array(smax), np.array(sl2)


def summarize(cv, seed=2024):
    nv = cv.shape[0]
    flat = cv.reshape(nv, -1)
    n = flat.shape[1]
    idx = np.sort(np.random.default_rng(seed).choice(n, size=min(N_SAMPLE, n), replace=False))
    smax, sl2 = scales(cv)
    return dict(idx=idx, cv_s=flat[:, idx].copy(), smax=smax, sl2=sl2, ksum=cv.sum(axis=(2, 3)),
                kabs=np.abs(cv).sum(axis=(2, 3)), jsum=cv.sum(axis=(1, 3)), jabs=np.abs(cv).sum(axis=(1, 3)))


def main(outdir: Path, only=None) -> int:
    outdir.mkdir(parents=True, exist_ok=True)
    failed = []
    for entry in CASES:
        name, gen, kw, steps = entry[:4]
        opts = entry[4] if len(entry) > 4 else {}
        if only and name not in only:
            continue
        case = make_case(gen, kw)
        sizes = [b.mx * b.my * b.mz for b in case.blocks] if hasattr(case, "blocks") else [case.nodes]
        if not all(reference_dt_defined(n) for n in sizes):
            # the reference's CFL minimum would read unwritten shared memory: no defined result to pin
            print(name, "SKIPPED: a block size for which the reference's dt is undefined", sizes, flush=True)
            failed.append(name)
            continue
        # inflow_seed: the clock the harness reported to the reference (its white-noise inflow seed)
        meta = json.dumps({"generator": gen, "kwargs": kw, "inflow_seed": refcase.REF_TIME})
        try:
            with tempfile.TemporaryDirectory(prefix="ostc_ref_") as wd:
                cv, bv, t = refcase.run_reference(case, steps, wd, setup_extra=opts.get("setup", ""))[:3]
                files = {}
                for rel in opts.get("files", []):
                    files["file_" + Path(rel).name] = np.frombuffer((Path(wd) / rel).read_bytes(), dtype=np.uint8)
        except (RuntimeError, OSError) as e:
            print(name, "FAILED:", e, flush=True)
            failed.append(name)
            continue
        common = dict(t=t, steps=steps, case=meta, **files)
        if hasattr(case, "blocks"):
            arrays = {f"cv_{b}": c for b, c in enumerate(cv)}
            np.savez_compressed(outdir / f"golden_{name}.npz", n_block=len(cv),
                                bv0_sum=float(sum(np.sum(b.bv) for b in case.blocks)), **common, **arrays)
            print(name, "t =", t, "blocks", len(cv), flush=True)
            continue
        if opts.get("sampled"):
            np.savez_compressed(outdir / f"golden_{name}.npz", sampled=True, bv0_sum=float(np.sum(case.bv)),
                                **common, **summarize(cv))
        else:
            np.savez_compressed(outdir / f"golden_{name}.npz", cv=cv, bv0_sum=float(np.sum(case.bv)), **common)
        print(name, "t =", t, "rho range", float(bv[0].min()), float(bv[0].max()), flush=True)
    return 1 if failed else 0


if __name__ == "__main__":
    sys.exit(main(Path(sys.argv[1]) if len(sys.argv) > 1 else Path(__file__).resolve().parent, sys.argv[2:] or None))
