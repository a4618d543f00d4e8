#!/usr/bin/env python
"""Benchmark: cell-steps/s of the OpenSTC RHS + SSP-RK3 path on B200 (one JSON line on rank 0).

Workload (default): the 3-D temporal mixing layer, 512 x 256 x 128 grid nodes (16.8 M), calorically
perfect air, WENO7-Z characteristic interpolation (AWENO7) + HLLC, 2nd-order viscous terms
(Sutherland, Pr = 0.72), Mc = 0.7, periodic x and z, far-field y, SSP-RK3 at CFL 0.5, seeded
synthetic initial data.  A "step" is one full SSP-RK3 step of the whole grid (3 stages: CFL dt,
inviscid + viscous RHS, update, boundaries).  One cell-step = one interior node advanced one step.

  value    plain FP64 path, inputs resident in HBM, CUDA events on the library stream
  mixed    FP32 flux/viscous arithmetic with FP64 state, same workload; its rel-L2 distance to the
           FP64 path after warmup+steps steps is stated
  e2e      the same metric through the C ABI with host buffers (ostc_run_states): each step copies
           its primitive input state from pinned host memory in, advances one step and copies the
           state back; the copies of neighbouring steps run on two copy streams under the compute
  roofline dominant kernel (by device time), algorithmic bytes per launch / average launch time
  cpu_baseline  the serial C restatement of the same path (oracle/) on a sub-grid sample
  reacting the 9-species H2/air mixing layer, 384 x 192 x 96, flux-split characteristic WENO7,
           finite-rate chemistry (explicit, and the point-implicit batched 9x9 LU extension), FP64
  multiblock  12 blocks whose three extents are each drawn uniform in [32, 256] (seeded), chained
           along x by 1:1 interfaces over the overlap of neighbouring faces, 39 M nodes, AWENO7 +
           HLLC, FP64; every block's sweeps, update, boundary faces and interface exchange are one
           CUDA graph per step, timed beside the per-block launch loop (block_loop)
  adjoint  192 x 96 x 48 reacting layer: one right-hand-side VJP against one right-hand side, and the
           momentum-thickness gradient after 200 steps w.r.t. 8 v' mode amplitudes by the
           checkpointed trajectory adjoint, with central differences for two of them
  statistics  one single-point statistics collection (Reynolds / Favre moments, every option on)
           over the default workload and its ghost layer: device time and HBM fraction

--only air|reacting|multiblock runs one workload for a few steps and prints its device time per step
(--only adjoint: that many right-hand-side VJPs of the 9-species layer, 192 x 96 x 48 unless --dims;
--only adjoint_air: of the air layer with outflow y faces, 512 x 256 x 128 unless --dims)
(the short command to put under a profiler, where the whole benchmark would launch too much); it
takes --dims, --steps, --precision and --chem.

--impl reference times that C restatement on all host cores (independent sub-grid replicas, one
process per core): the reference's own implementation of this path exists only as CUDA device code.
Multi-GPU (torchrun): the path is replicated, one independent case per GPU ("scaling": "weak").
"""
from __future__ import annotations

import argparse
import json
import math
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "openstc-mixinglayer_b200" / "python"))
sys.path.insert(0, str(ROOT / "openstc-mixinglayer_b200"))

METRIC = "cell-steps/s on 1 B200: mixed vs FP64 RHS at stated rel-L2 error; % of HBM peak"
UNIT = "cell-steps/s"
FALLBACK_HBM_GBS = 6650.0
# Compulsory bytes per interior node of each kernel family (FP64 loads/stores the kernel must make):
#   flux_x      cv(5) + rho,u,v,w,p(5) + metric row(3) + jac(1) read, dq(5) written          = 19 x 8
#   flux_y/z    the same reads, dq(5) read-modify-written                                     = 24 x 8
#   visc_update u,v,w,T(4) + mu + metric(9) + jac + dq(5) + cv_in(5) + q^n(5) read,
#               cv(5) + bv(6) + mu written                                                    = 42 x 8
#   cfl_dt      metric(9) + rho,u,v,w,T(5) + mu read                                          = 15 x 8
ALGO_BYTES_PER_NODE = {"flux_x": 152, "flux_y": 192, "flux_z": 192, "visc_update": 336, "cfl_dt": 120}
# DRAM bytes per node measured by one ncu capture of the kernel (dram__bytes_read.sum +
# dram__bytes_write.sum over the nodes of the launch, 256x128x64 case of the same workload; traffic
# grows with the node count, so a full-size launch moves this figure times its nodes).  The y/z
# sweeps have several designs picked by the library's autotuner; at 512x256x128 it keeps 16-lane
# tiles, and the capture is of the 16 x 16 x 1 tile (the column march moved 209.8, the 32x4x4 tile
# 194-203 B per node).
MEASURED_TRAFFIC_PER_NODE = {"flux_y": 214.5, "flux_z": 214.5}
# FP64 operations per face of the y/z sweep (AWENO7 + HLLC, central correction), from the same
# capture's instruction counters: 2 x DFMA + DMUL + DADD thread-instructions over the launch's faces.
# Against the FP64 FMA peak of the part (64 DFMA per cycle per SM) this is the roof the sweeps run
# into; the HBM fraction above stays far from 1 because the sweeps are arithmetic bound.
FP64_FLOP_PER_FACE = 3275
FP64_DFMA_PER_CYCLE_PER_SM = 64
# Whole fused stage (three state passes + metric): 8 (3 n_var + 10) bytes per cell-stage, n_var = 5
STAGE_BYTES = 8 * (3 * 5 + 10)
# steps after which the reacting layer's mixed-precision state is compared with the FP64 one
REACT_ERR_STEPS = 100


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--dims", type=int, nargs=3, default=[512, 256, 128])
    p.add_argument("--e2e-steps", type=int, default=6)
    p.add_argument("--no-mixed", action="store_true")
    p.add_argument("--cpu-sample", type=int, nargs=3, default=[96, 64, 48])
    p.add_argument("--cpu-steps", type=int, default=3)
    p.add_argument("--no-extra", action="store_true",
                   help="skip the reacting (9-species) and uneven multi-block workloads")
    p.add_argument("--only", choices=["air", "reacting", "multiblock", "adjoint", "adjoint_air"], default=None,
                   help="run one workload for --steps steps and print its device time per step")
    p.add_argument("--precision", choices=["fp64", "mixed"], default="fp64", help="with --only")
    p.add_argument("--chem", choices=["explicit", "point_implicit"], default="explicit", help="with --only")
    a = p.parse_args()
    a.dims_given = "--dims" in sys.argv
    return a


def run_only(args):
    """One workload for args.steps steps (no warm-up, no extras): the command profiled in profiles/."""
    import ostc
    import ostc_cases as oc

    tmp = tempfile.mkdtemp(prefix=f"ostc_{args.only}_")
    if args.only in ("adjoint", "adjoint_air"):
        return run_only_vjp(args, tmp)
    if args.only == "multiblock":
        case = oc.multiblock_mixing_layer_3d(seed=0, uneven_axes=True)
    elif args.only == "reacting":
        case = oc.reacting_mixing_layer_3d(*(args.dims if args.dims_given else (384, 192, 96)), seed=0)
    else:
        case = oc.mixing_layer_3d(*args.dims, seed=0)
    oc.write_case(case, tmp)
    s = ostc.Solver(tmp)
    s.set_precision(ostc.PREC_MIXED if args.precision == "mixed" else ostc.PREC_FP64)
    if args.only == "reacting":
        s.set_chem_mode(ostc.CHEM_POINT_IMPLICIT if args.chem == "point_implicit" else ostc.CHEM_EXPLICIT)
    if args.only == "multiblock":
        for b, blk in enumerate(case.blocks):
            s.set_state(blk.bv, block=b)
    else:
        s.set_state(case.bv, sv=getattr(case, "sv", None))
    ms = s.timed_steps(args.steps)
    flags = s.error_flags()
    print(json.dumps({"only": args.only, "nodes": s.total_nodes(), "steps": args.steps, "precision": args.precision,
                      "ms_per_step": ms / args.steps, "error_flags": flags}))
    s.close()
    raise SystemExit(1 if flags else 0)


def run_only_vjp(args, tmp):
    """args.steps right-hand-side VJPs (all terms) of the reacting or the air layer, device-resident
    buffers; the time of one right-hand side beside it."""
    import ctypes
    import time

    import ostc
    import ostc_cases as oc
    import torch

    if args.only == "adjoint_air":
        case = oc.mixing_layer_3d(*args.dims, seed=0, ybc="outflow")
    else:
        case = oc.reacting_mixing_layer_3d(*(args.dims if args.dims_given else (192, 96, 48)), seed=0)
    oc.write_case(case, tmp)
    s = ostc.Solver(tmp)
    s.set_state(case.bv, sv=getattr(case, "sv", None))
    shape = s.get_state()[0].shape
    dev = torch.device("cuda", 0)
    wb = torch.randn(shape, dtype=torch.float64, device=dev, generator=torch.Generator(dev).manual_seed(0))
    gb = torch.empty_like(wb)
    vjp = lambda: s.lib.ostc_rhs_vjp(s.h, 0, 7, ctypes.c_void_p(wb.data_ptr()), ctypes.c_void_p(gb.data_ptr()), 1)
    rhs = lambda: s.lib.ostc_rhs(s.h, 0, 7, ctypes.c_void_p(gb.data_ptr()), 1)
    times = {}
    for name, call in (("rhs", rhs), ("vjp", vjp)):
        assert call() == 0  # first call: scratch allocation, autotuning
        torch.cuda.synchronize(dev)
        t = time.perf_counter()  # the calls synchronise the library stream
        for _ in range(args.steps):
            assert call() == 0
        times[name] = (time.perf_counter() - t) * 1e3 / args.steps
    flags = s.error_flags()
    print(json.dumps({"only": args.only, "nodes": s.total_nodes(), "vjps": args.steps, "ms_per_rhs": times["rhs"],
                      "ms_per_vjp": times["vjp"], "vjp_over_rhs": times["vjp"] / times["rhs"],
                      "error_flags": flags}))
    s.close()
    raise SystemExit(1 if flags else 0)


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def measured_peaks():
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        d = json.loads(f.read_text())
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def config_dict(args):
    mx, my, mz = args.dims
    return {"workload": f"3-D temporal mixing layer {mx}x{my}x{mz} nodes, air, AWENO7 (WENO7-Z char.) + HLLC, "
                        f"viscous (Sutherland, Pr 0.72), Mc 0.7, periodic x/z, far-field y, SSP-RK3 CFL 0.5",
            "grid": [mx, my, mz], "n_var": 5, "nodes": mx * my * mz,
            "l2_policy": "inputs larger than L2 (state ~7 GB >> 126 MB L2); no flush needed",
            "parallelism": "replicas" if args.gpus > 1 else "single-gpu"}


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.index), "-lms", "200"], stdout=open(self.path, "w"),
                                         stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = [r.split(",") for r in Path(self.path).read_text().strip().splitlines() if r.strip()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        sm, smax, reasons = [], [], set()
        for r in rows:
            r = [x.strip() for x in r]
            try:
                sm.append(float(r[1]))
                smax.append(float(r[2]))
            except (ValueError, IndexError):
                continue
            for n, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------------------- CPU (oracle) legs

def _cpu_worker(dims, warm, steps, barrier, q):
    sys.path.insert(0, str(ROOT / "openstc-mixinglayer_b200" / "python"))
    sys.path.insert(0, str(ROOT / "oracle"))
    import ostc_cases as oc
    from oracle import Oracle
    case = oc.mixing_layer_3d(mx=dims[0], my=dims[1], mz=dims[2])
    o = Oracle(case)
    o.set_state(case.bv)
    if warm:
        o.step(warm)
    if barrier is not None:
        barrier.wait()
    t0 = time.time()
    o.step(steps)
    t1 = time.time()
    q.put((t0, t1, case.nodes * steps))


def cpu_run(dims, warm, steps, procs):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    barrier = ctx.Barrier(procs) if procs > 1 else None
    ps = [ctx.Process(target=_cpu_worker, args=(dims, warm, steps, barrier, q)) for _ in range(procs)]
    for p in ps:
        p.start()
    res = [q.get() for _ in ps]
    for p in ps:
        p.join()
    t0 = min(r[0] for r in res)
    t1 = max(r[1] for r in res)
    work = sum(r[2] for r in res)
    return work / (t1 - t0), t1 - t0


def ensure_oracle_built():
    subprocess.run(["make", "-C", str(ROOT / "oracle")], check=True, capture_output=True)


def run_reference(args):
    world, rank, _ = dist_env()
    if rank != 0:
        return
    ensure_oracle_built()
    procs = os.cpu_count() or 1
    dims = [64, 48, 32]
    value, wall = cpu_run(dims, args.warmup, args.steps, procs)
    sample = (f"{procs} independent {dims[0]}x{dims[1]}x{dims[2]} sub-grids of the workload (same scheme and "
              f"boundaries), one process per host core, {args.steps} timed steps after {args.warmup} warm-up")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": wall / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config_dict(args),
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": procs, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------- GPU leg

def reduce_max(x: float, dist, device) -> float:
    """Max over ranks of a per-rank device time (every rank calls it; identity without a group)."""
    if dist is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world: int, nodes_per_rank: int, steps: int, ms_max: float) -> float:
    """Cell-steps/s of the whole job: every rank advances its own replica of nodes_per_rank nodes by
    `steps` steps; the job takes as long as its slowest rank."""
    return world * nodes_per_rank * steps / (ms_max / 1e3)


def run_ours(args):
    world, rank, local = dist_env()
    import torch

    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        torch.cuda.set_device(local)
        dist_mod.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
        dist = dist_mod

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    def allmax(x):
        return reduce_max(x, dist, "cuda")

    import ostc
    import ostc_cases as oc
    import build as libbuild

    if rank == 0:
        libbuild.build()
    barrier()
    mx, my, mz = args.dims
    case = oc.mixing_layer_3d(mx=mx, my=my, mz=mz, seed=rank)
    tmp = tempfile.mkdtemp(prefix=f"ostc_bench_{rank}_")
    oc.write_case(case, tmp)
    hbm, peak_kind = measured_peaks()
    K, W = args.steps, args.warmup

    # ---- plain FP64, resident in HBM
    s = ostc.Solver(tmp, device=local)
    s.set_state(case.bv)
    s.step(W)
    barrier()
    sampler = ClockSampler(local)
    sampler.start()
    ms = s.timed_steps(K)
    clocks = sampler.stop()
    barrier()
    ms_max = allmax(ms)
    nodes = s.total_nodes()
    value = whole_job_rate(world, nodes, K, ms_max)
    launches_per_step = s.step_kernel_count()
    cv64, _ = s.get_state()
    flags = s.error_flags()

    # ---- mixed precision: same start, same step count
    mixed = None
    if not args.no_mixed:
        sm_ = ostc.Solver(tmp, device=local)
        sm_.set_precision(ostc.PREC_MIXED)
        sm_.set_state(case.bv)
        sm_.step(W)
        barrier()
        ms_m = allmax(sm_.timed_steps(K))
        cvm, _ = sm_.get_state()
        err = oc.relative_errors(cvm, cv64)
        l2 = math.sqrt(sum(e[1] ** 2 for e in err) / len(err))
        mixed = {"value": world * nodes * K / (ms_m / 1e3), "ms_per_step": ms_m / K,
                 "speedup_vs_fp64": ms_max / ms_m, "dtype": "f32 flux / f64 state",
                 "rel_l2_vs_fp64_per_var": [e[1] for e in err], "rel_l2_vs_fp64_rms": l2,
                 "rel_max_vs_fp64_per_var": [e[0] for e in err], "after_steps": W + K,
                 "flags": sm_.error_flags()}
        prof_m = sm_.profile(1)
        mixed["kernels_ms_per_step"] = {k: v[1] for k, v in prof_m.items()}
        sm_.close()

    # ---- per-kernel device times (CUDA events on the launching stream) for the roofline
    prof = s.profile(2)
    fam = {k: v for k, v in prof.items() if k in ALGO_BYTES_PER_NODE}
    dom = max(fam, key=lambda k: fam[k][1])
    n_launch, tot_ms = fam[dom]
    avg_ms = tot_ms / n_launch
    algo = ALGO_BYTES_PER_NODE[dom] * nodes
    achieved = algo / (avg_ms / 1e3) / 1e9
    traffic = None
    if dom in MEASURED_TRAFFIC_PER_NODE:
        traffic = MEASURED_TRAFFIC_PER_NODE[dom] * nodes
    step_ms = ms_max / K
    fp64_roof = None
    if dom in ("flux_y", "flux_z"):
        mhz = float(clocks.get("sm_mhz") or 1965.0) if isinstance(clocks, dict) else 1965.0
        n_sm = torch.cuda.get_device_properties(local).multi_processor_count
        peak_t = 2 * FP64_DFMA_PER_CYCLE_PER_SM * n_sm * mhz * 1e6 / 1e12
        ach_t = FP64_FLOP_PER_FACE * nodes / (avg_ms / 1e3) / 1e12
        fp64_roof = {"flop_per_face": FP64_FLOP_PER_FACE, "achieved_tflops": ach_t, "peak_tflops": peak_t,
                     "frac": ach_t / peak_t, "peak": f"{2 * FP64_DFMA_PER_CYCLE_PER_SM} FP64 FLOP per cycle per SM x "
                                                   f"{n_sm} SMs at the sampled {mhz:.0f} MHz"}
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "traffic": traffic, "algorithmic_bytes_per_launch": algo,
                "avg_launch_ms": avg_ms, "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                "note": "flux kernels are FP64-ALU bound (characteristic WENO7 + HLLC, 3.3 kFLOP per face); the "
                        "HBM fraction is reported as the contract asks, the FP64 fraction in fp64",
                "fp64": fp64_roof,
                "whole_step": {"achieved": value / world * 3 * STAGE_BYTES / 1e9,
                               "frac": value / world * 3 * STAGE_BYTES / 1e9 / hbm,
                               "bytes_per_cell_step": 3 * STAGE_BYTES},
                "kernels_ms_per_step": {k: v[1] / 2 for k, v in prof.items()}}

    # ---- single-point statistics (SinglePointStat): one collection over the block and its ghost layer,
    # every optional variable on, after the timed region; HBM bound (reads the 6 primitive planes,
    # read-modify-writes every accumulator plane once)
    s.stat_enable(0, ostc.STAT_REY_U | ostc.STAT_REY_V | ostc.STAT_REY_W | ostc.STAT_REY_T | ostc.STAT_RHO_P)
    sprof = s.profile(2)
    n_stat = s.stat_info()[0]
    points = (mx + 2) * (my + 2) * (mz + 2)
    st_ms = sprof["statistics"][1] / sprof["statistics"][0]
    st_bytes = (6 + 2 * sum(n_stat)) * 8 * points
    stat_line = {"ms_per_collection": st_ms, "bytes_per_point": st_bytes // points, "points": points,
                  "achieved_gbs": st_bytes / (st_ms / 1e3) / 1e9, "frac": st_bytes / (st_ms / 1e3) / 1e9 / hbm,
                  "n_var": n_stat, "share_of_step": st_ms / (ms_max / K)}
    s.stat_disable()

    # ---- end to end through the C ABI with host buffers
    e2e = None
    if args.e2e_steps > 0:
        import torch as _t
        hin = _t.empty((6,) + s.shape(), dtype=_t.float64, pin_memory=True)
        hin.copy_(_t.from_numpy(case.bv))
        hout = _t.empty((6,) + s.shape(), dtype=_t.float64, pin_memory=True)
        se = ostc.Solver(tmp, device=local)
        # ostc_run_states: every step takes its input state from pinned host memory and returns its
        # result there; the copies of neighbouring steps overlap the computation on copy streams
        se.run_states_ptr([hin.data_ptr()], [hout.data_ptr()], 1)  # allocations, graph capture
        barrier()
        t0 = time.perf_counter()
        se.run_states_ptr([hin.data_ptr()] * args.e2e_steps, [hout.data_ptr()] * args.e2e_steps, 1)
        t1 = time.perf_counter()
        barrier()
        el = allmax(t1 - t0)
        e2e = {"value": world * nodes * args.e2e_steps / el, "unit": UNIT,
               "h2d_bytes_per_step": int(hin.numel() * 8), "d2h_bytes_per_step": int(hout.numel() * 8),
               "steps": args.e2e_steps, "ms_per_step": el / args.e2e_steps * 1e3}
        se.close()
    s.close()

    extra = {}
    if not args.no_extra:
        extra = run_extra(args, local, barrier, allmax, world)

    cpu = None
    if rank == 0 and world == 1:
        ensure_oracle_built()
        cd = args.cpu_sample
        cval, cwall = cpu_run(cd, 0, args.cpu_steps, 1)
        cpu = {"value": cval, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": f"serial C restatement (oracle/) on a {cd[0]}x{cd[1]}x{cd[2]} sub-grid of the workload, "
                         f"{args.cpu_steps} steps ({cwall:.1f} s)"}

    if rank == 0:
        # compact figures first, so that a truncated copy of the line still carries them
        summary = {"mixed_speedup": mixed and mixed["speedup_vs_fp64"],
                   "mixed_rel_l2_rms": mixed and mixed["rel_l2_vs_fp64_rms"]}
        if extra:
            em = extra["reacting"]["explicit_mixed"]
            summary["reacting_mixed_speedup"] = em["speedup_vs_fp64"]
            summary["reacting_mixed_rel_l2_max"] = max(em["rel_l2_vs_fp64"].values())
            summary["adjoint_max_rel_diff"] = extra["adjoint"]["theta"]["max_rel_diff"]
            summary["adjoint_fd_spread"] = extra["adjoint"]["theta"]["max_fd_spread"]
            summary["multiblock_ms_per_step"] = extra["multiblock"]["ms_per_step"]
            summary["multiblock_speedup_vs_block_loop"] = extra["multiblock"]["speedup_vs_block_loop"]
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
                "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                **summary,
                "dtype": "f64", "data": "synthetic (seeded tanh shear layer + white noise; no dataset)",
                "config": config_dict(args), "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
                "statistics": stat_line,
                "mixed": mixed, "clocks": clocks, "gpu_launches": launches_per_step * K,
                "error_flags": flags, **extra}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_extra(args, local, barrier, allmax, world):
    """The reacting (C3-shaped) and multi-block (C4-shaped) workloads: device-timed cell-steps/s, the
    per-kernel split, and their settings.  Warm-up 2 steps, 5 timed steps each."""
    import ostc
    import ostc_cases as oc

    out = {}
    # reacting 9-species H2/air
    rc = oc.reacting_mixing_layer_3d(mx=384, my=192, mz=96, seed=0)
    tmp = tempfile.mkdtemp(prefix="ostc_bench_react_")
    oc.write_case(rc, tmp)
    react = {"workload": "reacting H2/air mixing layer 384x192x96, 9 species / 19 reactions, WENO7-Z "
                         "characteristic flux splitting (inviscid_scheme 72), mixture-averaged transport, FP64",
             "nodes": rc.nodes}
    ref_cv = None
    for mode, prec, key in ((ostc.CHEM_EXPLICIT, ostc.PREC_FP64, "explicit"),
                            (ostc.CHEM_POINT_IMPLICIT, ostc.PREC_FP64, "point_implicit"),
                            (ostc.CHEM_EXPLICIT, ostc.PREC_MIXED, "explicit_mixed")):
        s = ostc.Solver(tmp, device=local)
        s.set_chem_mode(mode)
        s.set_precision(prec)
        s.set_state(rc.bv, sv=rc.sv)
        s.step(2)
        barrier()
        ms = allmax(s.timed_steps(5))
        prof = s.profile(1)
        react[key] = {"value": world * rc.nodes * 5 / (ms / 1e3), "ms_per_step": ms / 5,
                      "kernels_ms_per_step": {k: v[1] for k, v in prof.items()}, "flags": s.error_flags()}
        if key != "point_implicit":
            # on to 100 steps (2 warm-up + 5 timed + 1 profiled + 92) for the error of the mixed mode
            s.step(REACT_ERR_STEPS - 8)
        if key == "explicit":
            ref_cv = s.get_state()[0]
        elif key == "explicit_mixed":
            # same 100 steps from the same state as the FP64 explicit run: error of the mixed mode
            cv = s.get_state()[0]
            names = ["rho", "rho_u", "rho_v", "rho_w", "rho_E"] + [f"rho_Y_{n}" for n in rc.mixture["tables"].names]
            react[key]["dtype"] = "f32 split fluxes / viscous fluxes / transport, f64 state / Newton / chemistry"
            # relative L2 per conserved variable; the momentum components against the momentum magnitude
            err = oc.relative_errors(cv, ref_cv)
            react[key]["rel_l2_vs_fp64"] = {names[l]: err[l][1] for l in range(cv.shape[0])}
            react[key]["rel_max_vs_fp64"] = {names[l]: err[l][0] for l in range(cv.shape[0])}
            react[key]["speedup_vs_fp64"] = react["explicit"]["ms_per_step"] / react[key]["ms_per_step"]
            react[key]["after_steps"] = REACT_ERR_STEPS
            react[key]["flags_after"] = s.error_flags()
        s.close()
    react["value"] = react["explicit"]["value"]
    out["reacting"] = react
    # uneven multi-block chain: every block's three extents drawn uniform in [32, 256]
    mc = oc.multiblock_mixing_layer_3d(nb=12, lo=32, hi=256, seed=0, uneven_axes=True)
    tmp = tempfile.mkdtemp(prefix="ostc_bench_mb_")
    oc.write_case(mc, tmp)
    mb = {"workload": f"{len(mc.blocks)} blocks, extents {[(b.mx, b.my, b.mz) for b in mc.blocks]}, chained "
                      "along x by 1:1 interfaces over the overlap of neighbouring faces, AWENO7 + HLLC, FP64",
          "nodes": mc.nodes}
    for mode, key in ((ostc.LAUNCH_GRAPH, "graph"), (ostc.LAUNCH_BLOCK_LOOP, "block_loop")):
        s = ostc.Solver(tmp, device=local)
        s.set_launch_mode(mode)
        for b, blk in enumerate(mc.blocks):
            s.set_state(blk.bv, block=b)
        s.step(2)
        barrier()
        ms = allmax(s.timed_steps(5))
        if key == "graph":
            prof = s.profile(1)
            mb.update({"value": world * mc.nodes * 5 / (ms / 1e3), "ms_per_step": ms / 5,
                       "kernels_per_step": s.step_kernel_count(),
                       "kernels_ms_per_step": {k: v[1] for k, v in prof.items()}, "flags": s.error_flags()})
        else:
            # the reference's launch structure: every kernel launched from the host, block after block
            mb["block_loop"] = {"value": world * mc.nodes * 5 / (ms / 1e3), "ms_per_step": ms / 5,
                                "flags": s.error_flags()}
        s.close()
    mb["speedup_vs_block_loop"] = mb["block_loop"]["ms_per_step"] / mb["ms_per_step"]
    out["multiblock"] = mb
    out["adjoint"] = run_adjoint(local)
    return out


def run_adjoint(local, n_steps=200, every=20):
    """The sensitivity workload of the adjoint (192 x 96 x 48 reacting layer, 9 species, FP64):
    device time of one right-hand-side VJP against one right-hand side, and the gradient of the
    momentum thickness after 200 steps w.r.t. 8 seeded v' mode amplitudes by one checkpointed
    trajectory adjoint (every 20 steps), checked for all eight modes against Richardson-combined central
    differences (steps 1e-5 and 2e-5).  dt fixed at the CFL dt of the initial state."""
    import ctypes
    import time

    import ostc
    import ostc_cases as oc
    import torch

    base = oc.reacting_mixing_layer_3d(mx=192, my=96, mz=48, seed=0)
    shapes = oc.mode_shapes(base)
    a0 = np.full(8, 1.0 / 8)
    c0 = oc.add_modes(base, a0, shapes)
    tmp = tempfile.mkdtemp(prefix="ostc_bench_adj_")
    oc.write_case(c0, tmp)
    s = ostc.Solver(tmp, device=local)
    s.set_state(c0.bv, sv=c0.sv)
    dt = s.step(1)
    s.close()
    c0.scheme["fixed_time_step"], c0.scheme["dt"] = 1, dt
    oc.write_case(c0, tmp)
    s = ostc.Solver(tmp, device=local)
    s.set_state(c0.bv, sv=c0.sv)
    cv0, _ = s.get_state()
    nv = cv0.shape[0]
    # one RHS against one RHS VJP, device buffers (the calls synchronise the library stream)
    dev = torch.device("cuda", local)
    dq = torch.empty(cv0.shape, dtype=torch.float64, device=dev)
    wb = torch.randn(cv0.shape, dtype=torch.float64, device=dev, generator=torch.Generator(dev).manual_seed(0))
    gb = torch.empty_like(dq)
    lib, h = s.lib, s.h
    times = {}
    for name, call in (("rhs", lambda: lib.ostc_rhs(h, 0, 7, ctypes.c_void_p(dq.data_ptr()), 1)),
                       ("rhs_vjp", lambda: lib.ostc_rhs_vjp(h, 0, 7, ctypes.c_void_p(wb.data_ptr()),
                                                            ctypes.c_void_p(gb.data_ptr()), 1))):
        assert call() == 0
        torch.cuda.synchronize(dev)
        t = time.perf_counter()
        for _ in range(5):
            assert call() == 0
        times[name] = (time.perf_counter() - t) / 5 * 1e3
    # momentum-thickness gradient
    du, dy = c0.extra["du"], c0.extra["h"]
    rho0 = float(cv0[0].mean())

    def theta(a):
        c = oc.add_modes(base, a, shapes)
        s.set_state(c.bv, sv=c.sv)
        s.step(n_steps)
        return oc.momentum_thickness(s.get_state()[0], du, rho0, dy)

    t = time.perf_counter()
    th, g_n = theta(a0)
    t_fwd = time.perf_counter() - t
    s.set_state(c0.bv, sv=c0.sv)
    t = time.perf_counter()
    lam0 = s.adjoint_steps(n_steps, g_n, every=every)
    t_adj = time.perf_counter() - t
    grad = [float(np.sum(lam0 * dm)) for dm in oc.dcv_dmodes(cv0, shapes)]
    # every mode by central differences at two step sizes, h and 2h, Richardson-combined; the gap
    # between the two plain differences shows how far the differences themselves resolve the gradient
    # (the Newton iterate's count and the |U| kink of the split fluxes make the 200-step map only
    # piecewise smooth)
    fd, spread = {}, {}
    hstep = 1e-5
    for m in range(8):
        e = np.zeros(8)
        e[m] = 1.0
        d1 = (theta(a0 + hstep * e)[0] - theta(a0 - hstep * e)[0]) / (2 * hstep)
        d2 = (theta(a0 + 2 * hstep * e)[0] - theta(a0 - 2 * hstep * e)[0]) / (4 * hstep)
        fd[m] = (4 * d1 - d2) / 3
        spread[m] = abs(d1 - d2)
    s.close()
    gmax = max(abs(g) for g in grad)
    return {"workload": "reacting H2/air mixing layer 192x96x48, 9 species, WENO7-Z flux splitting (72), FP64, "
                        f"fixed dt {dt:.3e}",
            "nodes": base.nodes, "rhs_ms": times["rhs"], "rhs_vjp_ms": times["rhs_vjp"],
            "vjp_over_rhs": times["rhs_vjp"] / times["rhs"],
            "theta": {"steps": n_steps, "checkpoint_every": every, "theta": th, "forward_s": t_fwd,
                      "adjoint_s": t_adj, "adjoint_over_forward": t_adj / t_fwd,
                      "dtheta_da": grad,
                      "central_difference_richardson_h1e-5_2e-5": {f"a{m}": fd[m] for m in fd},
                      "rel_diff": {f"a{m}": abs(fd[m] - grad[m]) / gmax for m in fd},
                      "fd_spread_h_vs_2h": {f"a{m}": spread[m] / gmax for m in fd},
                      "max_rel_diff": max(abs(fd[m] - grad[m]) for m in fd) / gmax,
                      "max_fd_spread": max(spread.values()) / gmax},
            "timing": "host wall clock around synchronising library calls (device-resident buffers)"}


def main():
    args = parse()
    world, _, _ = dist_env()
    if world > 1:
        args.gpus = world
    if args.only:
        run_only(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
