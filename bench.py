"""Benchmark of the B200 compressible-Euler step (one JSON line on rank 0).

Workload: the 3-D spherical explosion on [0,1]^3 with 256^3 cells (γ = 1.4,
ρ = 1, p = 1 for r < 0.3, ρ = 0.125, p = 0.1 outside, seeded ±1 % density
noise, transmissive boundaries), WCNS WENO5-Z + HLLC + positivity limiter +
SSP-RK3, CFL 0.5, each step's dt from the CFL reduction. One "step" is one
SSP-RK3 step of the whole grid; the metric is cell-updates/s (interior cells ×
steps / device time).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--precision f64|mixed]
  python bench.py --impl reference ...   # the reference CPU solver (C++ restatement) on host cores

Multi-GPU (torchrun): the path is one GPU per problem, so N ranks run N
independent replicas of the workload (weak scaling, no collective on the data
path); the step time is the max over ranks.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from emergence_b200 import replicas  # noqa: E402  (one process per GPU: barrier, max over ranks)

N_CELLS = 256
CPU_STEPS = 5  # timed steps of the CPU baseline on the full grid (about 5 s each on 16 host threads)
AMR_STEPS = 20
AMR_SC_STEPS = 5  # subcycled steps of the AMR sub-record (each spans about four global steps)
CELL_BYTES_3D = 320  # algorithmic bytes per 3-D cell-update (64·F, F = 5)
# flop per interior cell and sweep launch, counted by ncu on the 160^3 explosion
# (sm__sass_thread_inst_executed_op_{dadd,dmul,dfma,fadd,fmul,ffma}_pred_on, fma = 2)
SWEEP_FLOP = {"f64": {"fp64": 2104, "fp32": 120}, "mixed": {"fp64": 464, "fp32": 750}, "fast": {"fp64": 1332, "fp32": 0}}
# FP64 pipe of a B200: 148 SMs x 64 FMA lanes x 2 flop x 1.965 GHz (nominal; no measured FP64 peak exists here)
FP64_PEAK_TFLOPS = 148 * 64 * 2 * 1.965e9 / 1e12


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default: 100 for the uniform workload, the 3-D explosion's run length; "
                         "20 AMR steps; 3 whole runs or gradients for the batch and adjoint workloads)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="f64", choices=["f64", "mixed", "fast"],
                    help="fast: the fast FP64 form (uniform, AMR and batch workloads)")
    ap.add_argument("--n", "--grid", dest="n", type=int, default=N_CELLS, help="cells per side (default 256)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision leg of the uniform workload")
    ap.add_argument("--no-subrecords", action="store_true",
                    help="uniform workload: skip the AMR, batched-lines and adjoint records added to the line at N=1")
    ap.add_argument("--no-autotune", action="store_true", help="uniform and AMR workloads: use the planned sweep shapes")
    ap.add_argument("--no-reference-gpu", dest="reference_gpu", action="store_false",
                    help="uniform workload: skip the same-box GPU baseline, the reference's own GPU kernels timed on "
                         "the same grid (oracle/_ref/librefgpu.so, built from the reference tree by "
                         "`make -C oracle refgpu`; reported as unavailable where it is not built)")
    ap.add_argument("--workload", default="uniform",
                    choices=["uniform", "amr", "batch", "adjoint", "batch_adjoint", "five"],
                    help="uniform: 3-D explosion 256^3; amr: 3-D shock-bubble on block AMR (base 128^3, 3 levels); "
                         "batch: 4096 independent 1-D Riemann problems; adjoint: discrete adjoint of the 2-D "
                         "explosion 512^2 over 400 steps; batch_adjoint: gradients of the 4096 Riemann problems "
                         "with respect to their six initial values; five: five-equation two-phase shock-bubble")
    ap.add_argument("--five-n", type=int, default=128, help="five workload: cells per side")
    ap.add_argument("--adj-n", type=int, default=512, help="adjoint workload: cells per side")
    ap.add_argument("--adj-steps", type=int, default=400, help="adjoint workload: forward steps")
    ap.add_argument("--amr-base", type=int, default=8, help="AMR base blocks per side (16^3 cells each)")
    ap.add_argument("--subcycle", action="store_true", help="amr workload: subcycled steps (each level its own dt)")
    args = ap.parse_args()
    if args.precision == "fast" and args.workload not in ("uniform", "amr", "batch"):
        ap.error("--precision fast: the fast FP64 form is built for the uniform, AMR and batch workloads only")
    if args.steps is None:
        args.steps = {"uniform": 100, "amr": 20, "five": 10}.get(args.workload, 3)
        if args.impl == "reference":
            args.steps = 3
    return args


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.t.join(timeout=2)

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_init(args):
    return replicas.init_from_env("gloo" if args.impl == "reference" else "nccl")


def cpu_reference_steps(n, steps, warmup):
    """Time the reference CPU solver (C++ restatement, all host threads) on an
    n^3 instance of the same explosion; returns (cell-updates/s, seconds/step,
    threads, the hash of the final state as cpu_validate.rs:7-22 prints it)."""
    from emergence_b200 import workloads as W
    from emergence_b200.physics import FluxMode
    from oracle import pyoracle as O
    sys_, mesh, u, bc = W.explosion((n, n, n), 0.3)
    o = O.OracleSolver(sys_, mesh, u, bc=bc, mode=FluxMode.Weno, cfl=0.5)
    for _ in range(warmup):
        o.step(o.dt_cfl())
    t0 = time.perf_counter()
    for _ in range(steps):
        o.step(o.dt_cfl())
    el = time.perf_counter() - t0
    return mesh.cells() * steps / el, el / max(steps, 1), O.num_threads(), f"{O.state_hash(mesh, o.download()):016x}"


def uniform_config(n, world, precision):
    """The `config` of the uniform workload's line (both arms)."""
    return {"workload": f"3-D spherical explosion {n}^3 (r<0.3: rho=1,p=1; else 0.125,0.1; +-1% rho noise),"
                        " WCNS WENO5-Z + HLLC + positivity, SSP-RK3, CFL 0.5, outflow",
            "cells": n ** 3, "precision": precision,
            "parallelism": f"{world} independent replica(s), one GPU each",
            "l2": f"inputs larger than L2 (state {(n + 12) ** 3 * 40 / 1e9:.2f} GB per array)"}


def run_reference(args, world, rank):
    """--impl reference: the reference CPU solver on host cores (rank 0 only)."""
    if rank != 0:
        return
    # the full workload: the same 256^3 explosion, warmup + steps steps
    n = args.n
    value, sps, threads, fnv = cpu_reference_steps(n, args.steps, args.warmup)
    line = {
        "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": sps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": dict(uniform_config(n, world, "f64"), sample=f"the full {n}^3 grid, every step"),
        "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": threads, "kind": "port",
                         "sample": f"{args.steps} timed SSP-RK3 steps (after {args.warmup}) of the full {n}^3 explosion, "
                                   "C++ restatement of the reference CPU f64 solver (OpenMP over pencils)",
                         "state_fnv": fnv},
        "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, world, rank, local):
    import numpy as np
    import torch
    from emergence_b200 import GpuSolver, workloads as W
    from emergence_b200.physics import FluxMode, Precision

    torch.cuda.set_device(local)
    dev = torch.cuda.current_device()
    prec = {"mixed": Precision.Mixed, "fast": Precision.F64Fast}.get(args.precision, Precision.F64)
    n = args.n
    sys_, mesh, u, bc = W.explosion((n, n, n), 0.3)
    cells = mesh.cells()
    state_bytes = u.nbytes

    # ---- device-resident timing (value)
    tune = not args.no_autotune
    g = GpuSolver(sys_, mesh, u, bc=bc, mode=FluxMode.Weno, cfl=0.5, precision=prec, autotune=tune)
    g.advance(args.warmup)
    g.synchronize()
    stream = torch.cuda.ExternalStream(g.stream())
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g.set_profiling(True)
    g.kernel_times()  # reset
    replicas.barrier(world)
    torch.cuda.synchronize()
    l0 = g.launch_count()
    with ClockSampler(dev) as clk:
        start.record(stream)
        taken = g.advance(args.steps)
        end.record(stream)
        end.synchronize()
    torch.cuda.synchronize()
    launches = g.launch_count() - l0
    ms = start.elapsed_time(end)
    kt = g.kernel_times()
    g.set_profiling(False)
    ms = replicas.max_over_ranks(ms, world)
    replicas.barrier(world)
    assert taken == args.steps, taken
    value = cells * args.steps * world / (ms * 1e-3)

    # dominant kernel family: the fused sweeps (3 axes × 3 stages per step)
    sweep_ms = sum(kt[k][0] for k in ("axis0", "axis1", "axis2"))
    sweep_n = sum(kt[k][1] for k in ("axis0", "axis1", "axis2"))
    total_kernel_ms = sum(v[0] for v in kt.values())
    per_launch_ms = sweep_ms / max(sweep_n, 1)
    launches_per_step = sweep_n / max(args.steps, 1)
    alg_bytes_per_launch = CELL_BYTES_3D * cells / launches_per_step
    achieved = alg_bytes_per_launch / (per_launch_ms * 1e-3) / 1e9
    flop = SWEEP_FLOP[{Precision.Mixed: "mixed", Precision.F64Fast: "fast"}.get(prec, "f64")]
    fp64_tflops = flop["fp64"] * cells / (per_launch_ms * 1e-3) / 1e12
    fp64_roofline = {"bound": "fp64", "achieved": fp64_tflops, "peak": FP64_PEAK_TFLOPS, "unit": "TFLOP/s",
                     "frac": fp64_tflops / FP64_PEAK_TFLOPS, "flop_per_cell_per_launch": flop,
                     "flop_source": "ncu op counters, profiles/sweep_flops_uniform_160.md (plain form), "
                                    "profiles/sweep_fast_uniform_160.md (fast and mixed forms)",
                     "peak_source": "nominal FP64 FMA rate at 1965 MHz (148 SMs x 64 lanes x 2 flop)"}
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    traffic = None
    try:  # DRAM bytes per cell and launch of the FP64 sweep from the committed ncu capture
        tr = json.load(open(os.path.join(ROOT, "profiles", "sweep_traffic.json")))
        if prec == Precision.F64:
            traffic = tr["bytes_per_cell_per_launch"] * cells
    except Exception:
        pass
    row_staging = "TMA bulk tensor copies" if g.features() & 1 else "per-thread loads"
    u_main = g.download() if not (args.no_mixed and not args.reference_gpu) else None
    g.close()

    # ---- the reference's own GPU kernels on the same workload (same-box baseline)
    ref_gpu = None
    if args.reference_gpu and prec == Precision.F64 and rank == 0:
        ref_gpu = reference_gpu_leg(args, sys_, mesh, u, bc, cells, ms / args.steps, u_main)

    # ---- mixed-precision form (FP32 flux, FP64 state): same workload and steps
    mixed = None
    if not args.no_mixed and prec == Precision.F64:
        gm = GpuSolver(sys_, mesh, u, bc=bc, mode=FluxMode.Weno, cfl=0.5, precision=Precision.Mixed, autotune=tune)
        gm.advance(args.warmup)
        gm.synchronize()
        sm = torch.cuda.ExternalStream(gm.stream())
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(sm)
        gm.advance(args.steps)
        b.record(sm)
        b.synchronize()
        mms = a.elapsed_time(b)
        um = gm.download()
        gm.close()
        ia, ib = mesh.interior(um).reshape(-1, 5), mesh.interior(u_main).reshape(-1, 5)
        num, den = np.abs(ia - ib).sum(axis=0), np.abs(ib).sum(axis=0)
        den = np.maximum(den, 1e-3 * den[0])
        mixed = {"value": cells * args.steps * world / (mms * 1e-3), "ms_per_step": mms / args.steps,
                 "speedup_vs_f64": ms / mms,
                 "rel_l1_vs_f64_form": [float(x) for x in num / den],
                 "linf_vs_f64_form": [float(x) for x in np.abs(ia - ib).max(axis=0)],
                 "note": "after warmup+steps SSP-RK3 steps from the same initial state, each form with its own CFL dt; "
                         "the FP64 form is bit-exact with the CPU oracle in the parity tests"}

    # ---- fast FP64 form (FMA contraction, Newton-refined reciprocals): same workload and steps
    fast = None
    if not args.no_mixed and prec == Precision.F64:
        gf = GpuSolver(sys_, mesh, u, bc=bc, mode=FluxMode.Weno, cfl=0.5, precision=Precision.F64Fast, autotune=tune)
        gf.advance(args.warmup)
        gf.synchronize()
        sf = torch.cuda.ExternalStream(gf.stream())
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(sf)
        gf.advance(args.steps)
        b.record(sf)
        b.synchronize()
        fms = a.elapsed_time(b)
        uf = gf.download()
        gf.close()
        ia, ib = mesh.interior(uf).reshape(-1, 5), mesh.interior(u_main).reshape(-1, 5)
        num, den = np.abs(ia - ib).sum(axis=0), np.abs(ib).sum(axis=0)
        den = np.maximum(den, 1e-3 * den[0])
        fast = {"value": cells * args.steps * world / (fms * 1e-3), "ms_per_step": fms / args.steps,
                "speedup_vs_f64": ms / fms,
                "fp64_tflops_plain_equivalent": SWEEP_FLOP["f64"]["fp64"] * cells * 9 * args.steps / (fms * 1e-3) / 1e12,
                "fp64_tflops_executed": SWEEP_FLOP["fast"]["fp64"] * cells * 9 * args.steps / (fms * 1e-3) / 1e12,
                "rel_l1_vs_f64_form": [float(x) for x in num / den],
                "linf_vs_f64_form": [float(x) for x in np.abs(ia - ib).max(axis=0)],
                "note": "all arithmetic FP64 with FMA contraction and Newton-refined reciprocals/square roots "
                        "(about 1 ulp) in place of correctly rounded divisions; held to 1e-12 relative L1 against "
                        "the oracle in the parity tests; fp64_tflops_plain_equivalent counts the plain form's 2104 "
                        "flop per cell and launch, fp64_tflops_executed the fast form's own 1332 (ncu, "
                        "profiles/sweep_fast_uniform_160.md); both over the whole step time"}

    # ---- end to end through the C ABI with host buffers
    e2e = None
    if not args.no_e2e:
        # the caller's host buffers, page-locked (allocated and filled before the clock starts)
        host = torch.empty(tuple(u.shape), dtype=torch.float64, pin_memory=True).numpy()
        host[...] = u
        out_host = torch.empty(tuple(u.shape), dtype=torch.float64, pin_memory=True).numpy()
        # one untimed pass first (first-touch costs of the buffers and the CUDA driver's allocations)
        for timed in (False, True):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            h = GpuSolver(sys_, mesh, host, bc=bc, mode=FluxMode.Weno, cfl=0.5, precision=prec, autotune=tune)
            h.synchronize()
            t1 = time.perf_counter()
            h.advance(args.steps if timed else args.warmup)
            out = h.download(out=out_host)
            el = time.perf_counter() - t0
            h.close()
        e2e = {"value": cells * args.steps * world / el, "unit": "cell-updates/s",
               "h2d_bytes_per_step": state_bytes / args.steps, "d2h_bytes_per_step": out.nbytes / args.steps,
               "create_upload_ms": (t1 - t0) * 1e3, "total_ms": el * 1e3,
               "what": "GpuSolver(host AoS state) + advance(K) + download(host AoS), wall clock; host buffers "
                       "page-locked; after one untimed pass"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the same grid and initial state, the first CPU_STEPS steps (after one untimed step)
        v, sps, threads, fnv = cpu_reference_steps(n, CPU_STEPS, 1)
        cpu = {"value": v, "unit": "cell-updates/s", "cores": threads, "kind": "port",
               "sample": f"{CPU_STEPS} timed SSP-RK3 steps (after 1 untimed) of the same {n}^3 explosion, "
                         "C++ restatement of the reference CPU f64 solver (OpenMP over pencils)",
               "seconds_per_step": sps, "state_fnv": fnv}

    subs = {}
    if rank == 0 and world == 1 and not args.no_subrecords:
        subs = sub_records(args, world, rank, local)

    if rank == 0:
        line = {
            "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32-flux/f64-state" if prec == Precision.Mixed else "f64", "data": "synthetic",
            "config": dict(uniform_config(n, world, args.precision), sweep_row_loads=row_staging),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "traffic_source": "ncu capture on 160^3 scaled by cells (profiles/)", "kernel": "fused sweep (3 per stage)",
                         "alg_bytes_per_launch": alg_bytes_per_launch, "avg_launch_ms": per_launch_ms,
                         "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks else "fallback",
                         "compute_note": "the sweep is FP64-ALU bound (59 FP64 flop per algorithmic byte): FP64 pipe "
                                         "45-50 % active at 4 CTAs per SM (ncu, profiles/sweep_flops_uniform_160.md); "
                                         "the HBM fraction is small by construction",
                         "fp64": fp64_roofline},
            "kernel_ms_per_step": {k: v[0] / args.steps for k, v in kt.items()},
            "kernel_share": {k: (v[0] / total_kernel_ms if total_kernel_ms else None) for k, v in kt.items()},
            "gpu_launches": launches,
            "clocks": clk.summary(),
            "e2e": e2e,
            "cpu_baseline": cpu,
            "mixed": mixed,
            "fast_f64": fast,
        }
        if ref_gpu is not None:
            line["reference_gpu"] = ref_gpu
        line.update(subs)
        print(json.dumps(line), flush=True)


def _compact(line, keys):
    return {k: line[k] for k in keys if k in line}


def sub_records(args, world, rank, local):
    """The other workloads, each measured in both forms on the same box in
    the same run (one GPU): block AMR (20 steps of the shock-bubble), the
    4096 batched Riemann problems (one whole run), the 2-D adjoint (one
    gradient with its finite-difference check) and the batched gradients."""
    import numpy as np
    out = {}
    amr = {}
    for prec in ("f64", "mixed", "fast"):
        ln = measure_amr(args, world, rank, local, precision=prec, steps=AMR_STEPS, warmup=3, cpu_baseline=False,
                         keep_state=True)
        amr[prec] = ln
    a64, amx, afs = amr["f64"], amr["mixed"], amr["fast"]
    rec = {"workload": "3-D shock-bubble block AMR, base 128^3, 3 levels (eff. 512^3), 16^3 blocks, ng=5, CFL 0.4, "
                       f"regrid every 4 steps; {AMR_STEPS} timed steps after 3, each form with its own CFL dt",
           "unit": "leaf cell-updates/s"}
    for prec in ("f64", "mixed", "fast"):
        key = "fast_f64" if prec == "fast" else prec
        rec[key] = _compact(amr[prec], ("value", "ms_per_step", "effective_cell_updates_per_s", "phase_ms_per_step",
                                        "gpu_launches", "clocks"))
        rec[key]["leaves"] = amr[prec]["config"]["leaves"]
        rec[key]["build_s"] = amr[prec]["config"]["build_s"]
    rec["mixed_over_f64"] = a64["ms_per_step"] / amx["ms_per_step"]
    rec["fast_f64_over_f64"] = a64["ms_per_step"] / afs["ms_per_step"]
    (s64, u64), (smx, umx), (sfs, ufs) = a64.pop("_state"), amx.pop("_state"), afs.pop("_state")
    if s64.shape == sfs.shape and np.array_equal(s64, sfs):
        leaves = s64[:, 4] == 1
        ia, ib = ufs[leaves].reshape(-1, 5), u64[leaves].reshape(-1, 5)
        num, den = np.abs(ia - ib).sum(axis=0), np.abs(ib).sum(axis=0)
        rec["rel_l1_fast_f64_vs_f64"] = [float(x) for x in num / np.maximum(den, 1e-3 * den[0])]
    else:
        rec["rel_l1_fast_f64_vs_f64"] = "hierarchies differ after the regrids (a detail moved a decision)"
    if s64.shape == smx.shape and np.array_equal(s64, smx):
        leaves = s64[:, 4] == 1
        ia, ib = umx[leaves].reshape(-1, 5), u64[leaves].reshape(-1, 5)
        num, den = np.abs(ia - ib).sum(axis=0), np.abs(ib).sum(axis=0)
        rec["rel_l1_mixed_vs_f64"] = [float(x) for x in num / np.maximum(den, 1e-3 * den[0])]
        rec["linf_mixed_vs_f64"] = [float(x) for x in np.abs(ia - ib).max(axis=0)]
    else:
        rec["rel_l1_mixed_vs_f64"] = "hierarchies differ after the regrids (mixed-form details moved a decision)"
    # subcycled steps of the same workload (FP64): simulated time per second against the global step's
    sc = measure_amr(args, world, rank, local, precision="f64", steps=AMR_SC_STEPS, warmup=1, cpu_baseline=False,
                     subcycle=True)
    rec["subcycled_f64"] = _compact(sc, ("value", "ms_per_step", "sim_time_per_s", "gpu_launches", "clocks"))
    rec["subcycled_f64"]["steps"] = AMR_SC_STEPS
    rec["subcycled_f64"]["leaves"] = sc["config"]["leaves"]
    rec["subcycled_f64"]["leaves_per_level"] = sc["config"]["leaves_per_level"]
    rec["subcycled_f64"]["sim_time_per_s_global_f64"] = a64["sim_time_per_s"]
    rec["subcycled_f64"]["note"] = ("one step = one subcycled step (coarsest leaf level by dt, level l by dt/2^(l-lmin), "
                                    "a regrid after each); value counts every level's substeps")
    out["amr"] = rec

    bat = {}
    for prec in ("f64", "mixed", "fast"):
        bat[prec] = measure_batch(args, world, rank, local, precision=prec, steps=1, warmup=1, cpu_baseline=False)
    out["batch"] = {"workload": bat["f64"]["config"]["workload"], "unit": "cell-updates/s",
                    "f64": _compact(bat["f64"], ("value", "ms_per_step", "clocks")),
                    "mixed": _compact(bat["mixed"], ("value", "ms_per_step", "clocks")),
                    "fast_f64": _compact(bat["fast"], ("value", "ms_per_step", "clocks")),
                    "mixed_over_f64": bat["f64"]["ms_per_step"] / bat["mixed"]["ms_per_step"],
                    "fast_f64_over_f64": bat["f64"]["ms_per_step"] / bat["fast"]["ms_per_step"]}

    adj = measure_adjoint(args, world, rank, local, steps=1, warmup=1)
    out["adjoint"] = _compact(adj, ("value", "unit", "forward_ms", "recompute_ms", "reverse_ms",
                                    "forward_cell_updates_per_s", "fd_check", "clocks"))
    out["adjoint"]["workload"] = adj["config"]["workload"]
    rec = {}
    for prec in ("f64", "mixed"):
        badj = measure_batch_adjoint(args, world, rank, local, steps=1, warmup=1, dual_check=False, precision=prec)
        rec[prec] = _compact(badj, ("value", "unit", "forward_ms", "recompute_ms", "reverse_ms", "clocks"))
        rec["workload"] = badj["config"]["workload"]
    rec["note"] = ("value = backward/forward cost; the mixed batch records its FP32-flux run and applies the FP64 "
                   "step's transposed Jacobian at its stage states")
    out["batch_adjoint"] = rec
    out["five"] = measure_five(args, world, rank, local)
    out["five"]["amr"] = measure_five_amr(args, world, rank, local)
    fa = measure_five_amr(args, world, rank, local, fast=True)
    out["five"]["amr"]["fast_f64"] = {k: fa[k] for k in ("value", "ms_per_step", "phase_ms_per_step", "clocks")}
    out["five"]["amr"]["fast_f64"]["speedup_vs_f64"] = out["five"]["amr"]["ms_per_step"] / fa["ms_per_step"]
    return out


def measure_five_amr(args, world, rank, local, base=8, steps=5, warmup=2, fast=False):
    """The five-equation two-phase shock–bubble on the block hierarchy: the
    light-gas sphere (γ 1.67, ρ 0.138) in air hit by a Mach-2 shock, 16^3-cell
    blocks, base 8^3 blocks (128^3), 3 levels (effective 512^3), CFL 0.4 with
    the dilatation limit, regrid every 4 steps; global steps, FP64, timed with
    CUDA events on the solver's stream (leaf cell-updates per second); `fast`:
    the fast FP64 form of the sweeps."""
    import torch
    from emergence_b200 import GpuAmr, workloads as W
    from emergence_b200.physics import FluxMode, Precision
    torch.cuda.set_device(local)
    dev = torch.cuda.current_device()
    s, cfg, lo, hi, bc, init = W.two_phase_amr_bubble(dim=3, base=base, levels=3)
    t0 = time.perf_counter()
    g = GpuAmr(s, cfg, lo, hi, bc, init, mode=FluxMode.Weno, cfl=0.4,
               precision=Precision.F64Fast if fast else Precision.F64)
    build_s = time.perf_counter() - t0
    for _ in range(warmup):
        g.step(g.dt_cfl())
    g.synchronize()
    g.phase_times()  # reset the phase clocks after the warm-up
    stream = torch.cuda.ExternalStream(g.stream())
    leaf_cells = 0
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    with ClockSampler(dev) as clk:
        a.record(stream)
        for _ in range(steps):
            leaf_cells += g.block_count()[1] * g.bcells
            g.step(g.dt_cfl())
        b.record(stream)
        b.synchronize()
    ms = a.elapsed_time(b)
    st = g.structure()
    per_level = [int(((st[:, 0] == l) & (st[:, 4] == 1)).sum()) for l in range(cfg["levels"])]
    phases = g.phase_times()
    g.close()
    return {"workload": "five-equation two-phase shock-bubble on block AMR, base 128^3 = 8^3 blocks of 16^3, 3 levels "
                        "(eff. 512^3), WCNS WENO5-Z + HLLC + positivity, CFL 0.4 with the dilatation limit, regrid "
                        "every 4 steps, FP64",
            "unit": "leaf cell-updates/s", "steps": steps, "warmup": warmup,
            "value": leaf_cells / (ms * 1e-3), "ms_per_step": ms / steps, "leaves_per_level": per_level,
            "phase_ms_per_step": {k: v / steps for k, v in phases.items()}, "build_s": build_s,
            "clocks": clk.summary()}


def run_five(args, world, rank, local):
    rec = measure_five(args, world, rank, local, n=args.five_n, steps=args.steps, warmup=args.warmup,
                       reference=args.reference_gpu)
    if rank == 0:
        line = {"metric": "cell-updates/s", "value": rec["value"], "unit": "cell-updates/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": rec["ms_per_step"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": rec["workload"]}, "gpu_launches": rec["gpu_launches_total"],
                "clocks": rec["clocks"], "reference_gpu": rec["reference_gpu"], "fast_f64": rec["fast_f64"]}
        print(json.dumps(line), flush=True)


def measure_five(args, world, rank, local, n=128, steps=10, warmup=3, reference=True):
    """Five-equation two-phase shock–bubble (Kapila's model) on n^3 cells: this
    library's fused sweeps and, on the same box and grid, the reference's own
    `five` GPU kernels (the same-box baseline); each advances warmup + steps
    CFL steps with a device→host time step per step, timed with CUDA events on
    its stream."""
    import numpy as np
    import torch
    from emergence_b200 import GpuFiveSolver, workloads as W
    from emergence_b200.physics import FluxMode
    torch.cuda.set_device(local)
    dev = torch.cuda.current_device()
    sys_, mesh, u, bc = W.two_phase_shock_bubble(n)
    cells = mesh.cells()
    g = GpuFiveSolver(sys_, mesh, u, bc=bc, cfl=0.5, mode=FluxMode.Weno)
    for _ in range(warmup):
        g.step(g.dt_cfl())
    s = torch.cuda.ExternalStream(g.stream())
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    with ClockSampler(dev) as clk:
        a.record(s)
        for _ in range(steps):
            g.step(g.dt_cfl())
        b.record(s)
        b.synchronize()
    ms = a.elapsed_time(b)
    ours = g.download()
    l0 = g.launch_count()
    g.close()
    rec = {"workload": f"five-equation two-phase shock-bubble {n}^3 (light gas gamma 1.67 rho 0.138 sphere r=0.15 in "
                       "air, Mach-2 shock), WCNS WENO5-Z + HLLC + positivity, SSP-RK3, CFL 0.5, outflow, FP64",
           "unit": "cell-updates/s", "steps": steps, "warmup": warmup,
           "value": cells * steps / (ms * 1e-3), "ms_per_step": ms / steps, "gpu_launches_total": l0,
           "clocks": clk.summary()}
    # the fast FP64 form on the same grid and steps
    from emergence_b200.physics import Precision
    gf = GpuFiveSolver(sys_, mesh, u, bc=bc, cfl=0.5, mode=FluxMode.Weno, precision=Precision.F64Fast)
    for _ in range(warmup):
        gf.step(gf.dt_cfl())
    sf = torch.cuda.ExternalStream(gf.stream())
    a3, b3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a3.record(sf)
    for _ in range(steps):
        gf.step(gf.dt_cfl())
    b3.record(sf)
    b3.synchronize()
    fms = a3.elapsed_time(b3)
    uf = gf.download()
    gf.close()
    ia, ib = mesh.interior(uf).reshape(-1, 7), mesh.interior(ours).reshape(-1, 7)
    num, den = np.abs(ia - ib).sum(axis=0), np.abs(ib).sum(axis=0)
    rec["fast_f64"] = {"value": cells * steps / (fms * 1e-3), "ms_per_step": fms / steps, "speedup_vs_f64": ms / fms,
                       "rel_l1_vs_f64_form": [float(x) for x in num / np.maximum(den, 1e-3 * (den[0] + den[1]))]}
    from oracle import pyrefgpu
    if not reference:
        rec["reference_gpu"] = None
    elif pyrefgpu.available():
        r = pyrefgpu.RefGpuFiveSolver(sys_, mesh, u, bc=bc, cfl=0.5, mode=FluxMode.Weno)
        r.advance(warmup)
        r.synchronize()
        sr = torch.cuda.ExternalStream(r.stream())
        a2, b2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a2.record(sr)
        r.advance(steps)
        b2.record(sr)
        b2.synchronize()
        rms = a2.elapsed_time(b2)
        ur = r.download()
        r.close()
        ia, ib = mesh.interior(ur).reshape(-1, 7), mesh.interior(ours).reshape(-1, 7)
        num, den = np.abs(ia - ib).sum(axis=0), np.abs(ib).sum(axis=0)
        rec["reference_gpu"] = {"value": cells * steps / (rms * 1e-3), "ms_per_step": rms / steps,
                                "ours_speedup": rms / ms,
                                # the transverse momenta are round-off until the shock meets the
                                # bubble: measured against the total density
                                "rel_l1_vs_ours": [float(x) for x in num / np.maximum(den, 1e-3 * (den[0] + den[1]))],
                                "what": "the reference's compressible-cuda five_f64 kernels (unmodified source, nvcc "
                                        "sm_100a) in GpuSolver<f64> launch order"}
    else:
        rec["reference_gpu"] = {"unavailable": "oracle/_ref/librefgpu.so is not built"}
    return rec


def reference_gpu_leg(args, sys_, mesh, u, bc, cells, ours_ms_per_step, u_ours):
    """Same-box GPU baseline: the reference's uniform-solver kernels
    (fluid/crates/compressible-cuda/src/kernels.cu, compiled unmodified for
    sm_100a) driven in the order of its GpuSolver<f64> (oracle/ref_gpu.cu, bound
    by oracle/pyrefgpu.py) over warmup + steps steps of the same explosion, each
    step's dt from its own rate kernel and host max as in its run_to loop. Timed
    with CUDA events on its stream; the per-step device→host copy of the rates
    is part of that design and inside the timed region."""
    import numpy as np
    import torch
    from emergence_b200.physics import FluxMode
    from oracle import pyrefgpu

    if not pyrefgpu.available():
        return {"unavailable": "oracle/_ref/librefgpu.so is not built (make -C oracle refgpu needs the reference tree)"}
    try:
        r = pyrefgpu.RefGpuSolver(sys_, mesh, u, bc=bc, cfl=0.5, mode=FluxMode.Weno)
    except RuntimeError as ex:
        return {"error": str(ex)}
    try:
        r.advance(args.warmup)
        r.synchronize()
        s = torch.cuda.ExternalStream(r.stream())
        a, z = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(s)
        r.advance(args.steps)
        z.record(s)
        z.synchronize()
        rms = a.elapsed_time(z)
        out = r.download()
    except RuntimeError as ex:
        return {"error": str(ex)}
    finally:
        r.close()
    res = {"value": cells * args.steps / (rms * 1e-3), "unit": "cell-updates/s", "ms_per_step": rms / args.steps,
           "ours_speedup": (rms / args.steps) / ours_ms_per_step,
           "what": "the reference's compressible-cuda kernels (unmodified source, nvcc sm_100a) in GpuSolver<f64> "
                   "launch order: ghost, prim, theta/midflux/flux/accum per axis, rk per stage; dt_cfl each step"}
    if u_ours is not None:
        ia, ib = mesh.interior(out).reshape(-1, 5), mesh.interior(u_ours).reshape(-1, 5)
        num, den = np.abs(ia - ib).sum(axis=0), np.abs(ib).sum(axis=0)
        res["rel_l1_vs_ours"] = [float(x) for x in num / np.maximum(den, 1e-3 * den[0])]
    return res


def run_amr(args, world, rank, local):
    line = measure_amr(args, world, rank, local, subcycle=args.subcycle)
    if rank == 0:
        print(json.dumps(line), flush=True)


def measure_amr(args, world, rank, local, precision=None, steps=None, warmup=None, cpu_baseline=True, keep_state=False,
                subcycle=False):
    """3-D shock-bubble on block AMR: Mach-2 shock into a light sphere,
    16^3-cell blocks, base 8^3 blocks (128^3 cells), 3 levels (effective
    512^3), ng = 5, regrid every 4 steps, CFL 0.4. One step = one global
    SSP-RK3 step over all leaves (regrids included when due), dt from the
    CFL reduction over the leaves each step; with subcycle, one subcycled
    step (the coarsest leaf level by dt, level l by dt/2^(l-lmin), a regrid
    after every such step by the reference's schedule), whose leaf
    cell-updates count each level's substeps. Returns the JSON line (on every
    rank; rank 0 prints it); with keep_state, also the final hierarchy and
    leaf data under "_state"."""
    import numpy as np
    import torch
    from emergence_b200 import GpuAmr, workloads as W
    from emergence_b200.physics import FluxMode, Precision

    torch.cuda.set_device(local)
    dev = torch.cuda.current_device()
    precision = args.precision if precision is None else precision
    steps = args.steps if steps is None else steps
    warmup = args.warmup if warmup is None else warmup
    prec = {"mixed": Precision.Mixed, "fast": Precision.F64Fast}.get(precision, Precision.F64)
    s, cfg, lo, hi, bc, init = W.shock_bubble(dim=3, base=args.amr_base, levels=3)
    t0 = time.perf_counter()
    g = GpuAmr(s, cfg, lo, hi, bc, init, mode=FluxMode.Weno, cfl=0.4, precision=prec, autotune=not args.no_autotune,
               subcycle=subcycle)
    build_s = time.perf_counter() - t0

    def one_step():
        if subcycle:
            st = g.structure()
            lv = st[st[:, 4] == 1, 0]
            dt = g.dt_cfl_subcycled()
            g.step_subcycled(dt)
            return int((2.0 ** (lv - lv.min())).sum()) * g.bcells, dt
        n = g.block_count()[1] * g.bcells
        dt = g.dt_cfl()
        g.step(dt)
        return n, dt

    for _ in range(warmup):
        one_step()
    g.synchronize()
    g.phase_times()
    stream = torch.cuda.ExternalStream(g.stream())
    leaf_cells, sim_t = 0, 0.0
    l0 = g.launch_count()
    replicas.barrier(world)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev) as clk:
        a.record(stream)
        for _ in range(steps):
            n, dt = one_step()
            leaf_cells += n
            sim_t += dt
        b.record(stream)
        b.synchronize()
    ms = a.elapsed_time(b)
    phases = g.phase_times()
    launches = g.launch_count() - l0
    ms = replicas.max_over_ranks(ms, world)
    value = leaf_cells * world / (ms * 1e-3)
    eff_cells = 1
    for d in range(3):
        if cfg["base_blocks"][d] > 0:
            eff_cells *= cfg["base_blocks"][d] * cfg["b"] * 2 ** (cfg["levels"] - 1)
    nb, nl = g.block_count()
    st = g.structure()
    per_level = [int(((st[:, 0] == l) & (st[:, 4] == 1)).sum()) for l in range(cfg["levels"])]
    state = (st, g.download()) if keep_state else None
    g.close()
    cpu = None
    if rank == 0 and world == 1 and cpu_baseline and not args.no_cpu_baseline:
        from oracle import pyoracle as O
        sc, cfgc, loc, hic, bcc, initc = W.shock_bubble(dim=3, base=2, levels=3)
        o = O.OracleAmr(sc, cfgc, loc, hic, bcc, initc, mode=FluxMode.Weno, cfl=0.4)
        cells_c = o.block_count()[1] * (cfgc["b"] ** 3)
        tc = time.perf_counter()
        o.step(o.dt_cfl())
        el = time.perf_counter() - tc
        cpu = {"value": cells_c / el, "unit": "cell-updates/s", "cores": O.num_threads(), "kind": "port",
               "sample": f"1 step of the shock-bubble with base 2^3 blocks (32^3), 3 levels, {o.block_count()[1]} leaves; "
                         "C++ restatement of the reference CPU AMR solver"}
    line = {
        "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
        "steps": steps, "warmup": warmup, "ms_per_step": ms / steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32-flux/f64-state" if prec == Precision.Mixed else "f64",
        "data": "synthetic",
        "config": {"workload": "3-D shock-bubble block AMR: Mach-2 shock into rho=0.138 sphere r=0.15 (+-0.5% "
                               "seeded interface perturbation), base 128^3 = 8^3 blocks of 16^3, 3 levels (eff. 512^3), "
                               "ng=5, WCNS WENO5-Z + HLLC + positivity, CFL 0.4, regrid every 4 steps",
                   "blocks": nb, "leaves": nl, "leaves_per_level": per_level, "build_s": build_s,
                   "autotune": not args.no_autotune,
                   "precision": precision},
        "phase_ms_per_step": {k: v / steps for k, v in phases.items()},
        # the same steps counted at the finest level's resolution over the whole
        # domain (what a uniform grid of the finest spacing would update per step)
        "effective_cell_updates_per_s": eff_cells * steps * world / (ms * 1e-3),
        "effective_cells": eff_cells,
        "sim_time_per_s": sim_t / (ms * 1e-3),
        "subcycle": subcycle,
        "gpu_launches": launches,
        "clocks": clk.summary(),
        "cpu_baseline": cpu,
    }
    if state is not None:
        line["_state"] = state
    return line


def run_batch(args, world, rank, local):
    line = measure_batch(args, world, rank, local)
    if rank == 0:
        print(json.dumps(line), flush=True)


def measure_batch(args, world, rank, local, precision=None, steps=None, warmup=None, cpu_baseline=True):
    """4096 independent 1-D Riemann problems (cells log-uniform in [64, 2048],
    ρ, p ∈ U[0.1, 2], u ∈ U[−1, 1] on each side, interface at 0.5, outflow),
    each run to t = 0.15 with its own CFL steps, all instances in one launch
    per RK stage. One "step" = one whole run; the metric counts the cell
    updates of every instance."""
    import numpy as np
    import torch
    from emergence_b200 import GpuBatch1D, workloads as W
    from emergence_b200.physics import FluxMode, Precision

    torch.cuda.set_device(local)
    dev = torch.cuda.current_device()
    precision = args.precision if precision is None else precision
    steps = args.steps if steps is None else steps
    warmup = args.warmup if warmup is None else warmup
    prec = {"mixed": Precision.Mixed, "fast": Precision.F64Fast}.get(precision, Precision.F64)
    sys_, n, dx, u, st = W.riemann_batch()
    for _ in range(max(warmup, 1)):
        g = GpuBatch1D(sys_, n, dx, u, precision=prec)
        g.run_to(0.15)
        g.close()
    total_ms, updates = 0.0, 0
    replicas.barrier(world)
    with ClockSampler(dev) as clk:
        for _ in range(steps):
            g = GpuBatch1D(sys_, n, dx, u, precision=prec)
            stream = torch.cuda.ExternalStream(g.stream())
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            a.record(stream)
            launched = g.run_to(0.15)
            b.record(stream)
            b.synchronize()
            total_ms += a.elapsed_time(b)
            _, inst_steps = g.status()
            updates += int((n * inst_steps.astype(np.int64)).sum())
            g.close()
    total_ms = replicas.max_over_ranks(total_ms, world)
    value = updates * world / (total_ms * 1e-3)
    cpu = None
    if rank == 0 and world == 1 and cpu_baseline and not args.no_cpu_baseline:
        from oracle import pyoracle as O
        from emergence_b200.physics import Bc, Mesh
        sub = slice(0, 256, 8)  # 32 instances of the same batch
        cu, tc = 0, time.perf_counter()
        offs = np.concatenate([[0], np.cumsum(n)])
        for i in range(*sub.indices(len(n))):
            mesh = Mesh.new((int(n[i]), 1, 1), (0, 0, 0), (1, 1, 1), ng=6)
            uu = np.zeros((mesh.len(), 5))
            uu[6:6 + n[i]] = u[offs[i]:offs[i + 1]]
            o = O.OracleSolver(sys_, mesh, uu, bc=[[Bc.Outflow] * 2, [Bc.Periodic] * 2, [Bc.Periodic] * 2],
                               mode=FluxMode.Weno, cfl=0.5)
            cu += int(n[i]) * o.run_to(0.15)
        el = time.perf_counter() - tc
        cpu = {"value": cu / el, "unit": "cell-updates/s", "cores": O.num_threads(), "kind": "port",
               "sample": "32 of the 4096 instances (every 8th of the first 256), each run to t = 0.15; "
                         "C++ restatement of the reference CPU solver"}
    line = {
        "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
        "steps": steps, "warmup": warmup, "ms_per_step": total_ms / steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32-flux/f64-state" if prec == Precision.Mixed else "f64",
        "data": "synthetic",
        "config": {"workload": "4096 independent 1-D Riemann problems, cells log-uniform [64, 2048] (sum %d), "
                               "rho,p~U[0.1,2], u~U[-1,1], t_end 0.15, outflow, per-instance CFL 0.5" % int(n.sum()),
                   "step": "one whole batched run to t_end", "batch_steps": int(launched),
                   "precision": precision},
        "clocks": clk.summary(),
        "cpu_baseline": cpu,
    }
    return line


def run_adjoint(args, world, rank, local):
    line = measure_adjoint(args, world, rank, local)
    if rank == 0:
        print(json.dumps(line), flush=True)


def measure_adjoint(args, world, rank, local, steps=None, warmup=None):
    """Discrete adjoint of the 2-D explosion (radius 0.4, ±1 % density noise,
    outflow) on 512^2 cells over 400 CFL steps, FP64 forward and adjoint:
    J = ∫ p dA over [0.7, 0.9]^2 at the end, gradient with respect to the
    initial density field and γ with √N checkpointing. One "step" = one
    forward run + one backward pass; checked against central finite
    differences of the forward run along a seeded direction (h = 1e-6, time
    steps held fixed)."""
    import numpy as np
    import torch
    from emergence_b200 import DifferentiableSolver, workloads as W
    from emergence_b200.adjoint import OBJ_PRESSURE
    from emergence_b200.physics import Euler, Nasg, initial_state

    torch.cuda.set_device(local)
    dev = torch.cuda.current_device()
    steps = args.steps if steps is None else steps
    warmup = args.warmup if warmup is None else warmup
    n, N = args.adj_n, args.adj_steps
    sys_, mesh, w, bc = W.explosion_prim((n, n, 1), 0.4)
    u0 = initial_state(sys_, mesh, w)
    box = ([0.7, 0.7, 0.0], [0.9, 0.9, 0.0])
    g = DifferentiableSolver(sys_, mesh, u0, bc=bc)
    for _ in range(max(warmup, 1)):
        g.forward(N)
        g.objective(OBJ_PRESSURE, *box)
        g.backward()
    fwd_ms, rec_ms, rev_ms, wall = [], [], [], []
    with ClockSampler(dev) as clk:
        for _ in range(steps):
            t0 = time.perf_counter()
            g.forward(N)
            J = g.objective(OBJ_PRESSURE, *box)
            ub, wb, gam = g.backward()
            wall.append(time.perf_counter() - t0)
            ms = g.times()
            fwd_ms.append(ms[0])
            rec_ms.append(ms[1])
            rev_ms.append(ms[2])
    dts = g.dts()
    # finite-difference check along a seeded direction of (ρ⁰, γ)
    rng = np.random.default_rng(20261203)
    dw = np.zeros_like(w)
    dw[..., 0] = rng.uniform(-1.0, 1.0, w.shape[:-1])
    dgamma = 0.5
    adj = float((mesh.interior(wb)[..., 0] * dw[..., 0]).sum() + gam[1] * dgamma)
    h = 1e-6

    def J_of(step):
        s2 = Euler(Nasg.ideal(1.4 + step * dgamma))
        g2 = DifferentiableSolver(s2, mesh, initial_state(s2, mesh, w + step * dw), bc=bc)
        g2.forward(dts=dts)
        v = g2.objective(OBJ_PRESSURE, *box)
        g2.close()
        return v

    fd = (J_of(h) - J_of(-h)) / (2 * h)
    h7 = 1e-7
    fd7 = (J_of(h7) - J_of(-h7)) / (2 * h7)
    g.close()
    f, r, v = float(np.median(fwd_ms)), float(np.median(rec_ms)), float(np.median(rev_ms))
    # the slowest replica's phases (a ratio of device times; every rank takes the same steps)
    f, r, v = (replicas.max_over_ranks(x, world) for x in (f, r, v))
    cells = mesh.cells()
    line = {
        "metric": "adjoint/forward cost", "value": (r + v) / f, "unit": "ratio", "n_gpus": world,
        "steps": steps, "warmup": warmup, "ms_per_step": f + r + v, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"2-D explosion {n}^2 (r<0.4: rho=1,p=1; else 0.125,0.1; +-1% rho noise), "
                               f"{N} CFL steps, WCNS WENO5-Z + HLLC + positivity, SSP-RK3, CFL 0.5, outflow",
                   "objective": "J = sum p dA over [0.7,0.9]^2 at t_end", "checkpoints": "every ceil(sqrt(N)) steps",
                   "step": "one recorded forward run + one backward pass"},
        "forward_ms": f, "recompute_ms": r, "reverse_ms": v,
        "reverse_over_forward": v / f, "backward_over_forward": (r + v) / f,
        "forward_cell_updates_per_s": cells * N / (f * 1e-3),
        "wall_s_per_gradient": float(np.median(wall)),
        "J": J, "t_end": float(dts.sum()), "gamma_bar": [float(gam[0]), float(gam[1])],
        "fd_check": {"h": h, "direction": "seeded uniform(-1,1) on rho0 interior, 0.5 on gamma",
                     "fd": fd, "adjoint": adj, "rel_err": abs(fd - adj) / abs(adj),
                     "h_1e-7": {"fd": fd7, "rel_err": abs(fd7 - adj) / abs(adj)}},
        "clocks": clk.summary(),
    }
    return line


def run_batch_adjoint(args, world, rank, local):
    line = measure_batch_adjoint(args, world, rank, local)
    if rank == 0:
        print(json.dumps(line), flush=True)


def measure_batch_adjoint(args, world, rank, local, steps=None, warmup=None, dual_check=True, precision=None):
    """Gradients of the 4096 independent 1-D Riemann problems: J_i = total
    energy in the right half [0.5, 1] at t = 0.15, differentiated with respect
    to the six initial values (ρ, u, p left and right of x = 0.5) of every
    instance in one batched backward pass (FP64 forward recorded with its
    CFL steps, checkpoints every 64 batch steps). One "step" = one recorded
    run + one backward pass; checked against per-instance CPU dual-number
    runs (oracle) on a sample of instances."""
    import numpy as np
    import torch
    from emergence_b200 import GpuBatch1D, workloads as W
    from emergence_b200.adjoint import OBJ_ENERGY
    from emergence_b200.physics import Bc, FluxMode, Mesh

    torch.cuda.set_device(local)
    dev = torch.cuda.current_device()
    from emergence_b200.physics import Precision
    steps = args.steps if steps is None else steps
    warmup = args.warmup if warmup is None else warmup
    precision = args.precision if precision is None else precision
    prec = Precision.Mixed if precision == "mixed" else Precision.F64
    sys_, n, dx, u, st = W.riemann_batch()
    g = GpuBatch1D(sys_, n, dx, u, precision=prec)
    for _ in range(max(warmup, 1)):
        g.record(0.15)
        g.objective(OBJ_ENERGY, 0.5, 1.0)
        g.backward(0.5)
    fwd, rec, rev = [], [], []
    with ClockSampler(dev) as clk:
        for _ in range(steps):
            B = g.record(0.15)
            J = g.objective(OBJ_ENERGY, 0.5, 1.0)
            grad = g.backward(0.5)
            ms = g.adjoint_times()
            fwd.append(ms[0])
            rec.append(ms[1])
            rev.append(ms[2])
    _, inst_steps = g.status()
    g.close()
    f, r, v = float(np.median(fwd)), float(np.median(rec)), float(np.median(rev))
    f, r, v = (replicas.max_over_ranks(x, world) for x in (f, r, v))
    updates = int((n * inst_steps.astype(np.int64)).sum())
    check = None
    if rank == 0 and dual_check and not args.no_cpu_baseline:
        from oracle import pyoracle as O
        bc = [[Bc.Outflow, Bc.Outflow], [Bc.Periodic, Bc.Periodic], [Bc.Periodic, Bc.Periodic]]
        offs = np.concatenate([[0], np.cumsum(n)])
        sample = [int(i) for i in np.argsort(n)[:4]]  # the four shortest instances
        worst = 0.0
        for i in sample:
            mesh = Mesh.new((int(n[i]), 1, 1), (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), ng=6)
            uu = np.zeros((mesh.len(), 5))
            mesh.interior(uu)[...] = u[offs[i]:offs[i + 1]].reshape(int(n[i]), 1, 1, 5)
            o = O.OracleSolver(sys_, mesh, uu, bc=bc, mode=FluxMode.Weno)
            dts = []
            while o.t < 0.15 - 1e-10 * 0.15:
                dts.append(min(o.dt_cfl(), 0.15 - o.t))
                o.step(dts[-1])
            x = (np.arange(n[i]) + 0.5) * dx[i]
            left = x < 0.5
            wp = np.zeros((mesh.len(), 5))
            wi = mesh.interior(wp).reshape(int(n[i]), 5)
            wi[:, 0] = np.where(left, st[i, 0], st[i, 3])
            wi[:, 1] = np.where(left, st[i, 1], st[i, 4])
            wi[:, 4] = np.where(left, st[i, 2], st[i, 5])
            mesh.interior(wp)[...] = wi.reshape(int(n[i]), 1, 1, 5)
            for q, (side, field) in enumerate([(True, 0), (True, 1), (True, 4), (False, 0), (False, 1), (False, 4)]):
                dw = np.zeros_like(wp)
                sel = left if side else ~left
                mesh.interior(dw)[sel.reshape(-1, 1, 1), field] = 1.0
                _, dJ = O.dual_run(sys_, mesh, wp, dw, 0.0, dts, OBJ_ENERGY, [0.5, 0, 0], [1.0, 0, 0], bc)
                worst = max(worst, abs(grad[i, q] - dJ) / max(abs(dJ), 1e-12))
        check = {"instances": sample, "max_rel_err_vs_dual": worst,
                 "what": "CPU f64 forward-mode dual-number runs of the oracle, 6 directions per instance, same time steps"}
    line = {
        "metric": "adjoint/forward cost", "value": (r + v) / f, "unit": "ratio", "n_gpus": world,
        "steps": steps, "warmup": warmup, "ms_per_step": f + r + v, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32-flux/f64-state" if prec == Precision.Mixed else "f64", "data": "synthetic",
        "config": {"workload": "4096 independent 1-D Riemann problems, cells log-uniform [64, 2048] (sum %d), "
                               "rho,p~U[0.1,2], u~U[-1,1], t_end 0.15, outflow; J_i = sum E dx over [0.5, 1]; "
                               "gradient w.r.t. the six initial values" % int(n.sum()),
                   "batch_steps": int(B), "checkpoints": "every 64 batch steps",
                   "step": "one recorded FP64 run + one backward pass"},
        "forward_ms": f, "recompute_ms": r, "reverse_ms": v, "reverse_over_forward": v / f,
        "forward_cell_updates_per_s": updates / (f * 1e-3),
        "gradient_sample": {"instance0": [float(x) for x in grad[0]], "J0": float(J[0])},
        "dual_check": check,
        "clocks": clk.summary(),
    }
    return line


def main():
    args = parse()
    world, rank, local = dist_init(args)
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        elif args.workload == "amr":
            run_amr(args, world, rank, local)
        elif args.workload == "batch":
            run_batch(args, world, rank, local)
        elif args.workload == "adjoint":
            run_adjoint(args, world, rank, local)
        elif args.workload == "batch_adjoint":
            run_batch_adjoint(args, world, rank, local)
        elif args.workload == "five":
            run_five(args, world, rank, local)
        else:
            run_ours(args, world, rank, local)
    finally:
        replicas.finish(world)


if __name__ == "__main__":
    main()
