#!/usr/bin/env python
"""RHS solves/s of the gpu_iterative Helmholtz path on B200.

Workload (one "step" = one batch of `--batch` right-hand sides, each solved to
the scaled relative residual rtol): the 128^3 variable-medium scene at
h = 1 mm, 40 kHz, seeded Gaussian random c and rho (sigma = 4 cells, +-3
clip), a rho=1250/c=2200 blended sphere of radius 15 mm 60 mm above the
baffle, +x reflecting wall, 10-cell quadratic PML on the other open faces,
8 x 8 sinc_neumann array (radius 4.5 mm, pitch 10.5 mm), seeded phases (one
phase vector per right-hand side). Inputs are synthetic.

Our arm: mixed-precision batched solves on the matrix-free sm_100a stencil:
bfloat16 Krylov vectors (fp32 stencil, FP64 dots, Hessenberg/Givens, FP64
true residual and solution update at every restart) with deflated restarting
(GCRO-DR(32, 8): 8 harmonic Ritz vectors recycled across restarts, refreshed
every cycle). Two FP64
comparators run once beside it on the same batch of right-hand sides, one
launch each: plain FP64 GMRES(30) of the same stencil (the reference's
algorithm in FP64; `speedup_vs_plain_fp64`) and FP64 GCRO-DR(32, 8) (the same
algorithm as our arm; `speedup_precision_only`). The relative L2 difference
between the mixed and the FP64 GMRES fields is the metric's accuracy bar: above
1e-6 the line carries no `value` and the run exits non-zero. `--impl reference` times
the reference's CPU algorithm (the oracle's restatement: CSR assembly +
row-scaled Jacobi GMRES(30) in scipy/numpy) on the host cores.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "RHS solves/s at 128^3 (config-1 scene), mixed-precision GMRES, rel err <=1e-6 vs FP64"
# the reference's algorithm: row-scaled Jacobi GMRES(30)
REFERENCE_RESTART = 30
UNIT = "RHS solves/s"
FALLBACK_HBM_GBS = 6650.0
# Inner iterations the row-scaled Jacobi GMRES(30) needs on the 128^3 scene
# to reach rtol 1e-9: 53,310, measured by this bench's plain FP64 arm on a
# B200 (complex128 Krylov vectors, the reference's algorithm). A full CPU
# solve takes hours, so the CPU legs time bounded samples of Arnoldi steps and
# convert it/s to solves/s with this count; our own arm uses the count its FP64
# arm measures in the same run instead.
ITERATIONS_PER_SOLVE_FP64 = 53310
ITERATIONS_PROVENANCE = ("53,310 inner iterations: plain FP64 GMRES(30) of this bench to "
                         "rtol 1e-9 on the 128^3 scene, measured on a B200")
# the metric's accuracy bar: relative L2 error of the mixed-precision field
# against the FP64 solve of the same right-hand side
PARITY_BAR = 1e-6
# DRAM bytes / algorithmic bytes of the Arnoldi kernels from one ncu capture
# (profiles/arnoldi_kdots_korth_128cube_gcrodr36_8_bf16_b4_j24.md); the
# roofline's `traffic` is the algorithmic bytes per launch scaled by it.
TRAFFIC_RATIO = {"arnoldi_dots": 1.03, "arnoldi_orth": 1.00}


def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--grid", type=int, default=128)
    ap.add_argument("--restart", type=int, default=32)
    ap.add_argument("--recycle", type=int, default=8,
                    help="harmonic Ritz vectors recycled across restarts (0: plain GMRES)")
    ap.add_argument("--recycle-every", type=int, default=1)
    ap.add_argument("--precision", default="bf16", choices=("bf16", "mixed"))
    ap.add_argument("--batch", type=int, default=4, help="right-hand sides per step")
    ap.add_argument("--fp64-restart", type=int, default=REFERENCE_RESTART)
    ap.add_argument("--rtol", type=float, default=1e-9)
    ap.add_argument("--maxiter", type=int, default=80000)
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 GMRES comparator")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint-gradient timing")
    ap.add_argument("--no-stencil", action="store_true", help="skip the stencil-only timing")
    ap.add_argument("--cpu-iters", type=int, default=20)
    ap.add_argument("--kernel-variant", type=int, default=0,
                    help="usv_gmres_params.kernel_variant bits (0: the default kernel forms)")
    ap.add_argument("--capture", choices=("cycle", "stencil"), default=None,
                    help="run a short self-terminating workload for a profiler capture "
                         "(no bench line): `cycle` = --cycles restart cycles without CUDA "
                         "graphs, `stencil` = a few operator applies")
    ap.add_argument("--cycles", type=int, default=4)
    return ap.parse_args(argv)


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        try:
            return float(json.loads(path.read_text())["hbm_gbs"]), "measured"
        except (KeyError, ValueError):
            pass
    return FALLBACK_HBM_GBS, "fallback"


# ---------------------------------------------------------------- distributed
def dist_setup(n_gpus):
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900),
                                device_id=torch.device("cuda", local))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(value, world):
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(world, steps, batch, ms_max):
    """Whole-job RHS solves/s: every rank solves `steps` batches of `batch`
    independent right-hand sides (replicas), timed by the slowest rank."""
    return world * steps * batch / (ms_max / 1000.0)


def replica_seed(rank):
    """Seed of a rank's phase vectors: distinct right-hand sides per replica."""
    return 1 + rank


# ---------------------------------------------------------------- workload
def workload_config(args):
    from ultrasound_solver_b200 import workloads as W
    cfg = W.config1(n=args.grid)
    vb = 4 if args.precision == "bf16" else 8
    desc = {"workload": f"config-1 scene: {args.grid}^3 nodes h=1mm 40kHz, random c/rho "
                        "(sigma 4 cells), r=15mm rho=1250 sphere blended, +x reflecting, "
                        f"10-cell quadratic PML, 8x8 sinc_neumann array, {args.batch} RHS "
                        "(seeded phase vectors) per step",
            "grid": [args.grid] * 3, "nodes": args.grid ** 3, "rhs_per_step": args.batch,
            "solver": (f"GCRO-DR({args.restart},{args.recycle}) deflated restarting, "
                       f"recycled space refreshed every {args.recycle_every} cycles"
                       if args.recycle else f"GMRES({args.restart})"),
            "restart": args.restart, "recycle": args.recycle, "rtol": args.rtol,
            "precision": ("bfloat16" if args.precision == "bf16" else "complex64")
                         + " Krylov vectors, FP64 dots/Hessenberg + FP64 refinement",
            "fp64_comparator": (f"plain FP64 GMRES({args.fp64_restart}) and FP64 "
                                f"GCRO-DR({args.restart},{args.recycle}), the same {args.batch} "
                                "RHS per launch"),
            "l2": "inputs larger than L2 (Krylov basis %.1f GB per RHS)" % (
                2 * (args.restart + 1) * args.grid ** 3 * vb / 1e9),
            "parallelism": "replicas (independent RHS batches per GPU)"}
    return cfg, desc


def run_ours(args):
    import torch

    from ultrasound_solver_b200 import workloads as W

    rank, world, local = dist_setup(args.gpus)
    cfg, desc = workload_config(args)
    solver = W.build_solver(cfg, seed=0)
    rng = np.random.default_rng(replica_seed(rank))
    solver.assemble_matrix()
    rhs_list = []
    for _ in range(args.batch):
        solver.set_phases(rng.uniform(0, 2 * np.pi, solver.transducers.num_transducers))
        rhs_list.append(solver.update_rhs_device())
    rhs = torch.stack(rhs_list)
    it = solver.iterative_solver
    it.rtol, it.maxiter = args.rtol, args.maxiter
    it.backward_error_tol = 1e-4
    it.kernel_variant = args.kernel_variant
    stream = torch.cuda.current_stream()

    def configure(precision, profile=False, its=None):
        its = it if its is None else its
        its.precision, its.profile = precision, profile
        if precision == "fp64":
            its.restart, its.recycle = args.fp64_restart, 0
        else:
            its.restart, its.recycle, its.recycle_every = args.restart, args.recycle, args.recycle_every

    def solve(precision, profile=False, b=None):
        configure(precision, profile)
        return it.solve(solver.operator, rhs if b is None else b)

    # warm-up (untimed)
    for _ in range(args.warmup):
        x_mixed = solve(args.precision)
    torch.cuda.synchronize()
    # timed region: K solves from device-resident inputs
    barrier(world)
    torch.cuda.synchronize()
    prof_tot = {}
    launches = 0
    iterations = []
    cycles = []
    with ClockSampler(local) as clocks:
        start = torch.cuda.Event(enable_timing=True)
        stop = torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for _ in range(args.steps):
            x_mixed = solve(args.precision, profile=True)
            iterations.append(it.last_iterations)
            cycles.append(max(st["cycles"] for st in it.last_stats))
            for name, d in it.last_profile.items():
                agg = prof_tot.setdefault(name, dict(launches=0, ms=0.0, bytes=0.0))
                for k in agg:
                    agg[k] += d[k]
            # measured intervals + the second kernel of each projection interval
            # (one per recycled cycle: half of the recycle_dots intervals)
            launches += sum(d["launches"] for d in it.last_profile.values())
            launches += it.last_profile.get("recycle_dots", {}).get("launches", 0) // 2
        stop.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    ms_local = start.elapsed_time(stop)
    ms = max_over_ranks(ms_local, world)
    value = job_throughput(world, args.steps, args.batch, ms)
    stats = dict(it.last_stats[0])

    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": ("bf16" if args.precision == "bf16" else "c64") + "+f64",
           "data": "synthetic", "config": desc,
           "iterations_per_solve": iterations, "scaled_residual": stats["scaled_residual"],
           "backward_error": stats["backward_error"]}
    out["clocks"] = clocks.summary()
    out["gpu_launches"] = launches
    # time between the measured kernel intervals: one graph launch and one
    # status read-back per restart cycle (the cycles are not one persistent
    # launch), plus the final gates and the stats read
    kernel_ms = sum(v["ms"] for v in prof_tot.values())
    out["cycle_gaps"] = {"ms_per_step": (ms_local - kernel_ms) / args.steps,
                         "fraction_of_step": (ms_local - kernel_ms) / ms_local,
                         "restart_cycles_per_step": statistics.mean(cycles),
                         "us_per_cycle": 1000.0 * (ms_local - kernel_ms) / max(sum(cycles), 1)}

    # roofline of the dominant kernel family (live CUDA-event timing)
    peak, peak_kind = measured_peak()
    dom = max(prof_tot, key=lambda k: prof_tot[k]["ms"])
    d = prof_tot[dom]
    achieved = d["bytes"] / (d["ms"] / 1000.0) / 1e9 if d["ms"] > 0 else None
    out["roofline"] = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                       "peak_source": peak_kind, "unit": "GB/s",
                       "frac": achieved / peak if achieved else None,
                       "traffic": (d["bytes"] / max(d["launches"], 1) * TRAFFIC_RATIO[dom]
                                   if dom in TRAFFIC_RATIO else None),
                       "traffic_unit": "bytes per launch (ncu DRAM read+write)",
                       "avg_launch_us": 1000.0 * d["ms"] / max(d["launches"], 1),
                       "algorithmic_bytes_per_launch": d["bytes"] / max(d["launches"], 1),
                       "families": {k: {"launches": v["launches"], "ms": v["ms"],
                                        "GBps": (v["bytes"] / (v["ms"] / 1e3) / 1e9)
                                        if v["ms"] > 0 and v["bytes"] > 0 else None}
                                    for k, v in prof_tot.items()}}

    # the stencil alone: usv_operator_apply_kernel of the complex64 K rows (both
    # kernels: precomputed row coefficients, 48 B per node; 16-byte node
    # records with the rows formed in registers) and of the FP64 A rows on the
    # batch, launches timed with CUDA events after an L2 flush; algorithmic
    # bytes per launch: the per-node operator data the kernel reads once plus x
    # and y of every RHS
    if not args.no_stencil:
        from ultrasound_solver_b200 import _native as N
        op = solver.operator
        flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
        nn = op.n

        import ctypes

        def time_apply(x, variant, precision, kernel=N.STENCIL_AUTO, reps=20):
            # back-to-back launches through the C-ABI (the batch's operator data
            # and vectors exceed the 126 MB L2), after an L2 flush
            y = torch.empty_like(x)
            lib, sh = N.load(), N.stream_handle(torch, x.device)

            def launch():
                N.check(lib.usv_operator_apply_kernel(ctypes.byref(op.scene), N.ptr(op.buffer),
                                                      variant, precision, kernel, N.ptr(x), N.ptr(y),
                                                      x.shape[0], op.n, sh), "apply")
            for _ in range(3):
                launch()
            flush.fill_(1)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(reps):
                launch()
            e1.record(stream)
            torch.cuda.synchronize()
            return max_over_ranks(e0.elapsed_time(e1) / reps, world)

        x64 = rhs.to(torch.complex64).contiguous()
        peak, peak_kind = measured_peak()
        compulsory = nn * (16.0 + args.batch * 16.0)
        kernels = {"k_apply_kc_rhs (complex64 row coefficients, 48 B per node)":
                   (N.STENCIL_COEF_ROWS, nn * (48.0 + args.batch * 16.0))}
        if args.batch <= 4:
            kernels["k_apply_rec25 (16-byte node records, z-marching tiles)"] = (
                N.STENCIL_RECORD_TILES, nn * (16.0 + args.batch * 16.0))
        variants = {}
        for name, (kern, nbytes) in kernels.items():
            ms_k = time_apply(x64, N.APPLY_K, N.PREC_MIXED, kern)
            variants[name] = {"us_per_launch": 1000.0 * ms_k, "bytes_per_launch": nbytes,
                              "achieved": nbytes / (ms_k / 1e3) / 1e9,
                              "frac": nbytes / (ms_k / 1e3) / 1e9 / peak,
                              "compulsory_frac": compulsory / (ms_k / 1e3) / 1e9 / peak}
        best = min(variants, key=lambda k: variants[k]["us_per_launch"])
        ms_a = time_apply(rhs.contiguous(), N.APPLY_A, N.PREC_FP64)
        bytes_a = nn * (112.0 + args.batch * 32.0)
        b = variants[best]
        out["stencil"] = {
            "kernel": f"{best}, {args.batch} RHS per launch",
            "achieved": b["achieved"], "unit": "GB/s", "peak": peak, "peak_source": peak_kind,
            "frac": b["frac"], "us_per_launch": b["us_per_launch"],
            "bytes_per_launch": b["bytes_per_launch"],
            "l2": "inputs larger than L2 (20 launches back to back)",
            # compulsory traffic of a 16-byte-per-node operator record plus x
            # and y of every RHS, against the same time
            "compulsory_bytes_per_launch": compulsory, "compulsory_frac": b["compulsory_frac"],
            "kernels": variants,
            "fp64_A": {"kernel": f"k_apply_fp64 (complex128 A rows), {args.batch} RHS per launch",
                       "achieved": bytes_a / (ms_a / 1e3) / 1e9,
                       "frac": bytes_a / (ms_a / 1e3) / 1e9 / peak,
                       "us_per_launch": 1000.0 * ms_a, "bytes_per_launch": bytes_a}}
        del flush

    # FP64 comparators on the same batch: plain GMRES(30) (the reference's
    # algorithm in complex128) and GCRO-DR with our arm's (m, k) in complex128,
    # each one launch of args.batch RHS; parity of every field of the batch
    fp64_iters = None
    parity_ok = True
    if not args.no_fp64:
        def timed_fp64(restart, recycle):
            configure("fp64")
            it.restart, it.recycle, it.recycle_every = restart, recycle, args.recycle_every
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            x = it.solve(solver.operator, rhs)
            e1.record(stream)
            torch.cuda.synchronize()
            ms_ = max_over_ranks(e0.elapsed_time(e1), world)
            return x, ms_, [s_["iterations"] for s_ in it.last_stats]

        x64, ms64, its64 = timed_fp64(args.fp64_restart, 0)
        fp64_iters = statistics.mean(its64)
        per_rhs = [float((torch.linalg.norm(x_mixed[b] - x64[b]) / torch.linalg.norm(x64[b])).item())
                   for b in range(args.batch)]
        rel = max(per_rhs)
        v64 = world * args.batch / (ms64 / 1000.0)
        out["fp64_gmres"] = {"solves_per_s": v64, "ms_per_batch": ms64, "rhs_per_launch": args.batch,
                             "iterations": its64, "restart": args.fp64_restart,
                             "speedup_vs_plain_fp64": value / v64}
        out["rel_err_vs_fp64"] = rel
        out["rel_err_vs_fp64_per_rhs"] = per_rhs
        if args.recycle:
            xr, msr, itsr = timed_fp64(args.restart, args.recycle)
            vr = world * args.batch / (msr / 1000.0)
            out["fp64_gcrodr"] = {"solves_per_s": vr, "ms_per_batch": msr,
                                  "rhs_per_launch": args.batch, "iterations": itsr,
                                  "restart": args.restart, "recycle": args.recycle,
                                  "recycle_every": args.recycle_every,
                                  "speedup_precision_only": value / vr,
                                  "rel_err_vs_fp64_gmres": max(
                                      float((torch.linalg.norm(xr[b] - x64[b]) /
                                             torch.linalg.norm(x64[b])).item())
                                      for b in range(args.batch))}
        parity_ok = rel <= PARITY_BAR
        out["parity"] = {"bar": PARITY_BAR, "ok": parity_ok,
                         "against": f"FP64 GMRES({args.fp64_restart}) solutions of the same batch"}
        if not parity_ok:
            # an inaccurate mixed solve has no throughput under this metric
            out["value"] = None
        configure(args.precision)

    # end to end through the public API with host buffers
    if not args.no_e2e:
        configure(args.precision)
        rhs_host = np.ascontiguousarray(rhs.cpu().numpy().T)  # (N, B), the reference's layout
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        n_e2e = 1
        for _ in range(n_e2e):
            xh = solver.solve_rhs(rhs_host, verbose=False)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        e2e = max_over_ranks(dt, world)
        out["e2e"] = {"value": world * n_e2e * args.batch / e2e, "unit": UNIT,
                      "h2d_bytes_per_step": int(rhs_host.nbytes),
                      "d2h_bytes_per_step": int(xh.nbytes), "steps": n_e2e,
                      "api": "HelmholtzB200Solver.solve_rhs(numpy)"}

    # adjoint gradient: forward solve + A^H solve + phase VJP behind torch.autograd,
    # in the mixed path and (unless --no-fp64) with the plain FP64 GMRES
    # on the adjoint workload's scene: the same medium with a 16x16 array
    if not args.no_adjoint:
        from ultrasound_solver_b200.autograd import loss_of_field, phase_field
        from ultrasound_solver_b200.losses import ContrastRatioLoss
        asolver = W.build_solver(W.config3(n=args.grid), seed=0)
        asolver.assemble_matrix()
        asolver.set_phases(rng.uniform(0, 2 * np.pi, asolver.transducers.num_transducers))
        ait = asolver.iterative_solver
        ait.rtol, ait.maxiter, ait.backward_error_tol = args.rtol, args.maxiter, 1e-4
        centre = (args.grid - 1) * asolver.cfg.domain.dx / 2
        loss = ContrastRatioLoss(asolver.cfg, (centre, centre, 0.080), 0.006, 0.010)

        def grad_once(precision):
            configure(precision, its=ait)
            ph = torch.tensor(asolver.transducers.phases, dtype=torch.float64, device="cuda",
                              requires_grad=True)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            L = loss_of_field(phase_field(ph, asolver), loss)
            L.backward()
            e1.record(stream)
            torch.cuda.synchronize()
            return max_over_ranks(e0.elapsed_time(e1), world), ph.grad.detach().clone()

        ms_grad, grad = grad_once(args.precision)
        out["adjoint_grad"] = {"value": world * 1000.0 / ms_grad, "unit": "adjoint grads/s",
                               "ms_per_grad": ms_grad,
                               "scene": f"{args.grid}^3 random medium and sphere as above with a "
                                        f"{asolver.transducers.num_transducers}-element (16x16) array",
                               "loss": "-|u_t|^2 / mean_shell |u|^2 (target 80 mm above the array)",
                               "grad_norm": float(torch.linalg.norm(grad).item())}
        if not args.no_fp64:
            ms64g, grad64 = grad_once("fp64")
            out["adjoint_grad"]["fp64_grads_per_s"] = world * 1000.0 / ms64g
            out["adjoint_grad"]["speedup_mixed_vs_fp64"] = ms64g / ms_grad
            out["adjoint_grad"]["rel_err_vs_fp64"] = float(
                (torch.linalg.norm(grad - grad64) / torch.linalg.norm(grad64)).item())

    if rank == 0 and world == 1 and not args.no_cpu:
        out["cpu_baseline"] = cpu_sample(args, cfg, fp64_iters)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if not parity_ok:
        sys.exit(f"mixed-precision field error {out['rel_err_vs_fp64']:.3e} exceeds {PARITY_BAR:g}")


# ---------------------------------------------------------------- CPU side
def cpu_scene(args, cfg):
    """The same scene assembled by the oracle's restatement of the reference."""
    from oracle import helmholtz_oracle as O
    from ultrasound_solver_b200 import workloads as W
    n = args.grid
    shape = (n,) * 3
    dx = cfg["domain"]["box_size"][0] / (n - 1)
    rho_m, c_m = W.random_medium(shape, 0)
    ob = cfg["obstacles"][0]
    h = O.smoothed_heaviside(O.sphere_sdf(shape, dx, ob["center"], ob["radius"]), 1.2 * dx)
    rho, c = O.blend_obstacle_material(h, 1250.0, 2200.0, rho_m, c_m)
    c2 = dict(cfg)
    c2["obstacles"] = []
    m = cfg["transducer_specs"]["array_n"] ** 2
    phases = np.random.default_rng(1).uniform(0, 2 * np.pi, m)
    return O.build_scene(c2, material_fields=(rho, c), phases=phases)


def cpu_iterations_per_second(args, sc, iters):
    """Time `iters` Arnoldi steps of the restated row-scaled Jacobi GMRES."""
    from oracle import helmholtz_oracle as O
    A = sc.A
    R, inv_d = O.row_scale_and_jacobi(A)
    b = R * sc.rhs
    m = min(args.fp64_restart, iters)
    t0 = time.perf_counter()
    # one truncated cycle of the restated algorithm: m steps of CGS Arnoldi
    r = b.copy()
    beta = np.linalg.norm(r)
    V = np.empty((len(b), m + 1), dtype=np.complex128)
    V[:, 0] = r / beta
    for j in range(m):
        u = R * (A @ (inv_d * V[:, j]))
        h = V[:, :j + 1].conj().T @ u
        u = u - V[:, :j + 1] @ h
        V[:, j + 1] = u / np.linalg.norm(u)
    dt = time.perf_counter() - t0
    return m / dt, m, dt


def blas_threads():
    try:
        from threadpoolctl import threadpool_info
        n = [i.get("num_threads", 1) for i in threadpool_info() if i.get("user_api") == "blas"]
        return max(n) if n else 1
    except Exception:
        return 1


def host_threads():
    """What the CPU legs run on: the box's cores, the cores this process may
    use (no pinning is applied) and the BLAS threads of the Gram-Schmidt
    products; the CSR SpMV of scipy is single-threaded."""
    try:
        allowed = len(os.sched_getaffinity(0))
    except (AttributeError, OSError):
        allowed = os.cpu_count()
    return {"nproc": os.cpu_count(), "allowed_cores": allowed, "blas_threads": blas_threads(),
            "pinning": "none (process affinity as launched)",
            "spmv_threads": 1}


def cpu_sample(args, cfg, fp64_iters=None):
    sc = cpu_scene(args, cfg)
    its, m, dt = cpu_iterations_per_second(args, sc, args.cpu_iters)
    per_solve = fp64_iters or ITERATIONS_PER_SOLVE_FP64
    return {"value": its / per_solve, "unit": UNIT, "cores": blas_threads(),
            "threads": host_threads(), "kind": "port",
            "iterations_per_solve_source": ("this run's FP64 GMRES arm" if fp64_iters
                                            else ITERATIONS_PROVENANCE),
            "sample": (f"{m} Arnoldi steps of the restated row-scaled Jacobi "
                       f"GMRES({args.fp64_restart}) on the {args.grid}^3 scene in {dt:.1f}s "
                       f"({its:.2f} it/s, scipy CSR SpMV single-threaded); solves/s = it/s / "
                       f"{per_solve} iterations per solve (GMRES({args.fp64_restart}) to "
                       f"rtol {args.rtol:g} on this scene)")}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cfg, desc = workload_config(args)
    sc = cpu_scene(args, cfg)
    for _ in range(args.warmup):
        cpu_iterations_per_second(args, sc, 4)
    t0 = time.perf_counter()
    total_it = 0
    for _ in range(args.steps):
        its, m, dt = cpu_iterations_per_second(args, sc, args.cpu_iters)
        total_it += m
    dt = time.perf_counter() - t0
    its = total_it / dt
    value = its / ITERATIONS_PER_SOLVE_FP64
    cores = blas_threads()
    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": 1000.0 * dt / args.steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
           "data": "synthetic", "config": desc, "impl": "reference",
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                            "threads": host_threads(),
                            "iterations_per_solve_source": ITERATIONS_PROVENANCE,
                            "sample": (f"{args.cpu_iters} Arnoldi steps per step of the restated "
                                       f"row-scaled Jacobi GMRES({args.fp64_restart}) (reference CPU "
                                       f"algorithm, CuPy gmres restated in numpy/scipy); "
                                       f"{its:.3f} it/s; solves/s = it/s / "
                                       f"{ITERATIONS_PER_SOLVE_FP64} iterations per solve")},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def run_capture(args):
    """Small workloads for ncu captures (one GPU, exit 0 without converging).

    `cycle`: --cycles restart cycles of the bench's solver configuration on
    the --batch right-hand sides, without CUDA graphs, so every kernel is a
    separate launch. Plain GMRES(m): skipping 2j launches of k_dots|k_orth
    lands on Arnoldi step j of the first cycle. With --recycle k the first two
    cycles are plain and every later cycle launches k_dots|k_orth 2(m+1) times
    (the projection pair, then steps j = 0..m-1; steps j < k return at once):
    skipping 2(m+1)c + 2 + 2j lands on step j of cycle c >= 2.
    `stencil`: three applies each of the complex64 K rows, the complex128 K
    rows and the FP64 A rows on --batch vectors.
    """
    import torch

    from ultrasound_solver_b200 import _native as N
    from ultrasound_solver_b200 import workloads as W
    torch.cuda.set_device(0)
    solver = W.build_solver(W.config1(n=args.grid), seed=0)
    solver.assemble_matrix()
    rng = np.random.default_rng(1)
    cols = []
    for _ in range(args.batch):
        solver.set_phases(rng.uniform(0, 2 * np.pi, solver.transducers.num_transducers))
        cols.append(solver.update_rhs_device())
    rhs = torch.stack(cols)
    if args.capture == "cycle":
        it = solver.iterative_solver
        it.precision, it.restart = args.precision, args.restart
        it.recycle, it.recycle_every = args.recycle, args.recycle_every
        it.kernel_variant = args.kernel_variant
        plain = min(args.cycles, 2) if args.recycle else args.cycles
        it.maxiter = plain * args.restart + (args.cycles - plain) * (args.restart - args.recycle)
        it.rtol, it.use_graph = 1e-12, False
        it.solve(solver.operator, rhs, raise_on_failure=False)
        print("capture cycle:", it.last_stats[0])
    else:
        op = solver.operator
        x64 = torch.randn((args.batch, op.n), dtype=torch.complex128, device="cuda")
        for _ in range(3):
            op.apply(x64.to(torch.complex64), N.APPLY_K, N.PREC_MIXED)
            op.apply(x64, N.APPLY_K, N.PREC_FP64)
            op.apply(x64, N.APPLY_A, N.PREC_FP64)
        print("capture stencil: ok")
    torch.cuda.synchronize()


def main(argv=None):
    args = parse_args(argv)
    if args.capture:
        run_capture(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
