"""Config-4 workload: full phase optimisation at scale.

    python -m ultrasound_solver_b200.config4 [--grid 256] [--h 0.8e-3] [--steps 50]
                                             [--fp64-steps 1] [--out result.json]

256^3 nodes at h = 0.8 mm (16.8 M nodes), config-1 medium statistics, a
randomly rotated rigid ellipsoid (semi-axes 45 x 20 x 10 mm, an SDF blended
into the medium), +x reflecting, -y impedance Z = 2 rho c, a 16 x 16 array
and two focal-pressure targets. `--steps` Adam updates (lr 0.05) of the 256
phases, each evaluation a mixed-precision forward solve plus an A^H solve
(adjoint_optimizer.adam). The comparator runs the same evaluations with
plain FP64 GMRES(30) for `--fp64-steps` steps (a full FP64 loop of 50 steps
takes hours), and both report gradient steps/s. The first evaluation of both
arms is at the same phases, and their gradients are compared. Prints one
JSON line (synthetic inputs).
"""
from __future__ import annotations

import argparse
import json

import numpy as np
import torch

from . import workloads as W
from .adjoint_optimizer import adam, evaluate
from .losses import FocalPressureLoss


def build(args):
    cfg = W.config4(args.grid, args.h, args.array)
    solver = W.build_solver(cfg, seed=0, sdf=W.config4_sdf(cfg))
    solver.assemble_matrix()
    solver.iterative_solver.backward_error_tol = 1e-4
    return cfg, solver


def configure(it, precision, args):
    it.precision, it.rtol, it.maxiter = precision, args.rtol, args.maxiter
    if precision == "fp64":
        it.restart, it.recycle = 30, 0
    else:
        it.restart, it.recycle, it.recycle_every = args.restart, args.recycle, args.recycle_every


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--grid", type=int, default=256)
    ap.add_argument("--h", type=float, default=0.8e-3)
    ap.add_argument("--array", type=int, default=16)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--lr", type=float, default=0.05)
    ap.add_argument("--fp64-steps", type=int, default=1)
    ap.add_argument("--precision", default="bf16")
    ap.add_argument("--restart", type=int, default=36)
    ap.add_argument("--recycle", type=int, default=8)
    ap.add_argument("--recycle-every", type=int, default=2)
    ap.add_argument("--rtol", type=float, default=1e-8)
    ap.add_argument("--maxiter", type=int, default=400000)
    ap.add_argument("--out", default="")
    args = ap.parse_args(argv)
    torch.cuda.set_device(0)
    cfg, solver = build(args)
    loss = FocalPressureLoss(solver.cfg)
    it = solver.iterative_solver
    phases0 = np.random.default_rng(1).uniform(0, 2 * np.pi, solver.transducers.num_transducers)

    configure(it, args.precision, args)
    mixed = adam(solver, loss, phases0, args.steps, args.lr)
    out = {"workload": (f"config-4: {args.grid}^3 at h={args.h * 1e3:g} mm, random medium, "
                        "rotated ellipsoid (SDF), +x reflecting, -y impedance 2 rho c, "
                        f"{args.array}x{args.array} array, focal_pressure at 2 targets"),
           "nodes": args.grid ** 3, "adam_steps": mixed.steps, "lr": args.lr,
           "solver": f"{args.precision} GCRO-DR({args.restart},{args.recycle}), rtol {args.rtol:g}",
           "mixed": {"grad_steps_per_s": len(mixed.seconds) / sum(mixed.seconds),
                     "seconds_per_step": float(np.mean(mixed.seconds)),
                     "inner_iterations_per_solve_last": mixed.iterations[-1],
                     "loss_first": mixed.losses[0], "loss_last": mixed.losses[-1],
                     "loss_best": mixed.best_loss, "losses": mixed.losses},
           "data": "synthetic"}
    if args.fp64_steps > 0:
        g_mixed = evaluate(solver, loss, phases0).gradient
        configure(it, "fp64", args)
        fp = adam(solver, loss, phases0, args.fp64_steps - 1, args.lr) if args.fp64_steps > 1 \
            else None
        first = evaluate(solver, loss, phases0)
        secs = ([first.seconds] + (fp.seconds if fp else []))
        out["fp64_gmres"] = {"solver": "plain FP64 GMRES(30)", "evaluations": len(secs),
                             "grad_steps_per_s": len(secs) / sum(secs),
                             "seconds_per_step": float(np.mean(secs))}
        out["speedup_mixed_vs_fp64"] = out["mixed"]["grad_steps_per_s"] / \
            out["fp64_gmres"]["grad_steps_per_s"]
        out["grad_rel_err_vs_fp64"] = float(np.linalg.norm(g_mixed - first.gradient) /
                                            np.linalg.norm(first.gradient))
    line = json.dumps(out)
    print(line)
    if args.out:
        with open(args.out, "w") as f:
            f.write(line + "\n")


if __name__ == "__main__":
    main()
