"""Config-2 workload: batched response basis + a batch of uneven-grid scenes.

    python -m ultrasound_solver_b200.config2 [--columns 256] [--scenes 32] [--no-tune]

Part 1 builds the phase-response basis columns G[:, j] = A^-1 B e_j of one
96^3 scene with a 16x16 array (config-1 medium statistics), all columns
through batched GMRES launches whose width and Arnoldi kernel forms the
BatchTuner picks. Part 2 solves `--scenes` independent scenes whose grid
edges are drawn from {48, 64, 80, 96, 112} (random sphere obstacle, 8x8
array, seeded phases) three ways: all in one batched launch sequence
(scene_batch.solve_scenes_batched), concurrently on one stream per scene
(scene_batch.solve_scenes) and one after the other. `--restart 20
--recycle 0` runs the configuration's plain GMRES(20). Prints one JSON line
(synthetic inputs).
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch

from . import workloads as W
from .autotune import BatchTuner
from .scene_batch import solve_scenes, solve_scenes_batched


def _configure(solver, args):
    it = solver.iterative_solver
    it.precision, it.restart, it.recycle = args.precision, args.restart, args.recycle
    it.recycle_every, it.rtol, it.maxiter = args.recycle_every, args.rtol, args.maxiter
    return it


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--grid", type=int, default=96)
    ap.add_argument("--columns", type=int, default=256)
    ap.add_argument("--scenes", type=int, default=32)
    ap.add_argument("--precision", default="bf16")
    ap.add_argument("--restart", type=int, default=36)
    ap.add_argument("--recycle", type=int, default=8)
    ap.add_argument("--recycle-every", type=int, default=2)
    ap.add_argument("--rtol", type=float, default=1e-9)
    ap.add_argument("--maxiter", type=int, default=80000)
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--batch-width", type=int, default=0)
    ap.add_argument("--tune-cache", default=None)
    args = ap.parse_args(argv)
    torch.cuda.set_device(0)
    out = {"workload": "config-2", "precision": args.precision,
           "solver": f"GCRO-DR({args.restart},{args.recycle})" if args.recycle
           else f"GMRES({args.restart})", "rtol": args.rtol, "data": "synthetic"}

    # part 1: response basis of one scene
    if args.columns > 0:
        s = W.build_solver(W.config2_basis_scene(args.grid), seed=0)
        s.assemble_matrix()
        it = _configure(s, args)
        cols = s.sources.column_rhs(s.transducers.amplitudes, 0,
                                    min(args.columns, s.transducers.num_transducers))
        if args.batch_width:
            it.batch_width = args.batch_width
        elif not args.no_tune:
            BatchTuner(cache_path=args.tune_cache).tune(it, s.operator, cols)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        x = s.solve_rhs_device(cols)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        out["basis"] = {"grid": args.grid, "columns": int(cols.shape[0]),
                        "batch_width": it.batch_width, "seconds": dt,
                        "rhs_solves_per_s": cols.shape[0] / dt,
                        "max_iterations": it.last_iterations,
                        "max_scaled_residual": it.last_scaled_residual}
        del x, cols, s
        torch.cuda.empty_cache()

    # part 2: uneven scenes, concurrent vs one after the other
    if args.scenes > 0:
        cfgs = W.config2_scene_batch(args.scenes, seed=3)
        solvers, rhs = [], []
        for i, c in enumerate(cfgs):
            s = W.build_solver(c, seed=100 + i)
            s.assemble_matrix()
            _configure(s, args)
            solvers.append(s)
            rhs.append(s.update_rhs_device())
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        xs = solve_scenes(solvers, rhs)
        torch.cuda.synchronize()
        t_conc = time.perf_counter() - t0
        t0 = time.perf_counter()
        xs_seq = [s.solve_rhs_device(r) for s, r in zip(solvers, rhs)]
        torch.cuda.synchronize()
        t_seq = time.perf_counter() - t0
        # every scene in ONE batched launch sequence (usv_gmres_solve_scenes)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        xs_one = solve_scenes_batched(solvers, rhs)
        torch.cuda.synchronize()
        t_one = time.perf_counter() - t0

        def maxdiff(a_list, b_list):
            return max(float((torch.linalg.norm(a - b) / torch.linalg.norm(b)).item())
                       for a, b in zip(a_list, b_list))
        sizes = [int(c["domain"]["grid_size"][0]) for c in cfgs]
        out["scene_batch"] = {"scenes": len(cfgs), "grid_edges": sizes,
                              "nodes": int(sum(n ** 3 for n in sizes)),
                              "one_launch_seconds": t_one,
                              "concurrent_seconds": t_conc, "sequential_seconds": t_seq,
                              "rhs_solves_per_s": len(cfgs) / min(t_one, t_conc),
                              "speedup_one_launch": t_seq / t_one,
                              "speedup_concurrent": t_seq / t_conc,
                              "max_rel_diff_one_launch_vs_sequential": maxdiff(xs_one, xs_seq),
                              "max_rel_diff_concurrent_vs_sequential": maxdiff(xs, xs_seq)}
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
