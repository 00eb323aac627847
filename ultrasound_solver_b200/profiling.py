"""Small, self-terminating workloads for profiler captures.

    python -m ultrasound_solver_b200.profiling cycle --grid 128 --restart 112 --precision mixed
    python -m ultrasound_solver_b200.profiling cycle --grid 128 --restart 36 --recycle 8 \
        --recycle-every 2 --cycles 4 --precision bf16 --batch 4
    python -m ultrasound_solver_b200.profiling stencil --grid 128

`cycle` runs `--cycles` GMRES restart cycles (no CUDA graph, so every kernel
is a separate launch) on the config-1 scene. Plain GMRES(m): skipping 2*j
launches of k_dots|k_orth lands on Arnoldi step j of the first cycle. With
--recycle k the first two cycles are plain and every later cycle launches
k_dots|k_orth 2(m+1) times (the projection pair, then steps j = 0..m-1, the
steps j < k returning at once): skipping 2(m+1)c + 2 + 2j lands on step j of
cycle c >= 2. One launch covers all --batch right-hand sides (random
transducer phases, as in the bench). `stencil` applies the K and A operators
a few times (to --batch vectors in one launch). Both exit 0 without converging anything.
"""
from __future__ import annotations

import argparse

import numpy as np
import torch

from . import _native as N
from . import workloads as W


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=("cycle", "stencil"))
    ap.add_argument("--grid", type=int, default=128)
    ap.add_argument("--restart", type=int, default=112)
    ap.add_argument("--precision", default="mixed")
    ap.add_argument("--recycle", type=int, default=0)
    ap.add_argument("--recycle-every", type=int, default=1)
    ap.add_argument("--cycles", type=int, default=1)
    ap.add_argument("--batch", type=int, default=1)
    args = ap.parse_args(argv)
    torch.cuda.set_device(0)
    solver = W.build_solver(W.config1(n=args.grid), seed=0)
    solver.assemble_matrix()
    rng = np.random.default_rng(1)
    cols = []
    for _ in range(args.batch):
        solver.set_phases(rng.uniform(0, 2 * np.pi, solver.transducers.num_transducers))
        cols.append(solver.update_rhs_device())
    rhs = cols[0] if args.batch == 1 else torch.stack(cols)
    if args.what == "cycle":
        it = solver.iterative_solver
        it.precision, it.restart = args.precision, args.restart
        it.recycle, it.recycle_every = args.recycle, args.recycle_every
        plain = min(args.cycles, 2) if args.recycle else args.cycles
        it.maxiter = plain * args.restart + (args.cycles - plain) * (args.restart - args.recycle)
        it.rtol, it.use_graph = 1e-12, False
        it.solve(solver.operator, rhs, raise_on_failure=False)
        print("cycle", it.last_stats[0])
    else:
        op = solver.operator
        x64 = torch.randn((args.batch, op.n) if args.batch > 1 else op.n, dtype=torch.complex128,
                          device="cuda")
        for _ in range(3):
            op.apply(x64.to(torch.complex64), N.APPLY_K, N.PREC_MIXED)
            op.apply(x64, N.APPLY_K, N.PREC_FP64)
            op.apply(x64, N.APPLY_A, N.PREC_FP64)
        print("stencil ok")
    torch.cuda.synchronize()


if __name__ == "__main__":
    main()
