"""Small, self-terminating workloads for profiler captures.

    python -m ultrasound_solver_b200.profiling cycle --grid 128 --restart 112 --precision mixed
    python -m ultrasound_solver_b200.profiling stencil --grid 128

`cycle` runs exactly one GMRES restart cycle (maxiter = restart, no CUDA
graph, so every kernel is a separate launch) on the config-1 scene; skipping
2*j launches of k_dots|k_orth lands on Arnoldi step j. `stencil` applies the
K and A operators a few times. Both exit 0 without converging anything.
"""
from __future__ import annotations

import argparse

import torch

from . import _native as N
from . import workloads as W


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=("cycle", "stencil"))
    ap.add_argument("--grid", type=int, default=128)
    ap.add_argument("--restart", type=int, default=112)
    ap.add_argument("--precision", default="mixed")
    args = ap.parse_args(argv)
    torch.cuda.set_device(0)
    solver = W.build_solver(W.config1(n=args.grid), seed=0)
    solver.assemble_matrix()
    rhs = solver.update_rhs_device()
    if args.what == "cycle":
        it = solver.iterative_solver
        it.precision, it.restart, it.maxiter = args.precision, args.restart, args.restart
        it.rtol, it.use_graph = 1e-12, False
        it.solve(solver.operator, rhs, raise_on_failure=False)
        print("cycle", it.last_stats[0])
    else:
        op = solver.operator
        x64 = torch.randn(op.n, dtype=torch.complex128, device="cuda")
        for _ in range(3):
            op.apply(x64.to(torch.complex64), N.APPLY_K, N.PREC_MIXED)
            op.apply(x64, N.APPLY_K, N.PREC_FP64)
            op.apply(x64, N.APPLY_A, N.PREC_FP64)
        print("stencil ok")
    torch.cuda.synchronize()


if __name__ == "__main__":
    main()
