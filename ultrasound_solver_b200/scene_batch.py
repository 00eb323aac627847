"""Concurrent solves of independent scenes (uneven grid sizes) on one GPU.

Each scene keeps its own operator, workspace and CUDA stream; one host
thread per scene drives its restarted GMRES (usv_gmres_solve releases the
Python GIL and its per-cycle graph is captured on a thread-local stream), so
the kernels of all scenes share the GPU at the same time. Results are the
same as solving the scenes one after the other.
"""
from __future__ import annotations

from concurrent.futures import ThreadPoolExecutor

import torch


def solve_scenes(solvers, rhs_list, adjoint: bool = False, max_workers: int | None = None):
    """Solve rhs_list[i] with solvers[i] (HelmholtzB200Solver) concurrently.

    rhs_list[i]: complex128 device tensor (N_i,) or (B_i, N_i). Returns the
    solutions in the same order; exceptions of any scene are re-raised.
    """
    if len(solvers) != len(rhs_list):
        raise ValueError("one right-hand-side tensor per scene")
    for s in solvers:
        s.assemble_matrix()
    device = solvers[0].device if solvers else None
    streams = [torch.cuda.Stream(device=device) for _ in solvers]
    # inputs become visible to each scene's stream before its solve starts
    for st in streams:
        st.wait_stream(torch.cuda.current_stream(device))

    def run(i):
        with torch.cuda.stream(streams[i]):
            x = solvers[i].solve_rhs_device(rhs_list[i], adjoint=adjoint)
        return x

    with ThreadPoolExecutor(max_workers=max_workers or max(len(solvers), 1)) as pool:
        futures = [pool.submit(run, i) for i in range(len(solvers))]
        out = [f.result() for f in futures]
    cur = torch.cuda.current_stream(device)
    for st in streams:
        cur.wait_stream(st)
    return out
