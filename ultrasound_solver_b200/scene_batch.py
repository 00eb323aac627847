"""Solves of independent scenes (uneven grid sizes) on one GPU.

solve_scenes_batched puts the right-hand sides of every scene into ONE
batched GMRES launch sequence (usv_gmres_solve_scenes): each CTA row of a
kernel launch is one right-hand side and reads its scene (operator buffer,
node count, node steps) from a slot table, so a restart cycle of all scenes
is one CUDA graph and one status read. solve_scenes instead keeps each
scene's operator, workspace and CUDA stream and drives them from one host
thread per scene (usv_gmres_solve releases the Python GIL), so the kernels of
the scenes overlap on the GPU. Both give the same solutions as solving the
scenes one after the other.
"""
from __future__ import annotations

import ctypes as C
from concurrent.futures import ThreadPoolExecutor

import torch

from . import _native as N


def solve_scenes_batched(solvers, rhs_list, adjoint: bool = False, raise_on_failure: bool = True):
    """Solve rhs_list[i] with solvers[i]'s operator, all scenes in one launch sequence.

    rhs_list[i]: complex128 device tensor (N_i,) or (B_i, N_i). The GMRES
    settings (restart, recycling, precision, tolerances) are those of
    solvers[0].iterative_solver. Returns the solutions in the same shapes;
    per-RHS statistics are in solvers[0].iterative_solver.last_stats (scene
    order, then right-hand-side order).
    """
    if len(solvers) != len(rhs_list) or not solvers:
        raise ValueError("one right-hand-side tensor per scene")
    for s in solvers:
        s.assemble_matrix()
    ops = [s.operator for s in solvers]
    dev = ops[0].device
    blocks, owner, shapes = [], [], []
    for i, (op, r) in enumerate(zip(ops, rhs_list)):
        b = r.reshape(1, -1) if r.dim() == 1 else r
        if b.shape[-1] != op.n:
            raise ValueError(f"scene {i}: rhs length does not match the operator")
        blocks.append(b)
        owner += [i] * b.shape[0]
        shapes.append(r.shape)
    nrhs = len(owner)
    ld = max(op.n for op in ops)
    rhs = torch.zeros((nrhs, ld), dtype=torch.complex128, device=dev)
    row = 0
    for op, b in zip(ops, blocks):
        rhs[row:row + b.shape[0], :op.n] = b.to(device=dev, dtype=torch.complex128)
        row += b.shape[0]
    x = torch.empty_like(rhs)
    it = solvers[0].iterative_solver
    p = it.params(adjoint)
    scenes = (N.Scene * len(ops))(*[op.scene for op in ops])
    bufs = (C.c_void_p * len(ops))(*[op.buffer.data_ptr() for op in ops])
    of = (C.c_int * nrhs)(*owner)
    lib = N.load()
    nbytes = C.c_size_t()
    N.check(lib.usv_gmres_scenes_workspace_bytes(len(ops), scenes, of, C.byref(p), nrhs,
                                                 C.byref(nbytes)), "gmres workspace")
    ws = torch.empty(nbytes.value, dtype=torch.uint8, device=dev)
    stats = (N.GmresStats * nrhs)()
    hcap = p.history_capacity
    hist = (C.c_double * (hcap * nrhs))()
    p.history = C.cast(hist, C.POINTER(C.c_double))
    with torch.cuda.device(dev):
        N.check(lib.usv_gmres_solve_scenes(len(ops), scenes, bufs, of, C.byref(p), N.ptr(rhs),
                                           N.ptr(x), nrhs, ld, N.ptr(ws), nbytes.value, stats,
                                           N.stream_handle(torch, dev)), "gmres")
    del ws
    it.record_stats(stats, hist, hcap, None, raise_on_failure)
    out, row = [], 0
    for op, b, shp in zip(ops, blocks, shapes):
        out.append(x[row:row + b.shape[0], :op.n].reshape(shp))
        row += b.shape[0]
    return out


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
