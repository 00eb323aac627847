"""Row-scaled Jacobi GMRES on the B200: the drop-in for GpuIterativeSolver.

Mirrors src/algorithm/solvers/iterative_solver.py:12-104 — same constructor
arguments and defaults, same stats attributes (last_iterations,
last_scaled_residual, last_backward_error), same acceptance gates and the
same RuntimeError message — but the operator is the matrix-free sm_100a
stencil and the whole restarted GMRES runs in CUDA (usv_gmres_solve),
batched over right-hand sides.

precision="mixed": complex64 Krylov vectors and stencil inside each cycle,
FP64 Gram-Schmidt dots, Hessenberg/Givens, true residual and solution update
(iterative refinement at every restart). precision="bf16": the same with the
Krylov vectors stored as bfloat16 complex (4 bytes per node; the fp32
stencil and FP64 dots widen them on load), which halves the basis traffic;
the FP64 refinement at every restart keeps the converged solution the same.
precision="fp64": complex128 throughout — the plain FP64 comparator.

recycle=k > 0 turns each restart into a GCRO-DR(m, k) cycle (Parks et al.
2006): k harmonic Ritz vectors of the previous cycles are kept as a pair
(U, C = K U), every new residual is projected on C first and the Arnoldi
process runs m - k steps orthogonal to C. The host computes the harmonic Ritz
step of one cycle while the next runs (one cycle of lag). recycle=0 (the
default) is the reference's plain restarted GMRES.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _native as N

_PRECISIONS = {"mixed": N.PREC_MIXED, "fp64": N.PREC_FP64, "complex64": N.PREC_MIXED,
               "bf16": N.PREC_MIXED_BF16, "mixed_bf16": N.PREC_MIXED_BF16,
               "complex128": N.PREC_FP64}


class B200IterativeSolver:
    """GPU row-scaled Jacobi-GMRES solver for the matrix-free Helmholtz operator."""

    def __init__(self, restart: int = 30, maxiter: int = 3000, rtol: float = 1.0e-6,
                 backward_error_tol: float = 1.0e-4, precision: str = "mixed",
                 full_cycles: bool = True, use_graph: bool = True, block_nodes: int = 0,
                 verbose: bool = False, profile: bool = False, recycle: int = 0,
                 recycle_every: int = 1, batch_width: int = 0, max_ctas: int = 0,
                 kernel_variant: int = 0):
        if str(precision).lower() not in _PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(_PRECISIONS)}")
        self.restart = int(restart)
        self.maxiter = int(maxiter)
        self.rtol = float(rtol)
        self.backward_error_tol = float(backward_error_tol)
        self.precision = str(precision).lower()
        self.full_cycles = bool(full_cycles)
        self.use_graph = bool(use_graph)
        self.block_nodes = int(block_nodes)
        self.recycle = int(recycle)
        self.recycle_every = int(recycle_every)
        # right-hand sides per launch (0: all of them); autotune.BatchTuner picks it
        self.batch_width = int(batch_width)
        # cap on CTAs per right-hand side (0: fill the GPU); a small cap makes
        # every CTA of the streaming kernels loop over several node chunks
        self.max_ctas = int(max_ctas)
        # N.GMRES_* bits selecting other forms of the Arnoldi kernels than the
        # measured-fastest default (autotune.BatchTuner can pick them)
        self.kernel_variant = int(kernel_variant)
        self.verbose = bool(verbose)
        self.profile = bool(profile)
        self.last_profile = None
        self.last_iterations = 0
        self.last_scaled_residual = None
        self.last_backward_error = None
        self.last_stats = []
        self.last_history = []

    def history_capacity(self) -> int:
        return self.maxiter // max(self.restart - max(self.recycle, 0), 1) + 2

    def params(self, adjoint: bool = False) -> N.GmresParams:
        p = N.GmresParams()
        p.restart, p.maxiter = self.restart, self.maxiter
        p.rtol, p.backward_error_tol = self.rtol, self.backward_error_tol
        p.precision = _PRECISIONS[self.precision]
        p.adjoint = 1 if adjoint else 0
        p.full_cycles = 1 if self.full_cycles else 0
        p.use_graph = 1 if self.use_graph else 0
        p.block_nodes = self.block_nodes
        p.history_capacity = self.history_capacity()
        p.recycle = self.recycle
        p.recycle_every = self.recycle_every
        p.max_ctas = self.max_ctas
        p.kernel_variant = self.kernel_variant
        return p

    def workspace_bytes(self, operator, nrhs: int, adjoint: bool = False) -> int:
        nbytes = C.c_size_t()
        p = self.params(adjoint)
        N.check(N.load().usv_gmres_workspace_bytes(C.byref(operator.scene), C.byref(p), int(nrhs),
                                                   C.byref(nbytes)), "gmres workspace")
        return nbytes.value

    def solve(self, operator, rhs: torch.Tensor, adjoint: bool = False,
              raise_on_failure: bool = True) -> torch.Tensor:
        """Solve A x = rhs (or A^H x = rhs) on the device.

        rhs: complex128 device tensor of shape (N,) or (B, N) (row b is one
        right-hand side). Returns x with the same shape. With batch_width > 0
        the right-hand sides go through the solver in launches of at most
        batch_width (the stats then cover all of them).
        """
        squeeze = rhs.dim() == 1
        b = rhs.reshape(1, -1) if squeeze else rhs
        if b.shape[-1] != operator.n:
            raise ValueError("rhs length does not match the operator")
        if 0 < self.batch_width < b.shape[0]:
            parts, stats, hist, prof = [], [], [], None
            for lo in range(0, b.shape[0], self.batch_width):
                parts.append(self._solve_batch(operator, b[lo:lo + self.batch_width], adjoint,
                                               raise_on_failure))
                stats += self.last_stats
                hist += self.last_history
                if self.last_profile is not None:
                    prof = prof or {k: dict(launches=0, ms=0.0, bytes=0.0) for k in self.last_profile}
                    for k, v in self.last_profile.items():
                        for f in v:
                            prof[k][f] += v[f]
            self.last_stats, self.last_history, self.last_profile = stats, hist, prof
            self.last_iterations = max(s["iterations"] for s in stats)
            self.last_scaled_residual = max(s["scaled_residual"] for s in stats)
            self.last_backward_error = max(s["backward_error"] for s in stats)
            return torch.cat(parts)
        x = self._solve_batch(operator, b, adjoint, raise_on_failure)
        return x[0] if squeeze else x

    def _solve_batch(self, operator, b: torch.Tensor, adjoint: bool,
                     raise_on_failure: bool) -> torch.Tensor:
        b = b.to(device=operator.device, dtype=torch.complex128).contiguous()
        nrhs = b.shape[0]
        x = torch.empty_like(b)
        p = self.params(adjoint)
        nbytes = self.workspace_bytes(operator, nrhs, adjoint)
        ws = torch.empty(nbytes, dtype=torch.uint8, device=operator.device)
        stats = (N.GmresStats * nrhs)()
        hcap = p.history_capacity
        hist = (C.c_double * (hcap * nrhs))()
        p.history = C.cast(hist, C.POINTER(C.c_double))
        prof = N.GmresProfile() if self.profile else None
        if prof is not None:
            p.profile = C.pointer(prof)
        with torch.cuda.device(operator.device):
            N.check(N.load().usv_gmres_solve(C.byref(operator.scene), N.ptr(operator.buffer),
                                             C.byref(p), N.ptr(b), N.ptr(x), nrhs, operator.n,
                                             N.ptr(ws), nbytes, stats,
                                             N.stream_handle(torch, operator.device)),
                    "gmres")
        del ws
        self.record_stats(stats, hist, hcap, prof, raise_on_failure)
        return x

    def record_stats(self, stats, hist, hcap, prof, raise_on_failure: bool) -> None:
        """Per-RHS statistics of a finished launch (last_stats, last_history,
        last_profile, the maxima over the batch); raises the reference's
        RuntimeError for a right-hand side that failed its gates."""
        self.last_stats = [dict(status=s.status, info=s.info, iterations=s.iterations,
                                cycles=s.cycles, scaled_residual=s.scaled_residual,
                                backward_error=s.backward_error,
                                initial_residual=s.initial_residual) for s in stats]
        self.last_history = [list(hist[k * hcap:k * hcap + min(s.cycles, hcap)])
                             for k, s in enumerate(stats)]
        self.last_profile = None
        if prof is not None:
            self.last_profile = {name: dict(launches=prof.launches[i], ms=prof.milliseconds[i],
                                            bytes=prof.bytes[i])
                                 for i, name in enumerate(N.KFAMILY_NAMES)}
        self.last_iterations = max(s.iterations for s in stats)
        self.last_scaled_residual = max(s.scaled_residual for s in stats)
        self.last_backward_error = max(s.backward_error for s in stats)
        if raise_on_failure:
            for s in stats:
                if s.status != N.USV_OK:
                    raise RuntimeError(
                        f"info={s.info}, iterations={s.iterations}, "
                        f"scaled residual={s.scaled_residual:.3e}, "
                        f"backward error={s.backward_error:.3e}")
        if self.verbose:
            print(f"  --> GMRES iterations: {self.last_iterations} | scaled relative residual: "
                  f"{self.last_scaled_residual:.3e} | backward error: "
                  f"{self.last_backward_error:.3e}")
