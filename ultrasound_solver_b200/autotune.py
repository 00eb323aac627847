"""Autotuners for the batched GMRES launches and the stencil kernels.

How many right-hand sides go through one usv_gmres_solve launch decides how
well the persistent grids fill the GPU (few RHS: per-launch latency and the
per-cycle host round trip dominate; many: the Krylov workspace grows as
B (m+1) N and each RHS gets fewer CTAs). BatchTuner times a few restart
cycles of the real operator at each candidate width that fits the memory
budget and keeps the width with the lowest time per right-hand-side
iteration. It then times the kernel forms at that width
(usv_gmres_params.kernel_variant) and keeps the fastest: the bulk-copy
orthogonalisation ring or the per-thread cp.async pipeline and, with bf16
GCRO-DR(m, 4 or 8), the recycled pair on tcgen05 or on mma.sync.
StencilTuner picks the complex64 operator-apply
kernel (precomputed row coefficients, one thread per node, or 16-byte node
records with z-marching tiles) for a grid and batch width. Results are cached
in a JSON file keyed by GPU name, grid and the solver settings, so each
measurement runs once per machine and scene shape.
"""
from __future__ import annotations

import json
import os
import time
from pathlib import Path

import torch

DEFAULT_CACHE = Path(os.environ.get("USV_AUTOTUNE_CACHE",
                                    Path.home() / ".cache" / "ultrasound_solver_b200" / "autotune.json"))


def cache_key(device_name: str, shape, precision: str, restart: int, recycle: int,
              adjoint: bool) -> str:
    grid = "x".join(str(int(v)) for v in shape)
    return f"{device_name}|{grid}|{precision}|m{restart}|k{recycle}|{'adj' if adjoint else 'fwd'}"


class BatchTuner:
    """Pick iterative_solver.batch_width for one operator (see module docstring)."""

    def __init__(self, cache_path: str | Path | None = None, candidates=(1, 2, 4, 8, 16, 32, 64),
                 cycles: int = 2, memory_fraction: float = 0.6):
        self.cache_path = Path(cache_path) if cache_path else DEFAULT_CACHE
        self.candidates = tuple(int(c) for c in candidates)
        self.cycles = int(cycles)
        self.memory_fraction = float(memory_fraction)
        self.cache = self._load()
        self.last_timings = {}

    def _load(self) -> dict:
        try:
            return json.loads(self.cache_path.read_text())
        except (OSError, ValueError):
            return {}

    def _save(self) -> None:
        self.cache_path.parent.mkdir(parents=True, exist_ok=True)
        tmp = self.cache_path.with_suffix(".tmp")
        tmp.write_text(json.dumps(self.cache, indent=1, sort_keys=True))
        os.replace(tmp, self.cache_path)

    def feasible(self, solver, operator, nrhs_total: int, adjoint: bool = False,
                 free_bytes: int | None = None) -> list[int]:
        """Candidate widths <= nrhs_total whose workspace fits the memory budget."""
        if free_bytes is None:
            free_bytes, _ = torch.cuda.mem_get_info(operator.device)
        budget = self.memory_fraction * free_bytes
        out = []
        for b in self.candidates:
            if b > max(nrhs_total, 1):
                break
            need = solver.workspace_bytes(operator, b, adjoint) + 3 * b * operator.n * 16
            if need <= budget:
                out.append(b)
        return out or [1]

    def tune(self, solver, operator, rhs: torch.Tensor, adjoint: bool = False,
             force: bool = False) -> int:
        """Measure (or read from the cache) the best width; sets solver.batch_width."""
        rhs = rhs.reshape(-1, operator.n)
        name = torch.cuda.get_device_name(operator.device)
        key = cache_key(name, operator.shape, solver.precision, solver.restart, solver.recycle,
                        adjoint)
        if not force and key in self.cache:
            solver.batch_width = int(self.cache[key]["batch_width"])
            solver.kernel_variant = int(self.cache[key].get("kernel_variant", 0))
            return solver.batch_width
        saved = (solver.maxiter, solver.rtol, solver.batch_width, solver.profile)
        steps = max(solver.restart - max(solver.recycle, 0), 1)
        solver.maxiter = self.cycles * solver.restart + (3 if solver.recycle else 1) * steps
        solver.rtol, solver.batch_width, solver.profile = 0.0, 0, False
        timings = {}
        try:
            for b in self.feasible(solver, operator, rhs.shape[0], adjoint):
                idx = torch.arange(b, device=rhs.device) % rhs.shape[0]
                batch = rhs[idx]
                solver.solve(operator, batch, adjoint=adjoint, raise_on_failure=False)  # warm
                torch.cuda.synchronize(operator.device)
                t0 = time.perf_counter()
                solver.solve(operator, batch, adjoint=adjoint, raise_on_failure=False)
                torch.cuda.synchronize(operator.device)
                dt = time.perf_counter() - t0
                timings[b] = dt / max(solver.last_iterations, 1) / b
        finally:
            solver.maxiter, solver.rtol, solver.batch_width, solver.profile = saved
        best = min(timings, key=timings.get)
        self.last_timings = timings
        variant, variant_timings = self._tune_variant(solver, operator, rhs, best, adjoint)
        self.cache[key] = {"batch_width": best,
                           "seconds_per_rhs_iteration": {str(k): v for k, v in timings.items()},
                           "kernel_variant": variant,
                           "seconds_per_rhs_iteration_by_variant": variant_timings}
        self._save()
        solver.batch_width = best
        solver.kernel_variant = variant
        return best

    def _tune_variant(self, solver, operator, rhs, width, adjoint):
        """Time the Arnoldi kernel forms at `width` (complex64 / bfloat16 only)."""
        if solver.precision in ("fp64", "complex128"):
            return solver.kernel_variant, {}
        from . import _native as N
        saved = (solver.maxiter, solver.rtol, solver.batch_width, solver.profile,
                 solver.kernel_variant)
        steps = max(solver.restart - max(solver.recycle, 0), 1)
        solver.maxiter = self.cycles * solver.restart + (3 if solver.recycle else 1) * steps
        solver.rtol, solver.batch_width, solver.profile = 0.0, 0, False
        idx = torch.arange(width, device=rhs.device) % rhs.shape[0]
        batch = rhs[idx]
        timings = {}
        try:
            variants = [0, N.GMRES_ORTH_CPASYNC]
            if solver.precision == "bf16" and solver.recycle in (4, 8):
                variants.append(N.GMRES_COMBINE_MMA_SYNC)  # recycled pair: mma.sync form
            for variant in variants:
                solver.kernel_variant = variant
                solver.solve(operator, batch, adjoint=adjoint, raise_on_failure=False)
                torch.cuda.synchronize(operator.device)
                t0 = time.perf_counter()
                solver.solve(operator, batch, adjoint=adjoint, raise_on_failure=False)
                torch.cuda.synchronize(operator.device)
                timings[variant] = (time.perf_counter() - t0) / max(solver.last_iterations, 1) / width
        finally:
            (solver.maxiter, solver.rtol, solver.batch_width, solver.profile,
             solver.kernel_variant) = saved
        return min(timings, key=timings.get), {str(k): v for k, v in timings.items()}


class StencilTuner:
    """Pick the complex64 K / K^H apply kernel for one operator and batch width."""

    def __init__(self, cache_path: str | Path | None = None, reps: int = 10):
        self.cache_path = Path(cache_path) if cache_path else DEFAULT_CACHE
        self.reps = int(reps)
        self.last_timings = {}

    def tune(self, operator, nrhs: int, adjoint: bool = False, force: bool = False) -> int:
        """Measure (or read from the cache) the faster kernel; sets operator.stencil_kernel."""
        from . import _native as N
        name = torch.cuda.get_device_name(operator.device)
        grid = "x".join(str(int(v)) for v in operator.shape)
        key = f"stencil|{name}|{grid}|b{int(nrhs)}|{'adj' if adjoint else 'fwd'}"
        cache = BatchTuner(self.cache_path).cache
        if not force and key in cache:
            operator.stencil_kernel = int(cache[key]["kernel"])
            return operator.stencil_kernel
        variant = N.APPLY_KH if adjoint else N.APPLY_K
        x = torch.randn((int(nrhs), operator.n), dtype=torch.complex64, device=operator.device)
        candidates = [N.STENCIL_COEF_ROWS] + ([N.STENCIL_RECORD_TILES] if nrhs <= 4 else [])
        timings = {}
        for k in candidates:
            for _ in range(2):
                operator.apply(x, variant, N.PREC_MIXED, kernel=k)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(self.reps):
                operator.apply(x, variant, N.PREC_MIXED, kernel=k)
            e1.record()
            torch.cuda.synchronize(operator.device)
            timings[k] = e0.elapsed_time(e1) / self.reps
        best = min(timings, key=timings.get)
        self.last_timings = timings
        tuner = BatchTuner(self.cache_path)
        tuner.cache[key] = {"kernel": best, "ms_per_apply": {str(k): v for k, v in timings.items()}}
        tuner._save()
        operator.stencil_kernel = best
        return best
