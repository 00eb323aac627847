"""Adam phase optimisation driven by the adjoint gradient on the device.

The reference's `adjoint` baseline with `optimizer: adam`
(src/algorithm/baselines/adjoint/__init__.py:38-83): evaluate the loss and
its phase gradient at the initial phases, then for steps 1..n

    m  = 0.9 m + 0.1 g,   v = 0.999 v + 0.001 g^2
    phi -= lr * (m / (1 - 0.9^step)) / (sqrt(v / (1 - 0.999^step)) + 1e-8)

and evaluate again, stopping early when the best loss improved by at most
`tolerance` (relative) over `patience` steps (defaults 100, 1e-5, as in the
reference's _stagnated). Every evaluation is one forward solve and one
adjoint (A^H) solve behind torch.autograd (autograd.PhaseField), so a
gradient step costs two Helmholtz solves; the phases and moments stay on the
host in float64 like the reference's numpy arrays.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np
import torch

from .autograd import loss_of_field, phase_field


@dataclass
class Evaluation:
    phases: np.ndarray
    loss: float
    gradient: np.ndarray
    seconds: float


@dataclass
class AdamResult:
    phases: np.ndarray
    loss: float
    best_phases: np.ndarray
    best_loss: float
    losses: list = field(default_factory=list)       # after every evaluation
    seconds: list = field(default_factory=list)      # per evaluation (forward + adjoint)
    iterations: list = field(default_factory=list)   # inner GMRES iterations per evaluation
    steps: int = 0
    status: str = "iteration_limit"


def evaluate(solver, loss, phases) -> Evaluation:
    """Loss and phase gradient (forward + A^H solve) at `phases` (radians)."""
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ph = torch.tensor(np.asarray(phases, dtype=np.float64), device=solver.device,
                      requires_grad=True)
    value = loss_of_field(phase_field(ph, solver), loss)
    value.backward()
    grad = ph.grad.detach().cpu().numpy()
    lval = float(value.detach().item())
    torch.cuda.synchronize()
    return Evaluation(np.asarray(phases, dtype=np.float64).copy(), lval, grad,
                      time.perf_counter() - t0)


def adam(solver, loss, initial_phases, steps: int, learning_rate: float = 0.05,
         patience: int = 100, tolerance: float = 1.0e-5, callback=None) -> AdamResult:
    """Run `steps` Adam updates of the phases from `initial_phases`."""
    if not (learning_rate > 0 and np.isfinite(learning_rate)):
        raise ValueError("learning_rate must be finite and positive")
    if patience < 1 or not (tolerance > 0 and np.isfinite(tolerance)):
        raise ValueError("patience must be positive and tolerance finite and positive")
    it = solver.iterative_solver
    cur = evaluate(solver, loss, initial_phases)
    res = AdamResult(cur.phases, cur.loss, cur.phases, cur.loss, [cur.loss], [cur.seconds],
                     [it.last_iterations])
    first = np.zeros_like(cur.phases)
    second = np.zeros_like(cur.phases)
    checkpoint = res.best_loss
    for step in range(1, steps + 1):
        first = 0.9 * first + 0.1 * cur.gradient
        second = 0.999 * second + 0.001 * cur.gradient ** 2
        update = learning_rate * (first / (1 - 0.9 ** step)) / (
            np.sqrt(second / (1 - 0.999 ** step)) + 1e-8)
        cur = evaluate(solver, loss, cur.phases - update)
        res.steps = step
        res.losses.append(cur.loss)
        res.seconds.append(cur.seconds)
        res.iterations.append(it.last_iterations)
        res.phases, res.loss = cur.phases, cur.loss
        if cur.loss < res.best_loss:
            res.best_loss, res.best_phases = cur.loss, cur.phases
        if callback is not None:
            callback(step, cur)
        if step % patience == 0:
            if (checkpoint - res.best_loss) / max(1.0, abs(checkpoint)) <= tolerance:
                res.status = "converged"
                break
            checkpoint = res.best_loss
    return res
