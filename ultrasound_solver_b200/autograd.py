"""Differentiable phases -> field through the Helmholtz solve.

PhaseField.apply(phases, solver) returns the device field u = A^-1 B (a e^{i phi})
(Fortran node order, complex128). Its backward is the hand-written adjoint:
lambda = A^-H g (the matrix-free A^H GMRES), then
dL/dphi_m = Re(conj(a_m (B^H lambda)_m) i e^{i phi_m}) (usv_source_phase_grad).
Only the forward field is kept for backward, never a Krylov basis. The
gradient equals the reference's basis VJP (phase_response_basis.py:208-253)
because G^H g = diag(a) B^H A^-H g.
"""
from __future__ import annotations

import torch


class PhaseField(torch.autograd.Function):
    @staticmethod
    def forward(ctx, phases: torch.Tensor, solver):
        if solver.operator is None:
            solver.assemble_matrix()
        ph = phases.detach().to(dtype=torch.float64)
        amps = torch.as_tensor(solver.transducers.amplitudes, dtype=torch.float64,
                               device=solver.device)
        rhs = solver.sources.rhs((amps * torch.exp(1j * ph.to(solver.device))).view(1, -1))[0]
        u = solver.solve_rhs_device(rhs)
        ctx.solver = solver
        ctx.save_for_backward(ph, u)
        return u

    @staticmethod
    def backward(ctx, grad_u: torch.Tensor):
        ph, _u = ctx.saved_tensors
        solver = ctx.solver
        lam = solver.solve_rhs_device(grad_u.to(torch.complex128).contiguous(), adjoint=True)
        grad = solver.sources.phase_grad(lam, solver.transducers.amplitudes,
                                         ph.cpu().numpy())
        return grad.to(ph.device), None


def phase_field(phases: torch.Tensor, solver) -> torch.Tensor:
    """Differentiable field of the solver's scene for `phases` (radians)."""
    return PhaseField.apply(phases, solver)


class LossOfField(torch.autograd.Function):
    """A device loss (losses._DeviceLoss) as an autograd node: value, and its
    field cotangent as the backward (dL = Re(g^H du) is torch's convention)."""

    @staticmethod
    def forward(ctx, u: torch.Tensor, loss):
        value, cot = loss.evaluate_vector(u, with_cotangent=True)
        ctx.save_for_backward(cot)
        return value

    @staticmethod
    def backward(ctx, grad_out):
        (cot,) = ctx.saved_tensors
        return cot * grad_out.to(cot.dtype), None


def loss_of_field(u: torch.Tensor, loss) -> torch.Tensor:
    return LossOfField.apply(u, loss)
