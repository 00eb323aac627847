"""Parity at the benchmark's own sizes (128^3 = 2,097,152 nodes).

At this size every streaming GMRES kernel runs its full persistent grid and
each CTA loops over many node chunks -- the paths the bench times.

* config 1: the bfloat16 GCRO-DR(36,8) solution of the bench (rtol 1e-9)
  against a plain FP64 GMRES(30) solve of the same scene to rtol 1e-11
  (the reference's algorithm in complex128); bar 1e-6 (BASELINE metric).
* config 3: the adjoint phase gradient of the contrast-ratio focal loss
  (16 x 16 array) against central finite differences (step 1e-4 rad) on 8
  seeded phases, and against the same adjoint computed in complex128.
  The perturbed fields u(phi +- h e_k) come from the solve's linearity,
  u + G_k (e^{+-ih} - 1) e^{i phi_k}, with the single-emitter columns G_k
  solved as one batch: exactly the fields a full re-solve would give, up to
  the solver tolerance.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _config_solver(cfg, **solver):
    from ultrasound_solver_b200 import workloads as W
    s = W.build_solver(cfg, seed=0)
    s.assemble_matrix()
    it = s.iterative_solver
    it.backward_error_tol = 1e-4
    for k, v in solver.items():
        setattr(it, k, v)
    return s


def _rel(a, b):
    return float((torch.linalg.norm(a - b) / torch.linalg.norm(b)).item())


def test_config1_bf16_gcrodr_matches_fp64_gmres():
    from ultrasound_solver_b200 import workloads as W
    s = _config_solver(W.config1(128))
    rhs = s.update_rhs_device()
    it = s.iterative_solver
    it.precision, it.restart, it.recycle, it.rtol, it.maxiter = "fp64", 30, 0, 1e-11, 400000
    x64 = it.solve(s.operator, rhs)
    assert it.last_scaled_residual <= 1e-11
    it.precision, it.restart, it.recycle, it.recycle_every = "bf16", 36, 8, 2
    it.rtol, it.maxiter = 1e-9, 80000
    xb = it.solve(s.operator, rhs)
    assert it.last_scaled_residual <= 1e-9
    err = _rel(xb, x64)
    print(f"config1 128^3: bf16 GCRO-DR vs FP64 GMRES rel err {err:.2e}")
    assert err <= 1e-6


def test_config3_adjoint_gradient_vs_finite_differences():
    from ultrasound_solver_b200 import workloads as W
    from ultrasound_solver_b200.autograd import loss_of_field, phase_field
    from ultrasound_solver_b200.losses import ContrastRatioLoss
    s = _config_solver(W.config3(128), precision="bf16", restart=36, recycle=8,
                       recycle_every=2, rtol=1e-10, maxiter=100000)
    it = s.iterative_solver
    centre = 127 * s.cfg.domain.dx / 2
    loss = ContrastRatioLoss(s.cfg, (centre, centre, 0.080), focal_radius=0.006,
                             shell_thickness=0.010)
    m = s.transducers.num_transducers
    assert m == 256
    phases0 = np.random.default_rng(2).uniform(0, 2 * np.pi, m)

    def gradient(precision):
        it.precision = precision
        ph = torch.tensor(phases0, dtype=torch.float64, device="cuda", requires_grad=True)
        u = phase_field(ph, s)
        L = loss_of_field(u, loss)
        L.backward()
        return u.detach(), ph.grad.detach().cpu().numpy()

    u, grad = gradient("bf16")
    idx = np.random.default_rng(3).choice(m, size=8, replace=False)
    # single-emitter columns G_k = A^-1 (a_k B e_k) of the 8 phases, one batch
    coeff = np.zeros((len(idx), m), dtype=np.complex128)
    coeff[np.arange(len(idx)), idx] = np.asarray(s.transducers.amplitudes)[idx]
    cols = s.sources.rhs(torch.from_numpy(coeff))
    it.precision = "bf16"
    G = s.solve_rhs_device(cols)
    h = 1e-4

    def value(field):
        return float(loss.evaluate_vector(field, False)[0])

    fd = []
    for r, k in enumerate(idx):
        e = np.exp(1j * phases0[k])
        up = u + G[r] * complex((np.exp(1j * h) - 1) * e)
        dn = u + G[r] * complex((np.exp(-1j * h) - 1) * e)
        fd.append((value(up) - value(dn)) / (2 * h))
    fd = np.asarray(fd)
    err_fd = float(np.linalg.norm(grad[idx] - fd) / np.linalg.norm(fd))
    # the same gradient with complex128 Krylov vectors
    it.recycle, it.restart = 8, 36
    _, grad64 = gradient("fp64")
    err64 = float(np.linalg.norm(grad - grad64) / np.linalg.norm(grad64))
    print(f"config3 128^3: adjoint vs central FD rel {err_fd:.2e}, bf16 vs complex128 "
          f"adjoint rel {err64:.2e}")
    assert err_fd <= 1e-5
    assert err64 <= 1e-6
