"""Host-injected failures of the batched GMRES (no GPU fault is provoked).

* A non-finite value in one right-hand side of a batch: that column ends with
  USV_ERR_NONFINITE (the reference raises on a non-finite solve,
  src/algorithm/solvers/iterative_solver.py:86-97), the other columns of the
  same launch still converge to the reference's solutions, and the public
  API raises the reference's RuntimeError.
* Lucky breakdown: on an all-soft 3 x 3 x 3 grid (one free node) the
  operator has a degree-2 minimal polynomial, so the Arnoldi process breaks
  down at its second step; on 2 x 2 x 2 every node is fixed (A = I) and it
  breaks down at the first. The solve must end cleanly with the exact
  solution (with complex64 / bfloat16 vectors the rounded basis only nearly
  breaks down, and the FP64 restarts finish the solve).
"""
import numpy as np
import pytest
import torch

from tests.conftest import load_golden
from tests.helpers import golden_solver, rel

pytestmark = pytest.mark.gpu

SOLVERS = [
    ("fp64", 0), ("mixed", 0), ("bf16", 0), ("bf16", 8), ("fp64", 8),
]


@pytest.mark.parametrize("precision,recycle", SOLVERS)
def test_nonfinite_column_is_isolated(precision, recycle):
    from ultrasound_solver_b200 import _native as N
    g = load_golden("mid")
    s = golden_solver(g, precision=precision, gmres_rtol=1e-10, gmres_maxiter=200000,
                      gmres_restart=36 if recycle else 30, gmres_recycle=recycle,
                      gmres_recycle_every=2)
    cols = s.sources.column_rhs(s.transducers.amplitudes)[:3].clone()
    cols[1, 1234] = complex(float("nan"), 0.0)
    it = s.iterative_solver
    x = it.solve(s.operator, cols, raise_on_failure=False)
    st = it.last_stats
    assert st[1]["status"] == N.USV_ERR_NONFINITE
    G = g["G"].astype(np.complex128)
    for k in (0, 2):
        assert st[k]["status"] == N.USV_OK
        assert rel(x[k].cpu().numpy(), G[:, k]) <= 1e-6
    with pytest.raises(RuntimeError, match=r"info=.*iterations=.*scaled residual=.*backward error="):
        s.solve_rhs(cols.cpu().numpy().T, verbose=False)


def test_nonfinite_adjoint_column():
    from ultrasound_solver_b200 import _native as N
    g = load_golden("mid")
    s = golden_solver(g, precision="bf16", gmres_rtol=1e-10, gmres_maxiter=200000)
    rhs = torch.from_numpy(g["adj_rhs"].astype(np.complex128).T.copy()).cuda()
    rhs[0, 77] = complex(0.0, float("inf"))
    it = s.iterative_solver
    lam = it.solve(s.operator, rhs, adjoint=True, raise_on_failure=False)
    assert it.last_stats[0]["status"] == N.USV_ERR_NONFINITE
    for k in (1, 2):
        assert it.last_stats[k]["status"] == N.USV_OK
        assert rel(lam[k].cpu().numpy(), g["adj_sol"][:, k]) <= 1e-6


def _soft_box(n):
    from ultrasound_solver_b200.scene import DeviceOperator
    rho = torch.full((n ** 3,), 1.2, dtype=torch.float64, device="cuda")
    c = torch.full((n ** 3,), 343.0, dtype=torch.float64, device="cuda")
    faces = {f: "soft" for f in ("-x", "+x", "-y", "+y", "-z", "+z")}
    return DeviceOperator((n, n, n), 1e-3, 2 * np.pi * 40000.0, faces, rho, c)


@pytest.mark.parametrize("n", [2, 3])
@pytest.mark.parametrize("precision,recycle", SOLVERS)
def test_lucky_breakdown_ends_cleanly(n, precision, recycle):
    from ultrasound_solver_b200 import _native as N
    from ultrasound_solver_b200.iterative_solver import B200IterativeSolver
    op = _soft_box(n)
    nn = n ** 3
    recycle = min(recycle, nn - 2)  # GCRO-DR needs k < m = min(restart, N)
    A = op.apply(torch.eye(nn, dtype=torch.complex128, device="cuda")).cpu().numpy().T
    rng = np.random.default_rng(n)
    b = rng.standard_normal((2, nn)) + 1j * rng.standard_normal((2, nn))
    it = B200IterativeSolver(restart=36 if recycle else 30, maxiter=1000, rtol=1e-10,
                             precision=precision, recycle=recycle, recycle_every=2)
    for adjoint in (False, True):
        x = it.solve(op, torch.from_numpy(b).cuda(), adjoint=adjoint).cpu().numpy()
        M = A.conj().T if adjoint else A
        for k in range(2):
            want = np.linalg.solve(M, b[k])
            assert rel(x[k], want) <= (1e-9 if precision == "fp64" else 1e-8)
            assert it.last_stats[k]["status"] == N.USV_OK
        if precision == "fp64":  # exact breakdown: the first cycle ends it
            assert it.last_iterations <= 2 * it.restart
