"""Several scenes of different grid sizes in one batched GMRES launch sequence
(usv_gmres_solve_scenes through scene_batch.solve_scenes_batched) against the
reference's direct solutions of every scene.

Scenes: the four reference-generated goldens (14 x 13 x 12, 16 x 16 x 14,
12 x 10 x 11 and 36 x 32 x 30 nodes; every face kind, PML on subsets of faces,
obstacles and explicit media), with single-emitter columns and phased
right-hand sides mixed in one launch of seven right-hand sides.
"""
import numpy as np
import pytest
import torch

from tests.conftest import load_golden
from tests.helpers import golden_solver, rel

pytestmark = pytest.mark.gpu

CASES = {  # scene -> number of single-emitter columns (0: the phased RHS)
    "mixed": 2, "air_pml": 0, "fields": 1, "mid": 3,
}
SOLVERS = {
    "fp64_gmres30": dict(precision="fp64", gmres_restart=30),
    "mixed_gmres30": dict(precision="mixed", gmres_restart=30),
    "bf16_gcrodr36_8": dict(precision="bf16", gmres_restart=36, gmres_recycle=8,
                            gmres_recycle_every=2),
}


def _scenes(**solver):
    goldens = {name: load_golden(name) for name in CASES}
    solvers = {name: golden_solver(g, gmres_rtol=1e-10, gmres_maxiter=200000, **solver)
               for name, g in goldens.items()}
    return goldens, solvers


def _forward_case(g, s, ncols):
    if ncols == 0:
        return s.update_rhs_device().reshape(1, -1), [g["x_direct"]]
    cols = s.sources.column_rhs(s.transducers.amplitudes)[:ncols]
    return cols, [g["G"][:, k].astype(np.complex128) for k in range(ncols)]


@pytest.mark.parametrize("solver", list(SOLVERS))
def test_forward_scenes_in_one_launch(solver):
    from ultrasound_solver_b200.scene_batch import solve_scenes_batched
    goldens, solvers = _scenes(**SOLVERS[solver])
    rhs, want = [], []
    for name, ncols in CASES.items():
        r, w = _forward_case(goldens[name], solvers[name], ncols)
        rhs.append(r)
        want.append(w)
    order = list(CASES)
    xs = solve_scenes_batched([solvers[n] for n in order], rhs)
    it = solvers[order[0]].iterative_solver
    assert len(it.last_stats) == sum(r.shape[0] for r in rhs)
    for name, x, w in zip(order, xs, want):
        x = x.cpu().numpy()
        for k, ref in enumerate(w):
            assert rel(x[k], ref) <= 1e-6, (name, k, rel(x[k], ref))


def test_adjoint_scenes_in_one_launch():
    from ultrasound_solver_b200.scene_batch import solve_scenes_batched
    goldens, solvers = _scenes(precision="bf16", gmres_restart=30)
    order = list(CASES)
    rhs, want = [], []
    for name in order:
        g = goldens[name]
        a = np.asarray(g["adj_rhs"], dtype=np.complex128)
        sol = np.asarray(g["adj_sol"], dtype=np.complex128)
        if a.ndim == 1:
            a, sol = a[:, None], sol[:, None]
        rhs.append(torch.from_numpy(np.ascontiguousarray(a.T)).cuda())
        want.append(sol.T)
    xs = solve_scenes_batched([solvers[n] for n in order], rhs, adjoint=True)
    for name, x, w in zip(order, xs, want):
        x = x.cpu().numpy()
        for k in range(w.shape[0]):
            assert rel(x[k], w[k]) <= 1e-6, (name, k)
