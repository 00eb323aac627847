"""GPU parity on the mid-size reference golden (36 x 32 x 30 = 34,560 nodes).

The golden holds the reference's own direct solutions (tests/golden/make_golden.py,
`make_mid`) of a scene with a seeded random medium, a blended rho = 1250 sphere
and every face kind (open without PML, impedance, soft, open with PML,
reflecting baffle). The solves run with the CTA count of the streaming GMRES
kernels capped (`gmres_max_ctas`), so every CTA of k_dots / k_orth / k_update /
k_residual / the recycled-pair kernels loops over several node chunks (17
chunks of 2048 nodes, 9 of 4096 for the bfloat16 dots) and the last CTA
reduces partials from several CTAs -- the code paths the 128^3 workload takes.

Bar: relative L2 error <= 1e-6 against the reference's direct solve (the
stored solutions are rounded to complex64, 6e-8 relative).
"""
import numpy as np
import pytest
import torch

from tests.conftest import load_golden
from tests.helpers import golden_solver, rel

pytestmark = pytest.mark.gpu

ALGORITHMS = {
    "gmres30": dict(gmres_restart=30),
    "gcrodr36_8": dict(gmres_restart=36, gmres_recycle=8, gmres_recycle_every=2),
}
TOL = 1e-6


@pytest.fixture(scope="module")
def mid():
    return load_golden("mid")


def _solver(g, precision, algorithm, max_ctas=3):
    return golden_solver(g, precision=precision, gmres_rtol=1e-10, gmres_maxiter=200000,
                         gmres_max_ctas=max_ctas, **ALGORITHMS[algorithm])


def _adjoint_batch(g, nrhs):
    """Cotangents with known A^-H solutions: the stored three, then a complex
    multiple of the first (linearity)."""
    rhs = g["adj_rhs"].astype(np.complex128)
    sol = g["adj_sol"].astype(np.complex128)
    cols, sols = [], []
    for k in range(nrhs):
        if k < rhs.shape[1]:
            cols.append(rhs[:, k])
            sols.append(sol[:, k])
        else:
            z = 0.5 - 2.0j
            cols.append(z * rhs[:, 0])
            sols.append(z * sol[:, 0])
    return np.column_stack(cols), np.column_stack(sols)


@pytest.mark.parametrize("algorithm", list(ALGORITHMS))
@pytest.mark.parametrize("precision", ["fp64", "mixed", "bf16"])
@pytest.mark.parametrize("nrhs", [1, 3, 4])
def test_forward_batch(mid, precision, algorithm, nrhs):
    s = _solver(mid, precision, algorithm)
    G = mid["G"].astype(np.complex128)
    if nrhs == 1:
        # the phased right-hand side of the scene, through solve()
        field = s.solve().ravel(order="F")
        want = G @ np.exp(1j * mid["phases"])
        assert rel(field, want) <= TOL
        return
    cols = s.sources.column_rhs(s.transducers.amplitudes)[:nrhs]  # single-emitter columns
    x = s.solve_rhs(cols.cpu().numpy().T, verbose=False)
    assert x.shape == (s.total_dofs, nrhs)
    for k in range(nrhs):
        assert rel(x[:, k], G[:, k]) <= TOL, (k, rel(x[:, k], G[:, k]))
    assert s.iterative_solver.last_scaled_residual <= 1e-10


@pytest.mark.parametrize("algorithm", list(ALGORITHMS))
@pytest.mark.parametrize("precision", ["fp64", "mixed", "bf16"])
@pytest.mark.parametrize("nrhs", [1, 3, 4])
def test_adjoint_batch(mid, precision, algorithm, nrhs):
    s = _solver(mid, precision, algorithm)
    g, want = _adjoint_batch(mid, nrhs)
    lam = s.solve_adjoint(g)
    shape = tuple(mid["shape"])
    assert lam.shape == shape + (nrhs,)
    lam = lam.reshape((-1, nrhs), order="F")
    for k in range(nrhs):
        assert rel(lam[:, k], want[:, k]) <= TOL, (k, rel(lam[:, k], want[:, k]))


@pytest.mark.parametrize("max_ctas", [0, 1, 2, 5])
def test_cta_count_does_not_change_the_solution(mid, max_ctas):
    """The same bfloat16 GCRO-DR solve with the default grid (at most one chunk
    per CTA here), one CTA per RHS (every chunk in one CTA) and other caps."""
    s = _solver(mid, "bf16", "gcrodr36_8", max_ctas=max_ctas)
    cols = s.sources.column_rhs(s.transducers.amplitudes)[:2]
    x = s.solve_rhs_device(cols).cpu().numpy()
    G = mid["G"].astype(np.complex128)
    for k in range(2):
        assert rel(x[k], G[:, k]) <= TOL


def test_fp64_iterations_independent_of_cta_cap(mid):
    """FP64 GMRES(30): the fixed-order reductions give the same restart count
    whatever the number of CTAs that produced the partial sums."""
    counts = []
    for cap in (0, 2, 7):
        s = _solver(mid, "fp64", "gmres30", max_ctas=cap)
        s.solve()
        counts.append(s.iterative_solver.last_iterations)
    assert max(counts) - min(counts) <= 30, counts


@pytest.mark.parametrize("precision", ["mixed", "bf16"])
@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4, 5])
def test_arnoldi_kernel_variants(mid, precision, variant):
    """Every kernel form (orthogonalisation: bulk-copy tile ring or per-thread
    cp.async pipeline; bfloat16 recycled pair: tcgen05 or mma.sync; bfloat16
    stencil: packed-bf16 or complex64 row coefficients) gives the reference's
    solutions on the capped grid, plain and recycled."""
    for algorithm in ("gmres30", "gcrodr36_8"):
        s = _solver(mid, precision, algorithm)
        s.iterative_solver.kernel_variant = variant
        cols = s.sources.column_rhs(s.transducers.amplitudes)[:3]
        x = s.solve_rhs_device(cols).cpu().numpy()
        G = mid["G"].astype(np.complex128)
        for k in range(3):
            assert rel(x[k], G[:, k]) <= TOL, (algorithm, k)


@pytest.mark.parametrize("recycle", [4, 8])
def test_recycled_pair_tensor_core_forms_agree(mid, recycle):
    """bfloat16 GCRO-DR(36,k): the new recycled pair from tcgen05.mma (the
    default for k = 4, 8) and from mma.sync (kernel_variant bit) both give the
    reference's solutions, forward and adjoint, with the same iteration count
    within a few restart cycles (the two products round differently)."""
    from ultrasound_solver_b200 import _native as N
    cols = None
    counts = {}
    for variant in (0, N.GMRES_COMBINE_MMA_SYNC):
        s = golden_solver(mid, precision="bf16", gmres_rtol=1e-10, gmres_maxiter=200000,
                          gmres_max_ctas=3, gmres_restart=36, gmres_recycle=recycle,
                          gmres_recycle_every=2)
        it = s.iterative_solver
        it.kernel_variant = variant
        if cols is None:
            cols = s.sources.column_rhs(s.transducers.amplitudes)[:3]
        x = it.solve(s.operator, cols).cpu().numpy()
        counts[variant] = it.last_iterations
        G = mid["G"].astype(np.complex128)
        for k in range(3):
            assert rel(x[k], G[:, k]) <= TOL, (variant, k)
        rhs, sol = _adjoint_batch(mid, 2)
        lam = it.solve(s.operator, torch.from_numpy(rhs.T.copy()).cuda(), adjoint=True)
        for k in range(2):
            assert rel(lam[k].cpu().numpy(), sol[:, k]) <= TOL, (variant, "adjoint", k)
    assert abs(counts[0] - counts[N.GMRES_COMBINE_MMA_SYNC]) <= 4 * 36, counts
