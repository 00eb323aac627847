"""GPU parity against the reference-generated goldens (through the C ABI)."""
import numpy as np
import pytest
import torch

from oracle import helmholtz_oracle as O
from tests.helpers import golden_matrix, golden_solver, rel

pytestmark = pytest.mark.gpu


def test_materials_and_sources(golden):
    s = golden_solver(golden)
    op = s.operator
    np.testing.assert_allclose(op.rho.cpu().numpy(), golden["rho"].ravel(order="F"), rtol=1e-13)
    np.testing.assert_allclose(op.c.cpu().numpy(), golden["c"].ravel(order="F"), rtol=1e-13)
    nxy = int(golden["shape"][0] * golden["shape"][1])
    B = (s.sources.mass_matrix.cpu().numpy().T * (-2 * np.pi / (s.sources.reference_density
                                                             * s.cfg.domain.dx ** 3)))
    np.testing.assert_allclose(B, golden["B_top"], rtol=1e-13, atol=1e-13 * np.abs(B).max())
    assert rel(s.update_rhs(), golden["rhs"]) < 1e-13
    np.testing.assert_array_equal(op.fixed_dofs(), golden["fixed"])


def test_operator_apply_matches_reference_matrix(golden):
    s = golden_solver(golden)
    A = golden_matrix(golden)
    x = torch.from_numpy(golden["x_rand"]).cuda()
    from ultrasound_solver_b200 import _native as N
    y = s.operator.apply(x, N.APPLY_A).cpu().numpy()
    assert rel(y, golden["Ax_rand"]) < 1e-13
    yh = s.operator.apply(x, N.APPLY_AH).cpu().numpy()
    assert rel(yh, golden["AHx_rand"]) < 1e-13
    ya = s.operator.apply(x, N.APPLY_ABS_A).cpu().numpy()
    assert rel(ya.real, abs(A) @ np.abs(golden["x_rand"])) < 1e-13
    yah = s.operator.apply(x, N.APPLY_ABS_AH).cpu().numpy()
    assert rel(yah.real, abs(A.conj().T) @ np.abs(golden["x_rand"])) < 1e-13


def test_scaled_jacobi_operator(golden):
    """K = R A diag(inv_d) with the reference's row scale / Jacobi (iterative_solver.py:37-56)."""
    from ultrasound_solver_b200 import _native as N
    s = golden_solver(golden)
    A = golden_matrix(golden)
    x = golden["x_rand"]
    for adj, mat, var in ((False, A, N.APPLY_K), (True, A.conj().T.tocsr(), N.APPLY_KH)):
        R, inv_d = O.row_scale_and_jacobi(mat)
        want = R * (mat @ (inv_d * x))
        got = s.operator.apply(torch.from_numpy(x).cuda(), var, N.PREC_FP64).cpu().numpy()
        assert rel(got, want) < 1e-12
        got32 = s.operator.apply(torch.from_numpy(x).cuda().to(torch.complex64), var,
                                 N.PREC_MIXED).cpu().numpy()
        assert rel(got32, want) < 2e-6
        diag, rs, jac, rsa, jaca = s.operator.export()
        np.testing.assert_allclose((rsa if adj else rs).cpu().numpy(), R, rtol=1e-13)
        np.testing.assert_allclose((jaca if adj else jac).cpu().numpy(), inv_d, rtol=1e-12)


@pytest.mark.parametrize("kernel", ["coef_rows", "record_tiles"])
@pytest.mark.parametrize("nrhs", [1, 2, 3, 4, 5, 8, 11])
def test_mixed_apply_batches(golden, nrhs, kernel):
    """Complex64 K / K^H on a batch (coefficient rows: one-, two- and
    per-node-loop kernels by batch size; record tiles: z-marching kernel from
    the 16-byte node records, up to 4 right-hand sides) against the FP64 rows
    of every column."""
    from ultrasound_solver_b200 import _native as N
    k = {"coef_rows": N.STENCIL_COEF_ROWS, "record_tiles": N.STENCIL_RECORD_TILES}[kernel]
    if k == N.STENCIL_RECORD_TILES and nrhs > 4:
        pytest.skip("the record-tile kernel takes at most 4 right-hand sides")
    s = golden_solver(golden)
    rng = np.random.default_rng(nrhs)
    x = rng.standard_normal((nrhs, s.operator.n)) + 1j * rng.standard_normal((nrhs, s.operator.n))
    xt = torch.from_numpy(x).cuda()
    for var in (N.APPLY_K, N.APPLY_KH):
        got = s.operator.apply(xt.to(torch.complex64), var, N.PREC_MIXED, kernel=k).cpu().numpy()
        want = s.operator.apply(xt, var, N.PREC_FP64).cpu().numpy()
        for b in range(nrhs):
            assert rel(got[b], want[b]) < 2e-6


@pytest.mark.parametrize("precision", ["fp64", "mixed", "bf16"])
def test_forward_solve_matches_direct(golden, precision):
    s = golden_solver(golden, precision=precision, gmres_rtol=1e-10, gmres_maxiter=20000)
    field = s.solve()
    want = golden["x_direct"].reshape(tuple(golden["shape"]), order="F")
    assert rel(field, want) <= 1e-6
    it = s.iterative_solver
    assert it.last_scaled_residual <= 1e-10 and it.last_backward_error < 1e-8
    assert it.last_iterations % 30 == 0


@pytest.mark.parametrize("precision", ["fp64", "mixed", "bf16"])
def test_adjoint_solve_matches_direct(golden, precision):
    s = golden_solver(golden, precision=precision, gmres_rtol=1e-10, gmres_maxiter=20000)
    lam = s.solve_adjoint(golden["adj_rhs"])
    want = golden["adj_sol"].reshape(tuple(golden["shape"]), order="F")
    assert rel(lam, want) <= 1e-6


def test_iteration_count_matches_restated_gmres(golden):
    """FP64 GPU GMRES takes the same number of restart cycles as the CPU restatement."""
    s = golden_solver(golden, precision="fp64", gmres_rtol=1e-8, gmres_maxiter=20000)
    s.solve()
    ours = s.iterative_solver.last_iterations
    ref = O.iterative_solve(golden_matrix(golden), golden["rhs"], restart=30, maxiter=20000,
                            rtol=1e-8)
    assert abs(ours - ref.iterations) <= 30, (ours, ref.iterations)


@pytest.mark.parametrize("precision", ["mixed", "bf16"])
def test_batched_solve_matches_columns(golden, precision):
    s = golden_solver(golden, precision=precision, gmres_rtol=1e-10, gmres_maxiter=20000)
    m = s.transducers.num_transducers
    rhs = s.sources.column_rhs(s.transducers.amplitudes)
    x = s.solve_rhs_device(rhs).cpu().numpy()
    G = golden["G"]
    for k in range(m):
        assert rel(x[k], G[:, k]) <= 1e-6
    # host API with (N, nrhs) arrays returns the same
    xh = s.solve_rhs(rhs.cpu().numpy().T, verbose=False)
    assert xh.shape == (s.total_dofs, m)
    assert rel(xh, G) <= 1e-6


def test_zero_rhs_short_circuits(golden):
    s = golden_solver(golden)
    x = s.solve_rhs(np.zeros(s.total_dofs, complex), verbose=False)
    assert np.all(x == 0) and s.iterative_solver.last_iterations == 0


def test_maxiter_failure_raises(golden):
    s = golden_solver(golden, gmres_rtol=1e-14, gmres_maxiter=30)
    with pytest.raises(RuntimeError, match=r"info=30, iterations=30, scaled residual="):
        s.solve()


def test_material_vjp(golden):
    s = golden_solver(golden, precision="fp64", gmres_rtol=1e-12, gmres_maxiter=20000)
    shape = tuple(golden["shape"])
    u = golden["x_direct"].reshape(shape, order="F")
    gr, gc = s.material_vjp(u, golden["adj_rhs"])
    assert rel(gr.ravel(order="F"), golden["vjp_rho"].ravel(order="F")) < 1e-6
    assert rel(gc.ravel(order="F"), golden["vjp_c"].ravel(order="F")) < 1e-6


@pytest.mark.parametrize("precision", ["fp64", "mixed", "bf16"])
def test_recycled_gmres_matches_direct(golden, precision):
    """GCRO-DR(30, 8) cycles (recycled harmonic Ritz space, lagged host update) reach the
    reference direct solution, forward and adjoint, and a batch of columns."""
    s = golden_solver(golden, precision=precision, gmres_rtol=1e-10, gmres_maxiter=20000,
                      gmres_recycle=8)
    field = s.solve()
    want = golden["x_direct"].reshape(tuple(golden["shape"]), order="F")
    assert rel(field, want) <= 1e-6
    it = s.iterative_solver
    assert it.last_scaled_residual <= 1e-10 and it.last_backward_error < 1e-8
    lam = s.solve_adjoint(golden["adj_rhs"])
    assert rel(lam, golden["adj_sol"].reshape(tuple(golden["shape"]), order="F")) <= 1e-6
    m = s.transducers.num_transducers
    x = s.solve_rhs_device(s.sources.column_rhs(s.transducers.amplitudes)).cpu().numpy()
    for k in range(m):
        assert rel(x[k], golden["G"][:, k]) <= 1e-6


@pytest.mark.parametrize("k", [1, 3, 5, 13])
def test_recycled_bf16_other_sizes(k):
    """bfloat16 GCRO-DR(30, k) with recycled-space sizes whose tensor-core tiles
    are partly empty (k = 1, 3, 5, 13) reaches the direct solution for a batch
    of columns."""
    from tests.conftest import load_golden
    g = load_golden("mixed")
    s = golden_solver(g, precision="bf16", gmres_rtol=1e-10, gmres_maxiter=20000,
                      gmres_recycle=k, gmres_recycle_every=1)
    cols = s.sources.column_rhs(s.transducers.amplitudes)[:3]
    x = s.solve_rhs_device(cols).cpu().numpy()
    for c in range(x.shape[0]):
        assert rel(x[c], g["G"][:, c]) <= 1e-6


def test_recycling_reduces_iterations(golden):
    """On a scene where restarted GMRES(30) needs many cycles, deflated restarting with
    8 recycled vectors needs fewer inner iterations to the same residual."""
    plain = golden_solver(golden, precision="fp64", gmres_rtol=1e-10, gmres_maxiter=20000)
    plain.solve()
    rec = golden_solver(golden, precision="fp64", gmres_rtol=1e-10, gmres_maxiter=20000,
                        gmres_recycle=8)
    rec.solve()
    n_plain = plain.iterative_solver.last_iterations
    n_rec = rec.iterative_solver.last_iterations
    if n_plain > 120:
        assert n_rec < n_plain, (n_rec, n_plain)


def test_recycle_argument_checks(golden):
    from ultrasound_solver_b200 import _native as N
    s = golden_solver(golden, gmres_recycle=30)  # k must stay below the restart length
    with pytest.raises(ValueError):
        s.solve()
    s = golden_solver(golden, gmres_recycle=17)  # at most 16
    with pytest.raises(ValueError):
        s.solve()
    assert N.load() is not None
