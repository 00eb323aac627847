"""Pin the CPU oracle against vectors produced by the reference's own code."""
import json

import numpy as np
import scipy.sparse as sp

from oracle import helmholtz_oracle as O
from tests.conftest import load_golden


def _scene(g):
    cfg = json.loads(str(g["cfg_json"]))
    fields = (g["material_rho"], g["material_c"]) if "material_rho" in g else None
    return cfg, O.build_scene(cfg, material_fields=fields, phases=g["phases"])


def _ref_matrix(g):
    n = int(np.prod(g["shape"]))
    return sp.csr_matrix((g["A_data"], g["A_indices"], g["A_indptr"]), shape=(n, n))


def test_blend_known_answer():
    g = load_golden("blend")
    rho, c = O.blend_obstacle_material(g["h"], 1250.0, 2200.0, 1.21, 346.0)
    np.testing.assert_allclose(rho, g["rho"], rtol=1e-15)
    np.testing.assert_allclose(c, g["c"], rtol=1e-15)
    np.testing.assert_allclose([rho[0], c[0], rho[-1], c[-1]], [1250.0, 2200.0, 1.21, 346.0])
    np.testing.assert_allclose(np.diff(1 / rho, 2), 0, atol=1e-12)


def test_materials_match(golden):
    _, sc = _scene(golden)
    np.testing.assert_allclose(sc.rho, golden["rho"], rtol=1e-14)
    np.testing.assert_allclose(sc.c, golden["c"], rtol=1e-14)


def test_matrix_matches_reference(golden):
    _, sc = _scene(golden)
    A_ref = _ref_matrix(golden)
    A = sc.A.tocsr()
    A.sort_indices()
    assert A.nnz == A_ref.nnz
    np.testing.assert_array_equal(A.indptr, A_ref.indptr)
    np.testing.assert_array_equal(A.indices, A_ref.indices)
    scale = np.abs(A_ref.data).max()
    np.testing.assert_allclose(A.data, A_ref.data, rtol=1e-13, atol=1e-15 * scale)
    np.testing.assert_array_equal(np.flatnonzero(sc.op.fixed.ravel(order="F")), golden["fixed"])


def test_sources_and_rhs_match(golden):
    _, sc = _scene(golden)
    nxy = golden["shape"][0] * golden["shape"][1]
    np.testing.assert_allclose(sc.B[:nxy].toarray(), golden["B_top"], rtol=1e-13,
                               atol=1e-13 * np.abs(golden["B_top"]).max())
    assert sc.B[nxy:].nnz == 0
    np.testing.assert_allclose(sc.centers, golden["centers"], rtol=0, atol=1e-15)
    np.testing.assert_allclose(sc.rhs, golden["rhs"], rtol=1e-12, atol=1e-12 * np.abs(golden["rhs"]).max())


def test_direct_solution_and_adjoint(golden):
    _, sc = _scene(golden)
    x = O.direct_solve(sc.A, sc.rhs)
    err = np.linalg.norm(x - golden["x_direct"]) / np.linalg.norm(golden["x_direct"])
    assert err < 1e-10
    lam = O.direct_solve(sc.A.conj().T, golden["adj_rhs"])
    err = np.linalg.norm(lam - golden["adj_sol"]) / np.linalg.norm(golden["adj_sol"])
    assert err < 1e-10


def test_material_vjp(golden):
    _, sc = _scene(golden)
    gr, gc = sc.op.material_vjp(golden["x_direct"], golden["adj_sol"])
    np.testing.assert_allclose(gr, golden["vjp_rho"], rtol=1e-10, atol=1e-12 * np.abs(golden["vjp_rho"]).max())
    np.testing.assert_allclose(gc, golden["vjp_c"], rtol=1e-10, atol=1e-12 * np.abs(golden["vjp_c"]).max())


def test_basis_ops(golden):
    cfg, sc = _scene(golden)
    G = golden["G"]
    shape = tuple(golden["shape"])
    f = O.basis_field(G, golden["phi2"]).reshape(shape, order="F")
    np.testing.assert_allclose(f, golden["field_phi2"], rtol=1e-12, atol=1e-14 * np.abs(f).max())
    v = O.basis_phase_vjp(G, golden["cot"], golden["phi2"])
    np.testing.assert_allclose(v, golden["phase_vjp"], rtol=1e-11, atol=1e-13 * np.abs(v).max())
    tr = O.basis_target_response(G, golden["target_points"], shape, sc.dx)
    np.testing.assert_allclose(tr, golden["target_response"], rtol=1e-12)


def test_losses(golden):
    cfg, sc = _scene(golden)
    field = golden["field_phi2"]
    tr = cfg["training"]
    idx = [O.nearest_index(t["point"], sc.dx) for t in cfg["targets"]]
    np.testing.assert_array_equal(np.asarray(idx), golden["target_indices"])
    loss, cot = O.focal_pressure_loss(field, idx, 1.0, tr["background_weight"])
    assert abs(loss - float(golden["fp_loss"])) <= 1e-12 * abs(float(golden["fp_loss"]))
    np.testing.assert_allclose(cot, golden["fp_cot"], rtol=1e-12, atol=1e-18)
    box = cfg["domain"]["box_size"]
    mask = O.background_mask(shape=tuple(golden["shape"]), box=box,
                             targets=[t["point"] for t in cfg["targets"]],
                             target_radius=tr["target_radius"],
                             exclusion_layers=tr["source_exclusion_layers"])
    np.testing.assert_array_equal(mask, golden["fc_mask"])
    loss, cot = O.focal_contrast_loss(field, idx, mask, 1.0, tr["background_weight"],
                                      tr["sidelobe_temperature"])
    assert abs(loss - float(golden["fc_loss"])) <= 1e-12 * abs(float(golden["fc_loss"]))
    np.testing.assert_allclose(cot, golden["fc_cot"], rtol=1e-12, atol=1e-18)


def test_gmres_restatement_converges_to_direct(golden):
    """The restated row-scaled Jacobi GMRES reaches the direct solution."""
    _, sc = _scene(golden)
    res = O.iterative_solve(sc.A, sc.rhs, restart=30, maxiter=20000, rtol=1e-10)
    assert res.iterations % 30 == 0 and res.info == 0
    err = np.linalg.norm(res.x - golden["x_direct"]) / np.linalg.norm(golden["x_direct"])
    assert err < 1e-6
    assert res.scaled_residual <= 1e-10
    assert res.backward_error < 1e-8


def test_mid_scene_assembly_and_solutions():
    """Mid-size golden (36 x 32 x 30, random medium, blended sphere, every face
    kind): the oracle's assembly against the reference's A x for a probe, its
    sources, and the reference's direct solutions as residuals of its matrix."""
    g = load_golden("mid")
    _, sc = _scene(g)
    n = int(np.prod(g["shape"]))
    t = np.arange(n, dtype=np.float64)
    probe = np.cos(0.37 * t) + 1j * np.sin(0.11 * t + 0.5)
    ax = sc.A @ probe
    assert np.linalg.norm(ax - g["Ax_probe"]) <= 1e-13 * np.linalg.norm(g["Ax_probe"])
    nxy = int(g["shape"][0] * g["shape"][1])
    np.testing.assert_allclose(sc.B[:nxy].toarray(), g["B_top"], rtol=1e-13,
                               atol=1e-13 * np.abs(g["B_top"]).max())
    assert np.linalg.norm(sc.rhs - g["rhs"]) <= 1e-13 * np.linalg.norm(g["rhs"])
    np.testing.assert_array_equal(np.flatnonzero(sc.op.fixed.ravel(order="F")), g["fixed"])
    # the stored solutions solve the oracle's system up to their complex64
    # rounding (6e-8 per value; ||A|| ||x|| / ||b|| ~ 20 turns it into ~1e-6 of
    # residual; a wrong assembly leaves O(1))
    def resid(M, x, b):
        return np.linalg.norm(M @ x - b) / np.linalg.norm(b)
    for k in range(g["G"].shape[1]):
        assert resid(sc.A, g["G"][:, k].astype(np.complex128), sc.B[:, k].toarray().ravel()) < 1e-5
    AH = sc.A.conj().T.tocsr()
    for k in range(g["adj_sol"].shape[1]):
        assert resid(AH, g["adj_sol"][:, k].astype(np.complex128),
                     g["adj_rhs"][:, k].astype(np.complex128)) < 1e-5
