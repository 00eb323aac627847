"""Phase basis, device losses and the autograd adjoint gradient against the goldens."""
import json

import numpy as np
import pytest
import torch

from oracle import helmholtz_oracle as O
from tests.helpers import golden_config, golden_matrix, golden_solver, rel

pytestmark = pytest.mark.gpu


def _basis(g, tmp_path, **kw):
    from ultrasound_solver_b200.phase_response_basis import PhaseResponseBasis
    s = golden_solver(g, precision="mixed", gmres_rtol=1e-11, gmres_maxiter=40000)
    return s, PhaseResponseBasis(s, str(tmp_path / "basis.npy"), **kw)


@pytest.mark.parametrize("device_precision", ["complex128", "complex64"])
def test_basis_build_and_queries(golden, tmp_path, device_precision):
    s, basis = _basis(golden, tmp_path, rhs_batch_size=3, device_precision=device_precision)
    basis.build()
    assert basis.is_complete
    G = golden["G"]
    assert basis.basis.shape == G.shape and basis.basis.dtype == np.complex128
    assert rel(np.asarray(basis.basis), G) <= 1e-6
    tol = 1e-6
    f = basis.field(golden["phi2"])
    assert rel(f, golden["field_phi2"]) <= tol
    v = basis.phase_vjp(golden["cot"], golden["phi2"])
    assert rel(v, golden["phase_vjp"]) <= tol
    tr = basis.target_response(golden["target_points"])
    assert rel(tr, golden["target_response"]) <= tol
    meta = json.loads((tmp_path / "basis.npy.json").read_text())
    assert meta["format_version"] == 3 and meta["completed_columns"] == G.shape[1]
    assert meta["shape"] == list(G.shape) and meta["dtype"] == "complex128"
    basis.close()


def test_basis_resumes_after_interruption(tmp_path):
    from tests.conftest import load_golden
    g = load_golden("air_pml")
    s, basis = _basis(g, tmp_path, rhs_batch_size=2)
    real = s.solve_rhs_device
    calls = {"n": 0}

    def flaky(rhs, adjoint=False):
        calls["n"] += 1
        if calls["n"] == 2:
            raise KeyboardInterrupt("simulated interruption")
        return real(rhs, adjoint)

    s.solve_rhs_device = flaky
    with pytest.raises(KeyboardInterrupt):
        basis.build()
    basis.close()
    meta = json.loads((tmp_path / "basis.npy.json").read_text())
    assert meta["completed_columns"] == 2
    s.solve_rhs_device = real
    from ultrasound_solver_b200.phase_response_basis import PhaseResponseBasis
    again = PhaseResponseBasis(s, str(tmp_path / "basis.npy"), rhs_batch_size=2).build()
    assert again.is_complete and calls["n"] == 2
    assert rel(np.asarray(again.basis), g["G"]) <= 1e-6
    # a changed scene is refused
    s.cfg.physics.sound_speed = 345.0
    with pytest.raises((RuntimeError, ValueError)):
        PhaseResponseBasis(s, str(tmp_path / "basis.npy")).build()
    again.close()


def test_losses_match_reference(golden):
    from ultrasound_solver_b200.losses import FocalContrastLoss, FocalPressureLoss
    cfg = golden_config(golden)
    torch.cuda.set_device(0)
    field = golden["field_phi2"]
    fp = FocalPressureLoss(cfg)
    assert np.asarray(fp.target_indices).tolist() == golden["target_indices"].tolist()
    loss, cot = fp.evaluate(field)
    assert abs(loss - float(golden["fp_loss"])) <= 1e-12 * abs(float(golden["fp_loss"]))
    np.testing.assert_allclose(cot, golden["fp_cot"], rtol=1e-12, atol=1e-18)
    fc = FocalContrastLoss(cfg)
    np.testing.assert_array_equal(fc.background_mask, golden["fc_mask"])
    loss, cot = fc.evaluate(field)
    assert abs(loss - float(golden["fc_loss"])) <= 1e-12 * abs(float(golden["fc_loss"]))
    np.testing.assert_allclose(cot, golden["fc_cot"], rtol=1e-11, atol=1e-18)


def test_contrast_ratio_cotangent_is_the_gradient(golden):
    from ultrasound_solver_b200.losses import ContrastRatioLoss
    cfg = golden_config(golden)
    torch.cuda.set_device(0)
    L = ContrastRatioLoss(cfg, cfg.targets[0], focal_radius=0.0008, shell_thickness=0.002)
    rng = np.random.default_rng(5)
    u = torch.from_numpy(golden["field_phi2"].reshape(-1, order="F").copy()).cuda()
    du = torch.from_numpy(rng.standard_normal(u.numel()) + 1j * rng.standard_normal(u.numel())).cuda()
    du *= torch.linalg.norm(u) / torch.linalg.norm(du)
    val, cot = L.evaluate_vector(u)
    mask = torch.from_numpy(L.shell_mask.reshape(-1, order="F")).cuda()
    t = int(L._targets[0])
    ref = -(abs(u[t]) ** 2) / (abs(u[mask]) ** 2).mean()
    assert abs(float(val) - float(ref)) <= 1e-12 * abs(float(ref))
    eps = 1e-6
    lp, _ = L.evaluate_vector(u + eps * du, False)
    lm, _ = L.evaluate_vector(u - eps * du, False)
    fd = (float(lp) - float(lm)) / (2 * eps)
    an = float(torch.real(torch.vdot(cot, du)))
    assert abs(fd - an) <= 1e-6 * abs(an)


@pytest.mark.parametrize("precision", ["fp64", "mixed", "bf16"])
def test_autograd_phase_gradient(golden, precision):
    """Adjoint gradient through PhaseField vs central differences and the FP64 oracle adjoint."""
    from ultrasound_solver_b200.autograd import loss_of_field, phase_field
    from ultrasound_solver_b200.losses import FocalPressureLoss
    s = golden_solver(golden, precision=precision, gmres_rtol=1e-12, gmres_maxiter=60000)
    cfg = s.cfg
    cfg.training.background_weight = 0.05
    loss = FocalPressureLoss(cfg)
    phases0 = np.random.default_rng(11).uniform(0, 2 * np.pi, s.transducers.num_transducers)
    ph = torch.tensor(phases0, dtype=torch.float64, device="cuda", requires_grad=True)
    L = loss_of_field(phase_field(ph, s), loss)
    L.backward()
    grad = ph.grad.cpu().numpy()
    if len(phases0) == 1:
        # one emitter: |u| does not depend on the global phase, dL/dphi == 0
        assert abs(grad[0]) <= 1e-6 * abs(float(L))
        return

    def value(p):
        with torch.no_grad():
            u = phase_field(torch.tensor(p, dtype=torch.float64, device="cuda"), s)
            return float(loss.evaluate_vector(u, False)[0])

    h = 1e-4
    fd = np.array([(value(phases0 + h * e) - value(phases0 - h * e)) / (2 * h)
                   for e in np.eye(len(phases0))])
    assert rel(grad, fd) <= 1e-5, (grad, fd)
    # oracle: lambda = A^-H g with the reference matrix, grad = Re(conj(a B^H lam) i e^{i phi})
    A = golden_matrix(golden)
    u = O.direct_solve(A, _rhs(golden, phases0))
    _, cot = O.focal_pressure_loss(u.reshape(tuple(golden["shape"]), order="F"),
                                   [tuple(i) for i in golden["target_indices"]], 1.0, 0.05)
    lam = O.direct_solve(A.conj().T, cot.reshape(-1, order="F"))
    nxy = golden["B_top"].shape[0]
    r = golden["B_top"].T @ lam[:nxy]
    oracle = np.real(np.conj(r) * 1j * np.exp(1j * phases0))
    assert rel(grad, oracle) <= 1e-6


def _rhs(golden, phases):
    n = int(np.prod(golden["shape"]))
    b = np.zeros(n, complex)
    nxy = golden["B_top"].shape[0]
    b[:nxy] = golden["B_top"] @ np.exp(1j * phases)
    return b


def test_target_response_points_outside_the_grid():
    """usv_basis_target_response through the C ABI with a point just below the
    origin (extrapolated from the edge cell, all loads inside the basis), a
    non-finite point (NaN response) and an interior point (the reference's
    trilinear rows)."""
    from ultrasound_solver_b200 import _native as N
    nx, ny, nz, m, dx = 6, 5, 4, 3, 1e-3
    n = nx * ny * nz
    rng = np.random.default_rng(5)
    G = rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n))
    pts = np.array([[-0.3e-3, 1.5e-3, 2.25e-3],
                    [np.nan, 1e-3, 1e-3],
                    [2.6e-3, 3.1e-3, 0.4e-3]])
    dev = torch.device("cuda", 0)
    Gd = torch.from_numpy(G).to(dev)
    pd = torch.from_numpy(pts).to(dev)
    out = torch.empty((3, m), dtype=torch.complex128, device=dev)
    st = N.load().usv_basis_target_response(N.ptr(Gd), nx, ny, nz, m, N.PREC_FP64, N.ptr(pd), 3,
                                            dx, N.ptr(out), N.stream_handle(torch, dev))
    assert st == N.USV_OK
    got = out.cpu().numpy()
    # interior point: the reference's trilinear rows (oracle restatement)
    want = O.basis_target_response(G.T, pts[2:], (nx, ny, nz), dx)[0]
    assert rel(got[2], want) <= 1e-13
    assert np.isnan(got[1]).all()
    # below the origin in x: low corner 0, fraction -0.3 (linear extrapolation)
    pos = pts[0] / dx
    lo = np.array([0, 1, 2])
    fr = pos - lo
    acc = np.zeros(m, complex)
    for ci in (0, 1):
        for cj in (0, 1):
            for ck in (0, 1):
                w = ((fr[0] if ci else 1 - fr[0]) * (fr[1] if cj else 1 - fr[1])
                     * (fr[2] if ck else 1 - fr[2]))
                row = (lo[0] + ci) + nx * ((lo[1] + cj) + ny * (lo[2] + ck))
                acc += w * G[:, row]
    assert rel(got[0], acc) <= 1e-13
