"""Config-4 phase optimisation, reduced to 40^3 (h = 1 mm, 4 x 4 array): three
Adam steps (lr 0.05, the reference's adjoint baseline) on the device against
the oracle's trajectory (direct forward and A^H solves of the oracle's
assembly, the same Adam arithmetic), on the config-4 scene layout: random
medium, rotated ellipsoid SDF blended into it, +x reflecting, -y impedance
2 rho c, PML on the open faces, focal pressure at two targets."""
import numpy as np
import pytest

from oracle import helmholtz_oracle as O

pytestmark = pytest.mark.gpu


def _oracle(cfg, phases0, steps):
    from ultrasound_solver_b200 import workloads as W
    shape = tuple(cfg["domain"]["grid_size"])
    rho_m, c_m = W.random_medium(shape, 0)
    dx = cfg["domain"]["box_size"][0] / (shape[0] - 1)
    h = O.smoothed_heaviside(W.config4_sdf(cfg), 1.2 * dx)
    rho, c = O.blend_obstacle_material(h, 1250.0, 2200.0, rho_m, c_m)
    plain = dict(cfg)
    plain["obstacles"] = []
    sc = O.build_scene(plain, material_fields=(rho, c), phases=phases0)
    idx = [O.nearest_index(t["point"], sc.dx) for t in cfg["targets"]]
    tr = cfg["training"]

    def loss_fn(u):
        L, cot = O.focal_pressure_loss(u.reshape(shape, order="F"), idx, tr["target_weight"],
                                       tr["background_weight"])
        return L, cot.ravel(order="F")
    return O.adam_trajectory(sc.A, sc.B, np.ones(sc.B.shape[1]), phases0, loss_fn, steps)


@pytest.mark.parametrize("precision,recycle", [("bf16", 8), ("fp64", 0)])
def test_adam_trajectory_matches_oracle(precision, recycle):
    from ultrasound_solver_b200 import workloads as W
    from ultrasound_solver_b200.adjoint_optimizer import adam
    from ultrasound_solver_b200.losses import FocalPressureLoss
    cfg = W.config4(40, 1e-3, 4)
    s = W.build_solver(cfg, seed=0, sdf=W.config4_sdf(cfg))
    s.assemble_matrix()
    it = s.iterative_solver
    it.precision, it.rtol, it.maxiter = precision, 1e-11, 400000
    it.restart, it.recycle, it.recycle_every = (36, recycle, 2) if recycle else (30, 0, 1)
    phases0 = np.random.default_rng(1).uniform(0, 2 * np.pi, s.transducers.num_transducers)
    steps = 3
    seen = []
    res = adam(s, FocalPressureLoss(s.cfg), phases0, steps, 0.05,
               callback=lambda step, ev: seen.append(ev))
    ph_o, loss_o, grad_o = _oracle(cfg, phases0, steps)
    assert res.steps == steps and len(res.losses) == steps + 1
    for k in range(steps + 1):
        assert abs(res.losses[k] - loss_o[k]) <= 1e-8 * abs(loss_o[k]), (k, res.losses[k], loss_o[k])
    for k, ev in enumerate(seen, start=1):
        np.testing.assert_allclose(ev.phases, ph_o[k], rtol=0, atol=1e-8)
        assert np.linalg.norm(ev.gradient - grad_o[k]) <= 1e-7 * np.linalg.norm(grad_o[k])
    assert res.losses[-1] < res.losses[0]
