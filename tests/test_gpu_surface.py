"""Homogeneous surface solver (z-transfer kernel + modal transforms) against the
reference's own HomogeneousSurfaceSolver (golden_surface.npz, make_golden_surface.py)."""
import numpy as np
import pytest

from tests.conftest import load_golden

pytestmark = pytest.mark.gpu


def _solver(g):
    from ultrasound_solver_b200.homogeneous_surface import HomogeneousSurfaceSolver
    from tests.golden.make_golden_surface import BOUNDARIES, PML
    return HomogeneousSurfaceSolver(tuple(g["shape"]), float(g["dx"]), float(g["frequency"]),
                                    float(g["c0"]), float(g["rho0"]), BOUNDARIES, pml=PML)


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - b) / np.linalg.norm(b))


def test_surface_solver_matches_reference():
    g = load_golden("surface")
    s = _solver(g)
    assert rel(s.h[-1].cpu().numpy(), g["h_last"]) < 1e-11
    assert rel(s.schur.cpu().numpy(), g["schur"]) < 1e-11
    s.solve_flux(g["masses"], g["phases"], g["amplitudes"])
    assert rel(s.plane(0), g["surface"]) < 1e-11
    assert rel(s.plane(5), g["plane5"]) < 1e-11
    assert rel(s.plane(int(g["shape"][2]) - 1), g["plane_top"]) < 1e-10
    assert rel(s.sample(g["points"]), g["samples"]) < 1e-11
    assert rel(s.flux_target_response(g["masses"], g["points"]), g["response"]) < 1e-11


def test_surface_solver_checks():
    g = load_golden("surface")
    s = _solver(g)
    bad = g["masses"].copy()
    bad[0, 0] = 1.0  # a source on the side boundary
    with pytest.raises(ValueError, match="overlaps PML or side boundaries"):
        s.solve_flux(bad, g["phases"])
    with pytest.raises(ValueError, match="inside the local grid"):
        s.sample(np.array([[1.0, 0.0, 0.0]]))
    from ultrasound_solver_b200.homogeneous_surface import HomogeneousSurfaceSolver
    with pytest.raises(ValueError, match="open/reflecting/impedance"):
        HomogeneousSurfaceSolver((8, 8, 8), 1e-3, 4e4, 343.0, 1.2, {"+z": "soft"})


def test_solver_target_response_cache(tmp_path, monkeypatch):
    """HelmholtzB200Solver.target_response with solver.target_response_cache:
    the second call reads every response back from the store (no solve), a
    new point is computed and added, and a different scene ignores the file."""
    from ultrasound_solver_b200 import workloads as W
    from ultrasound_solver_b200.config import SimulationConfig
    from ultrasound_solver_b200.helmholtz_solver import HelmholtzB200Solver
    from ultrasound_solver_b200.homogeneous_surface import HomogeneousSurfaceSolver

    def make(freq):
        d = W.scene_dict(24, 1e-3, 2, 6e-3, 4e-3, radial=8, angular=16)
        d["transducer_specs"]["frequency"] = freq
        d["solver"]["pml"] = {"cells": 4, "strength": 2.0, "order": 2}
        d["solver"]["target_response_cache"] = str(tmp_path / "resp.npz")
        return HelmholtzB200Solver(SimulationConfig.from_dict(d))

    pts = np.array([[0.0115, 0.0115, 0.010], [0.010, 0.012, 0.013]])
    s = make(40000.0)
    first = s.target_response(pts)
    assert (tmp_path / "resp.npz").exists()
    calls = []
    orig = HomogeneousSurfaceSolver.flux_target_response

    def counting(self, masses, points):
        calls.append(len(points))
        return orig(self, masses, points)

    monkeypatch.setattr(HomogeneousSurfaceSolver, "flux_target_response", counting)
    again = make(40000.0).target_response(pts)
    assert calls == [] and np.array_equal(again, first)
    more = np.vstack((pts, [[0.012, 0.011, 0.008]]))
    out = make(40000.0).target_response(more)
    assert calls == [1] and np.array_equal(out[:2], first)
    other = make(41000.0).target_response(pts)  # another scene: recomputed
    assert calls == [1, 2] and not np.allclose(other, first)
