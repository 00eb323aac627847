"""Golden fixture for the homogeneous surface solver, from the reference itself.

    python tests/golden/make_golden_surface.py /path/to/ultrasound_solver

Runs the reference's HomogeneousSurfaceSolver (src/algorithm/solvers/
homogeneous_surface.py, CPU path) and source_mass_matrix
(src/algorithm/physics/sinc_aperture.py) on a small homogeneous scene and
writes golden_surface.npz: the masses, phases, the z=0 surface after
solve_flux, one interior plane, trilinear samples and flux_target_response
rows. The reference's GPU-only imports (pulled in by its package
__init__) are replaced by the inert stubs of make_golden.py.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent

SHAPE = (16, 15, 14)
DX = 1.0e-3
FREQ = 40000.0
C0, RHO0 = 343.0, 1.2
BOUNDARIES = {"-x": "open", "+x": "open", "-y": "open",
              "+y": {"type": "impedance", "impedance": [800.0, -120.0]},
              "-z": "reflecting", "+z": "open"}
PML = {"cells": 3, "strength": 2.0, "order": 2, "faces": ["-x", "+x", "-y", "+z"]}
CENTERS = np.array([[0.0065, 0.0062, 0.0], [0.0088, 0.0071, 0.0], [0.0071, 0.0090, 0.0]])
DIAMETER = 0.0021
POINTS = np.array([[0.0075, 0.0070, 0.0060], [0.0062, 0.0081, 0.0093], [0.0090, 0.0064, 0.0021],
                   [0.0080, 0.0080, 0.0]])


def main(ref_root: str) -> None:
    sys.path.insert(0, str(HERE))
    from make_golden import _install_stubs
    _install_stubs()
    sys.path.insert(0, str(Path(ref_root) / "src"))
    from algorithm.physics.sinc_aperture import source_mass_matrix
    from algorithm.solvers.homogeneous_surface import HomogeneousSurfaceSolver
    masses = source_mass_matrix(SHAPE[:2], DX, CENTERS, DIAMETER, 12, 24)
    solver = HomogeneousSurfaceSolver(SHAPE, DX, FREQ, C0, RHO0, BOUNDARIES, pml=PML, device="cpu")
    phases = np.random.default_rng(7).uniform(0, 2 * np.pi, len(CENTERS))
    amplitudes = np.array([1.0, 0.8, 1.3])
    solver.solve_flux(masses, phases, amplitudes)
    np.savez_compressed(
        HERE / "golden_surface.npz",
        shape=np.array(SHAPE), dx=DX, frequency=FREQ, c0=C0, rho0=RHO0,
        masses=masses.toarray(), phases=phases, amplitudes=amplitudes, points=POINTS,
        surface=solver.plane(0), plane5=solver.plane(5), plane_top=solver.plane(SHAPE[2] - 1),
        samples=solver.sample(POINTS), response=solver.flux_target_response(masses, POINTS),
        schur=np.asarray(solver.schur), h_last=np.asarray(solver.h[-1]))
    print("wrote", HERE / "golden_surface.npz")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden_surface.py REFERENCE_ROOT   (the checkout that holds src/algorithm)")
    main(sys.argv[1])
