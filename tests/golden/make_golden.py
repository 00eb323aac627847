"""Generate the golden fixtures in this folder from the reference implementation.

Run in a container where the reference project is checked out (read-only is
fine); the output ``*.npz`` files are committed and the tests never read the
reference at run time:

    python tests/golden/make_golden.py /path/to/ultrasound_solver

The reference's GPU-only imports (warp, cupy, cupyx, nvmath) are replaced by
inert stub modules; the reference then runs its own CPU assembly
(HelmholtzDirectSolver.assemble_matrix -> WarpAssemblyEngine ->
ConservativeHelmholtz.assemble, sinc_aperture) and its CPU loss / basis code.
Solutions are scipy direct solves of the reference's assembled matrices.
"""
from __future__ import annotations

import json
import sys
import tempfile
import types
from pathlib import Path

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla
import yaml

HERE = Path(__file__).resolve().parent

# Scenes: small grids (non-cubic) that exercise every boundary kind, PML on
# some faces, a low- and a high-contrast sphere obstacle and explicit fields.
SCENES = {
    "mixed": {
        "mode": "phase_optimization",
        "physics": {"sound_speed": 346.0, "medium_density": 1.21},
        "transducer_specs": {"frequency": 40000.0, "array_n": 2, "diameter": 0.001,
                             "pitch": 0.0025, "geometry": "ideal_grid",
                             "source_radial_order": 16, "source_angular_order": 32},
        "domain": {"box_size": [0.0065, 0.006, 0.0055], "grid_size": [14, 13, 12]},
        "boundary_conditions": {"-x": "reflecting",
                                "+x": {"type": "impedance", "impedance": [500.0, 100.0]},
                                "-y": "soft", "+y": "open", "-z": "reflecting", "+z": "open"},
        "targets": [{"point": [0.0032, 0.0031, 0.0035]}],
        "obstacles": [{"type": "sphere", "center": [0.0033, 0.003, 0.003], "radius": 0.0012,
                       "smoothing_width_cells": 1.2,
                       "material": {"density": 1.6, "sound_speed": 390.0}}],
        "solver": {"pml": {"cells": 2, "strength": 2.0, "order": 3, "faces": ["+y", "+z"]}},
        "training": {"background_weight": 0.05, "target_radius": 0.001,
                     "source_exclusion_layers": 2, "sidelobe_temperature": 25.0},
    },
    "air_pml": {
        "mode": "phase_optimization",
        "physics": {"sound_speed": 343.0, "medium_density": 1.2},
        "transducer_specs": {"frequency": 40000.0, "array_n": 2, "diameter": 0.003,
                             "pitch": 0.004, "geometry": "ideal_grid",
                             "source_radial_order": 16, "source_angular_order": 32},
        "domain": {"box_size": [0.015, 0.015, 0.013], "grid_size": [16, 16, 14]},
        "boundary_conditions": {"-x": "open", "+x": "open", "-y": "open", "+y": "open",
                                "-z": "reflecting", "+z": "open"},
        "targets": [{"point": [0.0075, 0.0075, 0.008]}, {"point": [0.006, 0.008, 0.007]}],
        "obstacles": [{"type": "sphere", "center": [0.0075, 0.0075, 0.006], "radius": 0.002}],
        "solver": {"pml": {"cells": 3, "strength": 2.0, "order": 2}},
        "training": {"background_weight": 0.05, "target_radius": 0.002,
                     "source_exclusion_layers": 3, "sidelobe_temperature": 25.0},
    },
    "fields": {
        "mode": "phase_optimization",
        "physics": {"sound_speed": 343.0, "medium_density": 1.2},
        "transducer_specs": {"frequency": 40000.0, "array_n": 1, "diameter": 0.002,
                             "pitch": 0.004, "geometry": "ideal_grid",
                             "source_radial_order": 8, "source_angular_order": 16},
        "domain": {"box_size": [0.011, 0.009, 0.01], "grid_size": [12, 10, 11]},
        "boundary_conditions": {"-x": "open", "+x": "reflecting",
                                "-y": {"type": "impedance", "impedance": [826.0, -40.0]},
                                "+y": "open", "-z": "reflecting", "+z": "soft"},
        "targets": [{"point": [0.005, 0.004, 0.006]}],
        "obstacles": [],
        "solver": {"pml": {"cells": 2, "strength": 1.5, "order": 2, "faces": ["-x", "+y"]}},
        "training": {"background_weight": 0.0, "target_radius": 0.0015,
                     "source_exclusion_layers": 1, "sidelobe_temperature": 10.0},
    },
}


def _install_stubs():
    class _Any(types.ModuleType):
        def __getattr__(self, key):
            if key.startswith("__"):
                raise AttributeError(key)
            return type(key, (), {})

    def stub(name, **attrs):
        mod = _Any(name)
        mod.__dict__.update(attrs)
        sys.modules[name] = mod
        if "." in name:
            parent, child = name.rsplit(".", 1)
            setattr(sys.modules[parent], child, mod)

    stub("warp", init=lambda: None, is_cuda_available=lambda: False,
         from_numpy=lambda a, **k: a, array=object, float64="float64", complex64="complex64")
    for name in ("cupy", "cupyx", "cupyx.scipy", "cupyx.scipy.sparse",
                 "cupyx.scipy.sparse.linalg", "nvmath", "nvmath.sparse",
                 "nvmath.sparse.advanced"):
        stub(name)


def _yaml_config(cfg):
    full = dict(cfg)
    full.setdefault("io", {"output_file": "unused.npz", "auto_visualize": False})
    return full


def make_scene(name, cfg, reference_src):
    from algorithm.config import SimulationConfig
    from algorithm.solvers.helmholtz_solver import HelmholtzDirectSolver
    from algorithm.training.phase_response_basis import PhaseResponseBasis
    from algorithm.training.phase_adjoint_optimizer import (
        AmplitudeTarget, FocalContrastLoss, FocalPressureLoss)

    rng = np.random.default_rng(sum(map(ord, name)))
    with tempfile.TemporaryDirectory() as tmp:
        path = Path(tmp) / f"{name}.yaml"
        path.write_text(yaml.safe_dump(_yaml_config(cfg)))
        config = SimulationConfig.from_yaml(str(path))
        solver = HelmholtzDirectSolver(config)
        shape = tuple(config.domain.grid_size)
        n = int(np.prod(shape))
        out = {"cfg_json": json.dumps(cfg, sort_keys=True)}
        if name == "fields":
            g1 = rng.standard_normal(shape)
            g2 = rng.standard_normal(shape)
            rho = 1.2 * (1 + 0.1 * np.tanh(g1))
            c = 343.0 * (1 + 0.05 * np.tanh(g2))
            solver.set_material_fields(rho, c)
            out["material_rho"], out["material_c"] = rho, c
        m = solver.transducers.num_transducers
        phases = rng.uniform(0, 2 * np.pi, m)
        solver.set_phases(phases)
        solver.assemble_matrix()
        rhs = solver.update_rhs()
        A = solver.A_cached_csr_cpu.tocsr()
        A.sort_indices()
        op = solver.warp_engine.operator
        B = solver.warp_engine.source_columns.tocsr()
        nxy = shape[0] * shape[1]
        assert B[nxy:].nnz == 0
        out.update(shape=np.array(shape), dx=config.domain.dx, omega=config.omega,
                   rho=np.asarray(op.rho), c=np.asarray(op.c),
                   A_data=A.data, A_indices=A.indices, A_indptr=A.indptr,
                   B_top=B[:nxy].toarray(), fixed=solver.warp_engine.fixed_dofs(),
                   centers=solver.transducers.centers, phases=phases, rhs=rhs)
        lu = spla.splu(sp.csc_matrix(A))
        x = lu.solve(rhs)
        out["x_direct"] = x
        xr = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        out["x_rand"], out["Ax_rand"] = xr, A @ xr
        AH = sp.csc_matrix(A.conj().T)
        out["AHx_rand"] = AH @ xr
        g = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        lam = spla.splu(AH).solve(g)
        out["adj_rhs"], out["adj_sol"] = g, lam
        grad_rho, grad_c = op.material_vjp(x, lam)
        out["vjp_rho"], out["vjp_c"] = grad_rho, grad_c
        amps = solver.transducers.amplitudes
        G = np.column_stack([lu.solve(B[:, k].toarray().ravel() * amps[k]) for k in range(m)])
        out["G"] = G
        basis = PhaseResponseBasis(solver, str(Path(tmp) / "basis.npy"))
        basis.basis = G
        basis.completed_columns = m
        phi2 = rng.uniform(0, 2 * np.pi, m)
        out["phi2"] = phi2
        field = basis.field(phi2)
        out["field_phi2"] = field
        cot = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
        out["cot"], out["phase_vjp"] = cot, basis.phase_vjp(cot, phi2)
        pts = np.asarray([t["point"] for t in cfg["targets"]], dtype=float)
        out["target_points"], out["target_response"] = pts, basis.target_response(pts)
        target = AmplitudeTarget.from_config(config)
        fp = FocalPressureLoss(config, target)
        loss, lcot = fp.evaluate(field)
        out["fp_loss"], out["fp_cot"] = loss, lcot
        fc = FocalContrastLoss(config, target)
        loss, lcot = fc.evaluate(field)
        out["fc_loss"], out["fc_cot"], out["fc_mask"] = loss, lcot, fc.background_mask
        out["target_indices"] = np.asarray(fp.target_indices)
    np.savez_compressed(HERE / f"golden_{name}.npz", **out)
    print(name, shape, "nnz", A.nnz, "m", m)


# Mid-size scene: large enough that the streaming GMRES kernels work through
# many node chunks (with a capped CTA count every CTA loops over several), with
# a seeded random medium, a blended high-contrast sphere and all face kinds.
MID = {
    "mode": "phase_optimization",
    "physics": {"sound_speed": 343.0, "medium_density": 1.2},
    "transducer_specs": {"frequency": 40000.0, "array_n": 2, "diameter": 0.006,
                         "pitch": 0.008, "geometry": "ideal_grid",
                         "source_radial_order": 16, "source_angular_order": 32},
    "domain": {"box_size": [0.035, 0.031, 0.029], "grid_size": [36, 32, 30]},
    "boundary_conditions": {"-x": "open",
                            "+x": {"type": "impedance", "impedance": [826.0, -40.0]},
                            "-y": "soft", "+y": "open", "-z": "reflecting", "+z": "open"},
    "targets": [{"point": [0.0175, 0.0155, 0.018]}],
    "obstacles": [],
    "solver": {"pml": {"cells": 6, "strength": 2.0, "order": 2, "faces": ["+y", "+z"]}},
    "training": {"background_weight": 0.05, "target_radius": 0.002,
                 "source_exclusion_layers": 2, "sidelobe_temperature": 25.0},
}
MID_ADJOINT_RHS = 3


def mid_materials(shape, dx):
    """Seeded random medium (Gaussian field smoothed over 2 cells, unit std,
    clipped to +-3; c = 343 (1 + 0.05 g), rho = 1.2 (1 + 0.1 g')) with a
    rho = 1250 / c = 2200 sphere (radius 5 mm) blended by the reference's
    smoothed step over 1.2 cells."""
    from scipy.ndimage import gaussian_filter
    from algorithm.physics.warp_utils import blend_obstacle_material
    rng = np.random.default_rng(40)
    fields = []
    for _ in range(2):
        g = gaussian_filter(rng.standard_normal(shape), 2.0)
        fields.append(np.clip(g / g.std(), -3.0, 3.0))
    c = 343.0 * (1 + 0.05 * fields[0])
    rho = 1.2 * (1 + 0.1 * fields[1])
    coords = np.ogrid[:shape[0], :shape[1], :shape[2]]
    centre = (0.018, 0.016, 0.015)
    sdf = np.sqrt(sum((coords[a] * dx - centre[a]) ** 2 for a in range(3))) - 0.005
    t = np.clip(sdf / (1.2 * dx), -1, 1)
    h = .5 * (1 + t + np.sin(np.pi * t) / np.pi)
    return blend_obstacle_material(h, 1250.0, 2200.0, rho, c)


def make_mid(reference_src):
    """golden_mid.npz: the reference's direct solutions of a 36 x 32 x 30 scene.

    Stored: the material fields, the source columns (z = 0 plane), the
    single-emitter responses G[:, k] = A^-1 (a_k B[:, k]) and three adjoint
    solutions A^-H g (solutions rounded once to complex64: 6e-8 relative, far
    below the 1e-6 parity bar), and A x for a deterministic probe vector (pins
    the assembly without storing the matrix)."""
    from algorithm.config import SimulationConfig
    from algorithm.solvers.helmholtz_solver import HelmholtzDirectSolver

    cfg = MID
    with tempfile.TemporaryDirectory() as tmp:
        path = Path(tmp) / "mid.yaml"
        path.write_text(yaml.safe_dump(_yaml_config(cfg)))
        config = SimulationConfig.from_yaml(str(path))
        solver = HelmholtzDirectSolver(config)
        shape = tuple(config.domain.grid_size)
        n = int(np.prod(shape))
        rho, c = mid_materials(shape, config.domain.dx)
        solver.set_material_fields(rho, c)
        m = solver.transducers.num_transducers
        rng = np.random.default_rng(41)
        phases = rng.uniform(0, 2 * np.pi, m)
        solver.set_phases(phases)
        solver.assemble_matrix()
        rhs = solver.update_rhs()
        A = solver.A_cached_csr_cpu.tocsr()
        B = solver.warp_engine.source_columns.tocsr()
        nxy = shape[0] * shape[1]
        assert B[nxy:].nnz == 0
        lu = spla.splu(sp.csc_matrix(A))
        amps = solver.transducers.amplitudes
        G = np.column_stack([lu.solve(B[:, k].toarray().ravel() * amps[k]) for k in range(m)])
        x = lu.solve(rhs)
        # superposition of the single-emitter solves (LU rounding ~1e-9 here)
        assert np.linalg.norm(G @ np.exp(1j * phases) - x) <= 1e-7 * np.linalg.norm(x)
        g = (rng.standard_normal((n, MID_ADJOINT_RHS))
             + 1j * rng.standard_normal((n, MID_ADJOINT_RHS))).astype(np.complex64)
        lam = lu.solve(g.astype(np.complex128), trans="H")
        probe = mid_probe(n)
        out = dict(cfg_json=json.dumps(cfg, sort_keys=True), shape=np.array(shape),
                   dx=config.domain.dx, omega=config.omega, material_rho=rho, material_c=c,
                   phases=phases, B_top=B[:nxy].toarray(), rhs=rhs,
                   G=G.astype(np.complex64), adj_rhs=g, adj_sol=lam.astype(np.complex64),
                   Ax_probe=A @ probe, fixed=solver.warp_engine.fixed_dofs())
    np.savez_compressed(HERE / "golden_mid.npz", **out)
    print("mid", shape, "nnz", A.nnz, "m", m)


def mid_probe(n):
    """Deterministic complex probe vector for the assembly check."""
    t = np.arange(n, dtype=np.float64)
    return np.cos(0.37 * t) + 1j * np.sin(0.11 * t + 0.5)


def make_blend(reference_src):
    from algorithm.physics.warp_utils import blend_obstacle_material
    h = np.linspace(0.0, 1.0, 11)
    rho, c = blend_obstacle_material(h, 1250.0, 2200.0, 1.21, 346.0)
    np.savez_compressed(HERE / "golden_blend.npz", h=h, rho=rho, c=c)


def main():
    if len(sys.argv) < 2:
        sys.exit("usage: make_golden.py REFERENCE_ROOT [scene ...]   "
                 "(the checkout that holds src/algorithm)")
    ref = Path(sys.argv[1]).resolve()
    if not (ref / "src" / "algorithm").is_dir():
        sys.exit(f"{ref} does not hold src/algorithm")
    only = set(sys.argv[2:])
    sys.path.insert(0, str(ref / "src"))
    _install_stubs()
    if not only or "blend" in only:
        make_blend(ref)
    for name, cfg in SCENES.items():
        if not only or name in only:
            make_scene(name, cfg, ref)
    if not only or "mid" in only:
        make_mid(ref)


if __name__ == "__main__":
    main()
