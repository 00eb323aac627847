"""Seeded synthetic scenes with the shapes of the benchmark configurations.

No dataset is involved: media are seeded Gaussian random fields, phases are
seeded uniform draws. Scenes are node-centred (box = (N-1) h), the PML is the
reference's polynomial stretch (strength 2, quadratic) on every open face,
-z is the reflecting baffle carrying the sinc_neumann apertures.

Arrays that do not fit the PML-free interior keep n x n and shrink:
pitch p = min(10.5 mm, floor_0.5mm((L_int - 2h)/(n - 0.1))) and
diameter d = min(9 mm, floor_0.5mm(0.9 p)), L_int = (N-1)h - 2*cells*h.
Obstacles use the reference's smoothed material blend (rho 1250, c 2200,
width 1.2 cells) applied on top of the random medium.
"""
from __future__ import annotations

import numpy as np

F0 = 40000.0
C_AIR, RHO_AIR = 343.0, 1.2
PML = {"cells": 10, "strength": 2.0, "order": 2}


def _floor_half_mm(x):
    return np.floor(x / 0.5e-3 + 1e-9) * 0.5e-3


def fit_array(n_side, n_grid, h, cells=10, pitch=10.5e-3, diameter=9e-3):
    """(pitch, diameter) of an n x n array that fits the PML-free interior."""
    l_int = (n_grid - 1) * h - 2 * cells * h
    p = min(pitch, float(_floor_half_mm((l_int - 2 * h) / (n_side - 0.1))))
    d = min(diameter, float(_floor_half_mm(0.9 * p)))
    return p, d


def gaussian_random_field(shape, sigma_cells, seed):
    """Unit-std smoothed Gaussian field clipped to +-3 (float64)."""
    from scipy.ndimage import gaussian_filter
    rng = np.random.default_rng(seed)
    g = gaussian_filter(rng.standard_normal(shape), sigma=sigma_cells, mode="wrap")
    g = (g - g.mean()) / g.std()
    return np.clip(g, -3.0, 3.0)


def random_medium(shape, seed=0, c0=C_AIR, rho0=RHO_AIR, sigma_cells=4.0):
    """c = c0 (1 + 0.05 g), rho = rho0 (1 + 0.1 g') with independent g, g'."""
    g = gaussian_random_field(shape, sigma_cells, seed)
    g2 = gaussian_random_field(shape, sigma_cells, seed + 1000)
    return rho0 * (1 + 0.1 * g2), c0 * (1 + 0.05 * g)


def scene_dict(n, h, array_n, pitch, diameter, boundaries=None, obstacle=None, targets=(),
               solver=None, c0=C_AIR, rho0=RHO_AIR, radial=64, angular=256):
    box = (n - 1) * h
    bcs = {"-x": "open", "+x": "open", "-y": "open", "+y": "open",
           "-z": "reflecting", "+z": "open"}
    bcs.update(boundaries or {})
    cfg = {
        "mode": "phase_optimization",
        "physics": {"sound_speed": c0, "medium_density": rho0},
        "transducer_specs": {"frequency": F0, "array_n": array_n, "diameter": diameter,
                             "pitch": pitch, "geometry": "ideal_grid",
                             "source_radial_order": radial, "source_angular_order": angular},
        "domain": {"box_size": [box, box, box], "grid_size": [n, n, n]},
        "boundary_conditions": bcs,
        "targets": [{"point": list(map(float, t))} for t in targets],
        "obstacles": [obstacle] if obstacle else [],
        "solver": {"pml": dict(PML), **(solver or {})},
        "training": {"target_radius": 0.006, "source_exclusion_layers": 4},
    }
    return cfg


def config0():
    """64^3 air, 4x4 array (r 4.5 mm, pitch 10.5 mm), PML on all but -z."""
    return scene_dict(64, 1e-3, 4, 10.5e-3, 9e-3,
                      solver={"gmres_restart": 30, "gmres_rtol": 1e-10, "gmres_maxiter": 20000})


def config1(n=128, h=1e-3, array_n=8):
    """Variable medium + r=15 mm sphere 60 mm above the baffle, +x reflecting."""
    p, d = fit_array(array_n, n, h)
    centre = (n - 1) * h / 2
    sphere = {"type": "sphere", "center": [centre, centre, 0.060], "radius": 0.015,
              "smoothing_width_cells": 1.2, "material": {"density": 1250.0, "sound_speed": 2200.0}}
    return scene_dict(n, h, array_n, p, d, boundaries={"+x": "reflecting"}, obstacle=sphere,
                      targets=[(centre, centre, 0.080)],
                      solver={"gmres_restart": 30, "precision": "mixed"})


def config3(n=128, h=1e-3):
    """Config-1 scene with a 16x16 array (adjoint-gradient workload)."""
    return config1(n, h, array_n=16)


def random_rotation(seed):
    """Uniformly random rotation matrix (QR of a seeded Gaussian matrix)."""
    rng = np.random.default_rng(seed)
    q, r = np.linalg.qr(rng.standard_normal((3, 3)))
    q = q * np.sign(np.diag(r))
    if np.linalg.det(q) < 0:
        q[:, 0] = -q[:, 0]
    return q


def ellipsoid_sdf(shape, h, centre, semi_axes, rotation):
    """Signed distance (m, Fortran-ordered grid) of a rotated ellipsoid.

    The ellipsoid has no closed-form distance; this is the first-order
    estimate f = (|q/a| - 1) |q/a| / |q/a^2| in the body frame q = R^T (x - c),
    exact on the surface, negative inside, within a few per cent of the true
    distance over the few cells of the material blend."""
    grids = np.meshgrid(*(np.arange(n) * h for n in shape), indexing="ij")
    x = np.stack([g - c for g, c in zip(grids, centre)], axis=-1)
    q = x @ np.asarray(rotation)          # body-frame coordinates (R^T x per point)
    a = np.asarray(semi_axes, float)
    k0 = np.linalg.norm(q / a, axis=-1)
    k1 = np.linalg.norm(q / a ** 2, axis=-1)
    return np.where(k1 > 0, (k0 - 1.0) * k0 / np.maximum(k1, 1e-300), -float(a.min()))


def config4(n=256, h=0.8e-3, array_n=16, seed=2):
    """Full phase optimisation scene: config-1 medium statistics on an n^3 grid
    at h, a randomly rotated rigid ellipsoid (semi-axes 45 x 20 x 10 mm at
    256^3 / 0.8 mm, scaled with the box on smaller grids) blended as a
    rho = 1250 / c = 2200 obstacle, +x reflecting, -y impedance Z = 2 rho0 c0,
    the other open faces with the 10-cell PML, an n_a x n_a array and two
    focal-pressure targets. The ellipsoid enters as a precomputed SDF
    (obstacle type "sdf"): pass `config4_sdf(cfg)` to build_solver."""
    L = (n - 1) * h
    scale = L / (255 * 0.8e-3)
    p, d = fit_array(array_n, n, h)
    centre = L / 2
    targets = [(centre - 0.1 * L, centre, 0.6 * L), (centre + 0.1 * L, centre, 0.6 * L)]
    obstacle = {"type": "sdf", "smoothing_width_cells": 1.2,
                "material": {"density": 1250.0, "sound_speed": 2200.0},
                "center": [centre, centre, 0.35 * L],
                "semi_axes": [0.045 * scale, 0.020 * scale, 0.010 * scale],
                "rotation_seed": seed}
    cfg = scene_dict(n, h, array_n, p, d,
                     boundaries={"+x": "reflecting",
                                 "-y": {"type": "impedance",
                                        "impedance": [2 * RHO_AIR * C_AIR, 0.0]}},
                     obstacle=obstacle, targets=targets,
                     solver={"gmres_restart": 30, "precision": "mixed"})
    cfg["training"].update({"target_weight": 1.0, "background_weight": 0.05})
    return cfg


def config4_sdf(cfg):
    """The ellipsoid SDF of a config4 scene dict."""
    ob = cfg["obstacles"][0]
    shape = tuple(cfg["domain"]["grid_size"])
    h = cfg["domain"]["box_size"][0] / (shape[0] - 1)
    return ellipsoid_sdf(shape, h, ob["center"], ob["semi_axes"],
                         random_rotation(ob["rotation_seed"]))


def config2_basis_scene(n=96, h=1e-3):
    """Config-2 basis scene: config-1 medium statistics, 16x16 array (10.5 mm pitch if it fits)."""
    p, d = fit_array(16, n, h)
    centre = (n - 1) * h / 2
    sphere = {"type": "sphere", "center": [centre, centre, min(0.060, 0.6 * (n - 1) * h)],
              "radius": min(0.015, 0.12 * (n - 1) * h), "smoothing_width_cells": 1.2,
              "material": {"density": 1250.0, "sound_speed": 2200.0}}
    return scene_dict(n, h, 16, p, d, boundaries={"+x": "reflecting"}, obstacle=sphere,
                      solver={"gmres_restart": 20, "precision": "mixed"})


def config2_scene_batch(count=32, seed=3, sizes=(48, 64, 80, 96, 112), h=1e-3):
    """Config-2 uneven batch: grid edges drawn from `sizes`, a random sphere obstacle
    (radius 8-20 mm, kept clear of the PML and the baffle) and an 8x8 array each."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(rng.choice(sizes))
        L = (n - 1) * h
        p, d = fit_array(8, n, h)
        inner = L - 2 * PML["cells"] * h
        r = float(min(rng.uniform(0.008, 0.020), 0.2 * inner))
        lo, hi = PML["cells"] * h + r + 2 * h, L - PML["cells"] * h - r - 2 * h
        centre = [float(rng.uniform(lo, hi)), float(rng.uniform(lo, hi)),
                  float(rng.uniform(max(lo, 0.4 * L), hi))]
        sphere = {"type": "sphere", "center": centre, "radius": r, "smoothing_width_cells": 1.2,
                  "material": {"density": 1250.0, "sound_speed": 2200.0}}
        out.append(scene_dict(n, h, 8, p, d, boundaries={"+x": "reflecting"}, obstacle=sphere,
                              solver={"gmres_restart": 20, "precision": "mixed"}))
    return out


def build_solver(cfg_dict, seed=0, device=None, random=True, sdf=None):
    """HelmholtzB200Solver for a scene dict; the obstacle is blended into the
    random medium (a sphere from its centre and radius, an "sdf" obstacle from
    the precomputed `sdf` array)."""
    import torch

    from .config import SimulationConfig
    from .helmholtz_solver import HelmholtzB200Solver
    from .scene import blend_materials, fortran_flat

    d = dict(cfg_dict)
    obstacle = d["obstacles"][0] if (random and d.get("obstacles")) else None
    if random:
        d["obstacles"] = []
    cfg = SimulationConfig.from_dict(d)
    solver = HelmholtzB200Solver(cfg, device=device)
    if random:
        shape = tuple(cfg.domain.grid_size)
        rho_m, c_m = random_medium(shape, seed, cfg.physics.sound_speed,
                                   cfg.physics.medium_density)
        if obstacle:
            dev = solver.device
            rho_t, c_t = blend_materials(shape, cfg.domain.dx, dev, obstacle,
                                         cfg.physics.medium_density, cfg.physics.sound_speed,
                                         rho_medium=fortran_flat(rho_m, dev),
                                         c_medium=fortran_flat(c_m, dev), sdf=sdf)
            rho_m = rho_t.cpu().numpy().reshape(shape, order="F")
            c_m = c_t.cpu().numpy().reshape(shape, order="F")
            torch.cuda.synchronize()
        solver.set_material_fields(rho_m, c_m)
    rng = np.random.default_rng(seed + 1)
    solver.set_phases(rng.uniform(0, 2 * np.pi, solver.transducers.num_transducers))
    return solver
