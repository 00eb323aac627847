"""Shared helpers for the parity tests (no GPU work at import time)."""
import json

import numpy as np
import scipy.sparse as sp

from tests.conftest import load_golden


def golden_config(g):
    from ultrasound_solver_b200.config import SimulationConfig
    return SimulationConfig.from_dict(json.loads(str(g["cfg_json"])))


def golden_matrix(g):
    n = int(np.prod(g["shape"]))
    return sp.csr_matrix((g["A_data"], g["A_indices"], g["A_indptr"]), shape=(n, n))


def golden_solver(g, **solver_overrides):
    from ultrasound_solver_b200.helmholtz_solver import HelmholtzB200Solver
    cfg = golden_config(g)
    cfg.solver.update(solver_overrides)
    s = HelmholtzB200Solver(cfg)
    if "material_rho" in g:
        s.set_material_fields(g["material_rho"], g["material_c"])
    s.set_phases(g["phases"])
    s.assemble_matrix()
    return s


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
