"""Emitter layout and phases (src/algorithm/physics/transducer_array.py:5-77)."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np


class TransducerArray:
    """n x n ideal grid on z=0, x-major order, unit amplitudes."""

    def __init__(self, config):
        self.cfg = config
        self.centers = self._compute_transducer_centers()
        self.num_transducers = len(self.centers)
        self.surface_p0 = 1.0
        self.amplitudes = np.ones(self.num_transducers, dtype=np.float64)
        self.phases = np.zeros(self.num_transducers, dtype=np.float64)
        if self.cfg.mode in {"same_phase", "sdf_inverse"}:
            self.phases.fill(self.cfg.same_phase_rad)

    def _compute_transducer_centers(self) -> np.ndarray:
        spec = self.cfg.specs
        if spec.geometry == "sonicsurface_reference":
            # The vendor layout is data shipped with the reference, not here;
            # point solver.sonicsurface_reference_json at that file to use it.
            path = self.cfg.solver.get("sonicsurface_reference_json")
            if not path:
                raise ValueError("geometry sonicsurface_reference needs "
                                 "solver.sonicsurface_reference_json (path to the layout file)")
            data = json.loads(Path(path).read_text(encoding="utf-8"))
            pos = np.asarray(data["positions_vendor_xyz_m"], dtype=np.float64)
            centers = pos[data["logical_to_device"]][:, [0, 2, 1]].copy()
            centers[:, :2] += spec.reference_anchor_m
            return centers
        n, pitch = int(spec.array_n), float(spec.pitch)
        origin = np.asarray(self.cfg.domain.origin_m, dtype=np.float64)
        cx, cy = origin[:2] + np.asarray([self.cfg.lx, self.cfg.ly]) * 0.5
        half = (n - 1) * pitch * 0.5
        xs = cx - half + np.arange(n) * pitch
        ys = cy - half + np.arange(n) * pitch
        grid = np.empty((n * n, 3), dtype=np.float64)
        grid[:, 0] = np.repeat(xs, n)
        grid[:, 1] = np.tile(ys, n)
        grid[:, 2] = 0.0
        return grid

    def compute_geometric_phases(self) -> np.ndarray:
        """Time-reversal focusing phases (transducer_array.py:46-70)."""
        targets = self.cfg.targets
        if not targets:
            return np.zeros(self.num_transducers, dtype=np.float64)
        if len(targets) == 1:
            d = np.linalg.norm(self.centers - np.asarray(targets[0], dtype=np.float64), axis=-1)
            cycles = d / self.cfg.wavelength
            return 2.0 * np.pi * (np.ceil(cycles) - cycles)
        field = np.zeros(self.num_transducers, dtype=np.complex128)
        for t in targets:
            d = np.linalg.norm(self.centers - np.asarray(t, dtype=np.float64), axis=-1)
            field += (1.0 / d) * np.exp(-1j * self.cfg.k0 * d)
        return np.angle(field)

    def set_phases(self, phases):
        phases = np.asarray(phases, dtype=np.float64)
        if phases.shape != (self.num_transducers,) or not np.isfinite(phases).all():
            raise ValueError("phases must be a finite vector matching the array")
        self.phases = phases.copy()
