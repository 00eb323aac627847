"""Scene configuration with the reference's YAML schema.

Field names, defaults and validation mirror the reference's dataclasses
(src/algorithm/config.py:8-213) so the same YAML files and config objects
drive both backends; HelmholtzB200Solver also accepts the reference's own
SimulationConfig objects (it only reads these attributes).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from pathlib import Path
from typing import Dict, List, Union

import numpy as np
import yaml


@dataclass
class PhysicsConfig:
    sound_speed: float = 343.0
    medium_density: float = 1.21
    material_field_file: str = ""


@dataclass
class TransducerSpecsConfig:
    frequency: float = 40000.0
    diameter: float = 0.0098
    pitch: float = 0.0105
    array_n: int = 6
    geometry: str = "ideal_grid"
    reference_anchor_m: List[float] = field(default_factory=lambda: [0.08, 0.08])
    source_radial_order: int = 64
    source_angular_order: int = 256

    def __post_init__(self):
        if (not isinstance(self.source_radial_order, int) or self.source_radial_order < 2
                or not isinstance(self.source_angular_order, int)
                or self.source_angular_order < 8):
            raise ValueError("Invalid source quadrature orders")
        if self.geometry not in {"ideal_grid", "sonicsurface_reference"}:
            raise ValueError("geometry must be ideal_grid or sonicsurface_reference")
        if self.geometry == "sonicsurface_reference" and self.array_n != 16:
            raise ValueError("SonicSurface reference geometry requires array_n=16")
        anchor = np.asarray(self.reference_anchor_m, dtype=float)
        if anchor.shape != (2,) or not np.isfinite(anchor).all():
            raise ValueError("reference_anchor_m must contain two finite coordinates")


@dataclass
class DomainConfig:
    box_size: List[float] = field(default_factory=lambda: [0.08, 0.08, 0.08])
    grid_size: List[int] = field(default_factory=lambda: [81, 81, 81])
    origin_m: List[float] = field(default_factory=lambda: [0.0, 0.0, 0.0])

    def __post_init__(self):
        origin = np.asarray(self.origin_m, dtype=float)
        if origin.shape != (3,) or not np.isfinite(origin).all():
            raise ValueError("domain.origin_m must contain three finite coordinates")

    nx = property(lambda self: self.grid_size[0])
    ny = property(lambda self: self.grid_size[1])
    nz = property(lambda self: self.grid_size[2])
    lx = property(lambda self: self.box_size[0])
    ly = property(lambda self: self.box_size[1])
    lz = property(lambda self: self.box_size[2])

    @property
    def dx(self) -> float:
        """Node spacing L/(N-1); the grid must be isotropic."""
        d = [self.box_size[a] / (self.grid_size[a] - 1) for a in range(3)]
        if not (np.isclose(d[0], d[1]) and np.isclose(d[0], d[2])):
            raise ValueError(
                f"the solver requires an isotropic grid (dx=dy=dz), got dx={d[0]*1000:.3f}mm, "
                f"dy={d[1]*1000:.3f}mm, dz={d[2]*1000:.3f}mm; check box_size against grid_size")
        return float(d[0])


@dataclass
class IOConfig:
    output_file: str = "ultrasound_field.npz"
    auto_visualize: bool = True
    colormap: str = "plasma"


@dataclass
class TrainingConfig:
    loss_type: str = "field_match"
    initial_phase: str = "geometric"
    compare_geometric: bool = False
    phase_basis_file: str = "phase_response_basis.npy"
    phase_basis_batch_size: int = 8
    voxel_chunk_size: int = 262144
    load_basis_to_gpu: bool = True
    release_factor_after_basis: bool = True
    target_field_file: str = ""
    target_peak_pressure: float = 600.0
    target_sigma: float = 0.006
    background_pressure: float = 0.0
    target_weight: float = 1.0
    background_weight: float = 0.05
    target_radius: float = 0.006
    source_exclusion_layers: int = 4
    sidelobe_temperature: float = 25.0
    iterations: int = 100
    seed: int = 0
    max_evaluations: int = 10000
    max_seconds: float = 0.0
    show_loss_curve: bool = True
    loss_curve_update_interval: int = 1
    loss_curve_pause_seconds: float = 0.01


@dataclass
class SimulationConfig:
    mode: str
    physics: PhysicsConfig
    specs: TransducerSpecsConfig
    domain: DomainConfig
    boundary_conditions: Dict[str, Union[str, dict]]
    targets: List[List[float]]
    obstacles: List[Dict]
    io: IOConfig = field(default_factory=IOConfig)
    training: TrainingConfig = field(default_factory=TrainingConfig)
    solver: Dict[str, Union[str, int, float, bool, dict]] = field(default_factory=dict)
    algorithm: str = "adjoint"
    algorithm_options: dict = field(default_factory=dict)
    same_phase_rad: float = 0.0

    def __post_init__(self):
        if self.mode not in {"phase_optimization", "same_phase", "sdf_inverse"}:
            raise ValueError("mode must be phase_optimization, same_phase or sdf_inverse")
        if not np.isfinite(self.same_phase_rad):
            raise ValueError("same_phase_rad must be finite")
        if not isinstance(self.algorithm_options, dict):
            raise ValueError("algorithm_options must be a mapping")

    frequency = property(lambda self: self.specs.frequency)
    omega = property(lambda self: 2.0 * np.pi * self.specs.frequency)
    k0 = property(lambda self: self.omega / self.physics.sound_speed)
    wavelength = property(lambda self: self.physics.sound_speed / self.specs.frequency)
    lx = property(lambda self: self.domain.lx)
    ly = property(lambda self: self.domain.ly)
    lz = property(lambda self: self.domain.lz)

    @classmethod
    def from_dict(cls, raw: dict, base: Path | None = None) -> "SimulationConfig":
        """Same mapping as the reference's from_yaml (config.py:168-213)."""
        base = Path.cwd() if base is None else base
        training = dict(raw.get("training", {}))
        obstacles = []
        for item in raw.get("obstacles", []) or []:
            ob = dict(item)
            if ob.get("type", "").lower() == "mesh":
                if "file" not in ob:
                    raise ValueError("mesh obstacle requires a 'file' path")
                if "center_m" not in ob:
                    raise ValueError("mesh obstacle requires 'center_m'")
                p = Path(ob["file"]).expanduser()
                ob["file"] = str((p if p.is_absolute() else base / p).resolve())
            obstacles.append(ob)
        physics = dict(raw["physics"])
        if physics.get("material_field_file"):
            p = Path(physics["material_field_file"]).expanduser()
            physics["material_field_file"] = str((p if p.is_absolute() else base / p).resolve())
        return cls(
            mode=str(raw.get("mode", "phase_optimization")).lower(),
            physics=PhysicsConfig(**physics),
            specs=TransducerSpecsConfig(**raw["transducer_specs"]),
            domain=DomainConfig(**raw["domain"]),
            boundary_conditions=raw["boundary_conditions"],
            targets=[t["point"] for t in raw.get("targets", []) or []],
            obstacles=obstacles,
            io=IOConfig(**raw.get("io", {})),
            training=TrainingConfig(**training),
            solver=raw.get("solver", {}) or {},
            algorithm=str(raw.get("algorithm", "adjoint")).lower(),
            algorithm_options=raw.get("algorithm_options", {}) or {},
            same_phase_rad=float(raw.get("same_phase_rad", 0.0)),
        )

    @classmethod
    def from_yaml(cls, yaml_path: str) -> "SimulationConfig":
        path = Path(yaml_path).expanduser().resolve()
        with open(path, "r", encoding="utf-8") as f:
            raw = yaml.safe_load(f)
        return cls.from_dict(raw, base=path.parent)
