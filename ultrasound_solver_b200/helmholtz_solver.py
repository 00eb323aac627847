"""HelmholtzB200Solver: the gpu_iterative backend of HelmholtzDirectSolver on B200.

Drop-in for the methods of src/algorithm/solvers/helmholtz_solver.py that the
gpu_iterative backend serves (assemble_matrix, update_rhs, set_phases,
set_material_fields, scene_fingerprint, solve, solve_rhs, solve_adjoint,
material_vjp, build_phase_response_basis, invalidate_factorization,
factorize, close, target_response, field_at, field_at_direct), with the same
argument shapes (Fortran voxel order),
return shapes, exceptions and stats. Differences, all deliberate:

* the operator never exists as a CSR matrix: assembly is the per-node
  coefficient kernel and every solve is the matrix-free CUDA GMRES;
* ``solve_rhs`` accepts batches of right-hand sides (the reference's
  gpu_iterative rejects nrhs > 1, helmholtz_solver.py:594-595);
* the phase-response basis is built with this iterative backend (the
  reference requires cudss_hybrid_direct, phase_response_basis.py:70-77);
* ``*_device`` variants take and return torch CUDA tensors (no host copies).
"""
from __future__ import annotations

import hashlib
import json
import time
import warnings
from dataclasses import asdict, is_dataclass
from pathlib import Path

import numpy as np
import torch

from . import _native as N
from .iterative_solver import B200IterativeSolver
from .scene import (FACES, DeviceOperator, SourceColumns, as_grid, blend_materials,
                    boundary_type, fortran_flat, require_cuda)
from .transducers import TransducerArray

VALID_BACKENDS = ("gpu_iterative", "b200_iterative")


def _as_dict(obj):
    return asdict(obj) if is_dataclass(obj) else dict(vars(obj))


def _array_record(array) -> bytes:
    a = np.ascontiguousarray(array)
    return f"{a.dtype.str}{a.shape}".encode() + a.tobytes()


def _digest_records(records) -> str:
    """BLAKE2b over (label, payload) records, each length-prefixed."""
    h = hashlib.blake2b(digest_size=32)
    for label, payload in records:
        tag = label.encode()
        h.update(len(tag).to_bytes(4, "little") + tag)
        h.update(len(payload).to_bytes(8, "little"))
        h.update(payload)
    return h.hexdigest()


class _ResponseStore:
    """Target responses kept in one .npz file, valid for one cache key.

    Points are matched on a 1 nm lattice (their coordinates rounded to
    integer nanometres); entries written for another key are ignored and
    replaced on the next write. Writes go to a temporary file that is then
    renamed over the store.
    """

    def __init__(self, path: Path, key: str, channels: int):
        self.path, self.key, self.channels = path, key, channels
        self.points = np.empty((0, 3))
        self.values = np.empty((0, channels), complex)
        try:
            with np.load(path, allow_pickle=False) as data:
                if str(data["key"]) == key:
                    pts, vals = np.asarray(data["points"], float), np.asarray(data["values"])
                    if (pts.ndim == 2 and pts.shape[1] == 3 and vals.shape == (len(pts), channels)
                            and np.isfinite(pts).all() and np.isfinite(vals).all()):
                        self.points, self.values = pts, vals.astype(complex)
        except (OSError, KeyError, ValueError):
            pass

    @staticmethod
    def _lattice(points):
        return [tuple(r) for r in np.rint(np.asarray(points) * 1e9).astype(np.int64)]

    def lookup(self, points, out) -> np.ndarray:
        """Fill out[i] for stored points; returns the mask of points found."""
        index = {k: i for i, k in enumerate(self._lattice(self.points))}
        found = np.zeros(len(points), bool)
        for i, k in enumerate(self._lattice(points)):
            j = index.get(k)
            if j is not None:
                out[i] = self.values[j]
                found[i] = True
        return found

    def add(self, points, values):
        self.points = np.vstack((self.points, points))
        self.values = np.vstack((self.values, values))
        self.path.parent.mkdir(parents=True, exist_ok=True)
        tmp = self.path.with_name(self.path.name + ".partial.npz")
        np.savez_compressed(tmp, key=self.key, points=self.points, values=self.values)
        tmp.replace(self.path)


class HelmholtzB200Solver:
    """Assemble and solve the discrete Helmholtz system on one B200."""

    MODEL_VERSION = "helmholtz_conservative_sources_v5"
    field_unit = "normalized_1_per_m"

    def __init__(self, config, device=None):
        self.cfg = config
        self.device = require_cuda(device)
        self.transducers = TransducerArray(config)
        self.origin = np.asarray(config.domain.origin_m, dtype=np.float64)
        if not np.isclose(self.origin[2], 0.0):
            raise ValueError("The transducer plane requires domain.origin_m[2] == 0")
        self.shape = tuple(int(v) for v in config.domain.grid_size)
        self.total_dofs = int(np.prod(self.shape))
        self.operator: DeviceOperator | None = None
        self.sources: SourceColumns | None = None
        self.rhs_cached = None
        self._rhs_device = None
        self._obs_sdf = None
        self._scene_key = None
        self._material_fields = None
        self._grid_definition = _as_dict(config.domain)
        self._source_definition = _as_dict(config.specs)
        self.condensed_solver = None
        self._target_surface_solver = None
        self._target_source_masses = None
        s = config.solver
        self.iterative_solver = B200IterativeSolver(
            restart=int(s.get("gmres_restart", 30)),
            maxiter=int(s.get("gmres_maxiter", 3000)),
            rtol=float(s.get("gmres_rtol", 1.0e-6)),
            backward_error_tol=float(s.get("gmres_backward_error_tol", 1.0e-4)),
            precision=str(s.get("precision", "mixed")),
            full_cycles=bool(s.get("gmres_full_cycles", True)),
            use_graph=bool(s.get("cuda_graph", True)),
            block_nodes=int(s.get("block_nodes", 0)),
            recycle=int(s.get("gmres_recycle", 0)),
            recycle_every=int(s.get("gmres_recycle_every", 1)),
            batch_width=int(s.get("gmres_batch_width", 0)),
            max_ctas=int(s.get("gmres_max_ctas", 0)),
            kernel_variant=int(s.get("gmres_kernel_variant", 0)),
        )

    # ----------------------------------------------------------- scene
    @property
    def obstacle_sdf(self):
        return self._obs_sdf

    def set_obstacle_sdf(self, sdf):
        """Precomputed (nx,ny,nz) SDF for a mesh obstacle (the reference samples it with pyvista)."""
        self._obs_sdf = np.array(sdf, dtype=np.float64, copy=True)
        self.invalidate_factorization()

    def set_material_fields(self, density, sound_speed):
        """Spatial material arrays (nx,ny,nz), copied (helmholtz_solver.py:238-247)."""
        arrays = tuple(np.array(a, dtype=np.float64, copy=True) for a in (density, sound_speed))
        if any(a.shape != self.shape or not np.isfinite(a).all() or np.any(a <= 0) for a in arrays):
            raise ValueError("Material fields must match the grid and be finite and positive")
        if self.cfg.obstacles or self.cfg.physics.material_field_file:
            raise ValueError("Choose one material input: arrays, NPZ file, or obstacle")
        self._material_fields = arrays
        self.invalidate_factorization()

    def scene_fingerprint(self):
        """Digest of every input that defines the matrix and the sources.

        The reference keys cached factorizations and stored bases on such a
        digest (helmholtz_solver.py:249-271); this one is built as a sequence
        of labelled, length-prefixed records (the scene description as
        canonical JSON, then each array input with its dtype and shape, then
        each referenced file), so two scenes share a fingerprint only if every
        record matches.
        """
        if (_as_dict(self.cfg.domain) != self._grid_definition
                or _as_dict(self.cfg.specs) != self._source_definition):
            raise ValueError("Grid or source specification changed; construct a new solver")
        description = {
            "model": self.MODEL_VERSION, "physics": _as_dict(self.cfg.physics),
            "domain": _as_dict(self.cfg.domain), "specs": _as_dict(self.cfg.specs),
            "boundaries": self.cfg.boundary_conditions, "obstacles": self.cfg.obstacles,
            "pml": self.cfg.solver.get("pml", {}),
            "source_centres_from_origin": (self.transducers.centers - self.origin).tolist()}
        records = [("scene", json.dumps(description, sort_keys=True, default=str).encode())]
        if self._material_fields is not None:
            records += [(f"material[{i}]", _array_record(a))
                        for i, a in enumerate(self._material_fields)]
        if self._obs_sdf is not None:
            records.append(("obstacle_sdf", _array_record(self._obs_sdf)))
        referenced = [o["file"] for o in self.cfg.obstacles
                      if o.get("type", "").lower() == "mesh"]
        if self.cfg.physics.material_field_file:
            referenced.append(self.cfg.physics.material_field_file)
        for name in referenced:
            records.append((f"file:{Path(name).name}", Path(name).read_bytes()))
        return _digest_records(records)

    def source_diagnostics(self):
        centers = (self.transducers.centers - self.origin)[:, :2]
        radius = self.cfg.specs.diameter * 0.5
        clipped = np.any((centers - radius < 0)
                         | (centers + radius > np.asarray([self.cfg.lx, self.cfg.ly])), axis=1)
        return {"points_per_wavelength": self.cfg.wavelength / self.cfg.domain.dx,
                "kdx": self.cfg.k0 * self.cfg.domain.dx,
                "clipped_emitters": np.flatnonzero(clipped).tolist()}

    def _device_materials(self, obstacle, rho0, c0):
        dev, dx = self.device, self.cfg.domain.dx
        materials = self._material_fields
        if self.cfg.physics.material_field_file:
            if materials is not None or obstacle:
                raise ValueError("Material NPZ is mutually exclusive with arrays or obstacles")
            with np.load(self.cfg.physics.material_field_file, allow_pickle=False) as data:
                materials = (data["density"], data["sound_speed"])
        if materials is not None:
            if obstacle:
                raise ValueError("Explicit material fields and obstacle materials are mutually exclusive")
            rho, c = (np.asarray(a, dtype=np.float64) for a in materials)
            if rho.shape != self.shape or c.shape != self.shape:
                raise ValueError(f"Material fields must match grid {self.shape}")
            return fortran_flat(rho, dev), fortran_flat(c, dev)
        if obstacle:
            kind = obstacle.get("type", "sphere").lower()
            if kind == "mesh" and self._obs_sdf is None:
                raise ValueError("mesh obstacle requires a precomputed SDF (obs_sdf); "
                                 "pass it with set_obstacle_sdf()")
            return blend_materials(self.shape, dx, dev, obstacle, rho0, c0, sdf=self._obs_sdf)
        n = self.total_dofs
        return (torch.full((n,), rho0, dtype=torch.float64, device=dev),
                torch.full((n,), c0, dtype=torch.float64, device=dev))

    def assemble_matrix(self, force: bool = False):
        """Build the device operator and sources; returns the current RHS (numpy)."""
        key = self.scene_fingerprint()
        if self.operator is not None and not force and key == self._scene_key:
            return self.update_rhs()
        self.invalidate_factorization()
        diag = self.source_diagnostics()
        if diag["points_per_wavelength"] < 6:
            raise ValueError("PDE grid has fewer than 6 points per background wavelength; "
                             "refine grid_size before solving")
        if diag["points_per_wavelength"] < 10:
            warnings.warn(f"PDE resolution: {diag['points_per_wavelength']:.2f} points/wavelength; "
                          "small algebraic residual does not establish phase accuracy.",
                          RuntimeWarning)
        if diag["clipped_emitters"]:
            warnings.warn(f"Source discs clipped by the domain: {diag['clipped_emitters']}",
                          RuntimeWarning)
        if len(self.cfg.obstacles) > 1:
            raise NotImplementedError("The solver currently supports one obstacle at a time")
        obstacle = dict(self.cfg.obstacles[0]) if self.cfg.obstacles else {}
        if obstacle.get("type", "").lower() == "sphere":
            obstacle["center"] = (np.asarray(obstacle.get("center", [.04, .04, .02]), dtype=float)
                                  - self.origin).tolist()
        rho0 = float(self.cfg.physics.medium_density)
        c0 = float(self.cfg.physics.sound_speed)
        rho, c = self._device_materials(obstacle, rho0, c0)
        centers = self.transducers.centers - self.origin
        if (centers.shape != (self.transducers.num_transducers, 3) or not np.isfinite(centers).all()
                or np.any(centers[:, 2] != 0)):
            raise ValueError("PDE sources require finite bottom-plane centers matching phases")
        bcs = self.cfg.boundary_conditions
        if boundary_type(bcs.get("-z", "reflecting")) != "reflecting":
            raise ValueError("The sinc Neumann source requires a reflecting baffled bottom plane")
        dx = self.cfg.domain.dx
        self.operator = DeviceOperator(self.shape, dx, self.cfg.omega, bcs, rho, c,
                                       pml=self.cfg.solver.get("pml"))
        spec = self.cfg.specs
        self.sources = SourceColumns(self.operator, centers, spec.diameter, rho0,
                                     spec.source_radial_order, spec.source_angular_order)
        if float(c.min()) / self.cfg.frequency / dx < 6:
            raise ValueError("PDE grid has fewer than 6 points per shortest local wavelength; "
                             "refine grid_size before solving (10+ points and convergence checks recommended)")
        self._scene_key = key
        return self.update_rhs()

    def update_rhs_device(self) -> torch.Tensor:
        self._rhs_device = self.sources.phase_rhs(self.transducers.amplitudes,
                                                  self.transducers.phases)
        return self._rhs_device

    def update_rhs(self) -> np.ndarray:
        self.rhs_cached = self.update_rhs_device().cpu().numpy()
        return self.rhs_cached

    def set_phases(self, phases):
        self.transducers.set_phases(phases)

    def invalidate_factorization(self):
        self.operator = None
        self.sources = None
        self.rhs_cached = None
        self._rhs_device = None

    def factorize(self):
        """No factorisation exists for the iterative backend; assembles the operator."""
        self.assemble_matrix()

    def close(self):
        self._target_surface_solver = None
        self._target_source_masses = None
        self.invalidate_factorization()

    def _requested_backend(self) -> str:
        backend = str(self.cfg.solver.get("backend", "gpu_iterative")).lower()
        if backend not in VALID_BACKENDS:
            raise ValueError(f"solver.backend={backend!r} is not served by HelmholtzB200Solver; "
                             f"valid values are {list(VALID_BACKENDS)}")
        return backend

    # ----------------------------------------------------------- homogeneous targets
    # helmholtz_solver.py:79-226: exact target responses of homogeneous scenes
    # through the surface Schur complement (homogeneous_surface.py).
    def _ensure_target_surface_solver(self):
        from .homogeneous_surface import HomogeneousSurfaceSolver
        if self.cfg.obstacles or self.cfg.physics.material_field_file or self._material_fields is not None:
            raise ValueError("Surface condensation requires a homogeneous medium")
        if boundary_type(self.cfg.boundary_conditions.get("-z", "reflecting")) != "reflecting":
            raise ValueError("Surface condensation requires a reflecting baffled -z face")
        if self._target_surface_solver is not None:
            return
        self.assemble_matrix()
        self._target_source_masses = self.sources.mass_matrix.T.cpu().numpy()
        self._target_surface_solver = HomogeneousSurfaceSolver(
            self.shape, self.cfg.domain.dx, self.cfg.frequency, self.cfg.physics.sound_speed,
            self.cfg.physics.medium_density, self.cfg.boundary_conditions,
            pml=self.cfg.solver.get("pml", {}), device=self.device)

    def _local_target_points(self, points):
        points = np.asarray(points, dtype=float)
        local = points - self.origin
        extent = np.asarray(self.cfg.domain.box_size, dtype=float)
        if (points.ndim != 2 or points.shape[1] != 3 or not np.isfinite(points).all()
                or np.any(local < -1e-12) or np.any(local > extent + 1e-12)):
            raise ValueError("Targets must be finite physical coordinates inside the PDE domain")
        pml = self.cfg.solver.get("pml", {}) or {}
        cells = int(pml.get("cells", 0))
        if cells:
            faces = pml.get("faces", [f for f in FACES
                                      if boundary_type(self.cfg.boundary_conditions[f]) == "open"])
            thickness = cells * self.cfg.domain.dx
            for face in faces:
                axis = "xyz".index(face[1])
                distance = local[:, axis] if face[0] == "-" else extent[axis] - local[:, axis]
                if np.any(distance < thickness - 1e-12):
                    raise ValueError("Target lies in PML; enlarge the physical interior")
        return local

    def _target_response_cache(self):
        """The optional on-disk store of computed target responses
        (solver.target_response_cache), keyed to this scene and to the code
        that computes the responses."""
        filename = str(self.cfg.solver.get("target_response_cache", "")).strip()
        if not filename:
            return None
        here = Path(__file__)
        code = [(f.name, f.read_bytes()) for f in
                (here, here.with_name("homogeneous_surface.py"), here.with_name("scene.py"))]
        key = _digest_records([("scene", self.scene_fingerprint().encode()),
                               ("origin", self.origin.tobytes()), *code])
        return _ResponseStore(Path(filename), key, self.transducers.num_transducers)

    def target_response(self, points):
        """(P, M) target x channel responses of the discrete PDE (homogeneous scenes)."""
        points = np.asarray(points, dtype=float)
        local = self._local_target_points(points)
        store = self._target_response_cache()
        result = np.empty((len(points), self.transducers.num_transducers), complex)
        found = store.lookup(points, result) if store else np.zeros(len(points), bool)
        todo = np.flatnonzero(~found)
        if todo.size:
            self._ensure_target_surface_solver()
            result[todo] = self._target_surface_solver.flux_target_response(
                self._target_source_masses, local[todo])
            if store:
                store.add(points[todo], result[todo])
        return result

    def field_at(self, points, phases=None):
        values = self.transducers.phases if phases is None else np.asarray(phases, dtype=float)
        if values.shape != (self.transducers.num_transducers,) or not np.isfinite(values).all():
            raise ValueError("phases must match the transducer array and be finite")
        return self.target_response(points) @ np.exp(1j * values)

    def field_at_direct(self, points, phases=None):
        values = self.transducers.phases if phases is None else np.asarray(phases, dtype=float)
        if values.shape != (self.transducers.num_transducers,) or not np.isfinite(values).all():
            raise ValueError("phases must match the transducer array and be finite")
        self._ensure_target_surface_solver()
        self._target_surface_solver.solve_flux(self._target_source_masses, values)
        return self._target_surface_solver.sample(self._local_target_points(points))

    # ----------------------------------------------------------- solves
    def solve(self) -> np.ndarray:
        """Field of the current phases, (nx,ny,nz) complex128."""
        start = time.perf_counter()
        self.assemble_matrix(force=not bool(self.cfg.solver.get("reuse_matrix", True)))
        self.update_rhs_device()
        x = self.solve_rhs_device(self._rhs_device)
        out = x.cpu().numpy().reshape(self.shape, order="F")
        self.last_solve_seconds = time.perf_counter() - start
        return out

    def solve_rhs_device(self, rhs: torch.Tensor, adjoint: bool = False) -> torch.Tensor:
        """(N,) or (B, N) complex128 device tensor(s) -> solution(s), same shape."""
        self._requested_backend()
        if self.operator is None:
            raise RuntimeError("The matrix has not been assembled; call assemble_matrix() first")
        self.assemble_matrix()
        return self.iterative_solver.solve(self.operator, rhs, adjoint=adjoint)

    def solve_rhs(self, rhs: np.ndarray, verbose: bool = True) -> np.ndarray:
        """(N,) or (N, nrhs) complex128 -> solution of the same rank (helmholtz_solver.py:450-511)."""
        if self.operator is None:
            raise RuntimeError("The matrix has not been assembled; call assemble_matrix() first")
        self.assemble_matrix()
        mat, squeeze = self._as_rhs_matrix(rhs)
        dev = torch.from_numpy(np.ascontiguousarray(mat.T)).to(self.device)
        self.iterative_solver.verbose = bool(verbose)
        x = self.solve_rhs_device(dev).cpu().numpy().T
        return x[:, 0] if squeeze else x

    def solve_adjoint(self, adjoint_rhs: np.ndarray) -> np.ndarray:
        """A^H lambda = g; g (nx,ny,nz[,k]) or (N[,k]) -> (nx,ny,nz[,k]) (helmholtz_solver.py:513-530)."""
        self.assemble_matrix()
        mat, squeeze = self._as_adjoint_rhs_matrix(adjoint_rhs)
        dev = torch.from_numpy(np.ascontiguousarray(mat.T)).to(self.device)
        lam = self.solve_rhs_device(dev, adjoint=True).cpu().numpy().T
        if squeeze:
            lam = lam[:, 0]
        return self._reshape_solution(lam)

    def material_vjp(self, field, field_cotangent):
        """Voxel density/speed gradients with one A^H solve (helmholtz_solver.py:532-539)."""
        lam = self.solve_adjoint(field_cotangent)
        u = torch.from_numpy(np.ascontiguousarray(np.asarray(field, dtype=np.complex128)
                                                  .reshape(-1, order="F"))).to(self.device)
        la = torch.from_numpy(np.ascontiguousarray(lam.reshape(-1, order="F"))).to(self.device)
        gr, gc = self.material_vjp_device(u, la)
        return (gr.cpu().numpy().reshape(self.shape, order="F"),
                gc.cpu().numpy().reshape(self.shape, order="F"))

    def material_vjp_device(self, u: torch.Tensor, lam: torch.Tensor):
        import ctypes as C
        op = self.operator
        gr = torch.empty(op.n, dtype=torch.float64, device=self.device)
        gc = torch.empty_like(gr)
        N.check(N.load().usv_material_vjp(C.byref(op.scene), N.ptr(op.buffer), N.ptr(op.rho),
                                          N.ptr(op.c), N.ptr(u.contiguous()),
                                          N.ptr(lam.contiguous()), N.ptr(gr), N.ptr(gc),
                                          N.stream_handle(torch, self.device)), "material vjp")
        return gr, gc

    def build_phase_response_basis(self, **kwargs):
        from .phase_response_basis import PhaseResponseBasis
        t = self.cfg.training
        return PhaseResponseBasis(solver=self, storage_path=t.phase_basis_file,
                                  rhs_batch_size=kwargs.pop("rhs_batch_size",
                                                            t.phase_basis_batch_size),
                                  voxel_chunk_size=t.voxel_chunk_size,
                                  release_factor_after_build=t.release_factor_after_basis,
                                  **kwargs).build()

    # ----------------------------------------------------------- shapes
    def _as_rhs_matrix(self, rhs):
        array = np.asarray(rhs, dtype=np.complex128)
        if array.ndim == 1 and array.size == self.total_dofs:
            return np.asfortranarray(array.reshape((-1, 1))), True
        if array.ndim == 2 and array.shape[0] == self.total_dofs:
            return np.asfortranarray(array), False
        raise ValueError(f"rhs must have shape ({self.total_dofs},) or "
                         f"({self.total_dofs}, nrhs), got {array.shape}")

    def _as_adjoint_rhs_matrix(self, rhs):
        array = np.asarray(rhs, dtype=np.complex128)
        if array.shape == self.shape:
            return np.asfortranarray(array.reshape((-1, 1), order="F")), True
        if array.ndim == 4 and array.shape[:3] == self.shape:
            return np.asfortranarray(array.reshape((self.total_dofs, -1), order="F")), False
        return self._as_rhs_matrix(array)

    def _reshape_solution(self, solution):
        array = np.asarray(solution)
        if array.ndim == 1:
            return array.reshape(self.shape, order="F")
        return array.reshape(self.shape + (array.shape[1],), order="F")

    def field_grid(self, vec: torch.Tensor) -> torch.Tensor:
        """Device vector -> (nx,ny,nz) view."""
        return as_grid(vec, self.shape)


HelmholtzDirectSolver = HelmholtzB200Solver  # name used by the reference's callers
