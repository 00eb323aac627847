"""Phase response basis u(phi) = G exp(i phi) on the B200.

Drop-in for src/algorithm/training/phase_response_basis.py:16-416: same
constructor, properties (num_transducers, shape, is_complete, basis),
methods (build, to_gpu, release_gpu, target_response, field, phase_vjp,
close) and the same on-disk format (`.npy` complex128 (N, M) C-order rows in
Fortran voxel order + JSON metadata with FORMAT_VERSION 3, scene fingerprint
and completed_columns, atomic .tmp -> replace), so builds resume and bases are
interchangeable. Differences: columns are computed by the batched matrix-free
GMRES (no cuDSS factorisation), and field / phase_vjp / target_response always
run as CUDA kernels on a device copy of G (`usv_basis_*`).
"""
from __future__ import annotations

import ctypes as C
import hashlib
import json
from dataclasses import asdict, is_dataclass
from pathlib import Path

import numpy as np
import torch

from . import _native as N
from .scene import FACES, as_grid, boundary_type

_DEVICE_PRECISION = {"complex128": (torch.complex128, N.PREC_FP64),
                     "complex64": (torch.complex64, N.PREC_MIXED)}


def _as_dict(obj):
    return asdict(obj) if is_dataclass(obj) else dict(vars(obj))


class PhaseResponseBasis:
    """Full-field response basis of a fixed scene; column r = field of emitter r."""

    FORMAT_VERSION = 3

    def __init__(self, solver, storage_path: str, rhs_batch_size: int = 8,
                 voxel_chunk_size: int = 262144, release_factor_after_build: bool = True,
                 device_precision: str = "complex128"):
        self.solver = solver
        self.storage_path = Path(storage_path)
        self.metadata_path = Path(f"{self.storage_path}.json")
        self.rhs_batch_size = int(rhs_batch_size)
        self.voxel_chunk_size = int(voxel_chunk_size)
        self.release_factor_after_build = bool(release_factor_after_build)
        if device_precision not in _DEVICE_PRECISION:
            raise ValueError(f"device_precision must be one of {sorted(_DEVICE_PRECISION)}")
        self.device_precision = device_precision
        self.dtype = np.dtype(np.complex128)
        self.basis = None
        self.basis_gpu = None  # torch (M, N) tensor: column m contiguous
        self.completed_columns = 0
        self._built_fingerprint = None
        if self.rhs_batch_size < 1:
            raise ValueError("rhs_batch_size must be at least 1")
        if self.voxel_chunk_size < 1:
            raise ValueError("voxel_chunk_size must be at least 1")

    # ----------------------------------------------------------- properties
    @property
    def num_transducers(self) -> int:
        return int(self.solver.transducers.num_transducers)

    @property
    def shape(self) -> tuple[int, int]:
        return self.solver.total_dofs, self.num_transducers

    @property
    def is_complete(self) -> bool:
        return self.completed_columns == self.num_transducers

    # ----------------------------------------------------------- build
    def build(self):
        backend = str(self.solver.cfg.solver.get("backend", "gpu_iterative")).lower()
        if backend not in ("gpu_iterative", "b200_iterative"):
            raise ValueError("the B200 phase basis is built with solver.backend='gpu_iterative'")
        self._open_or_create_storage()
        if self.is_complete:
            return self
        self.solver.assemble_matrix()
        counts = self.solver.sources.coverage()
        missing = np.flatnonzero(counts == 0)
        if missing.size:
            raise ValueError(f"The grid does not cover transducers {missing.tolist()}")
        amplitudes = self.solver.transducers.amplitudes
        dev_dtype, _ = _DEVICE_PRECISION[self.device_precision]
        if self.basis_gpu is None:
            self.basis_gpu = torch.zeros(self.shape[::-1], dtype=dev_dtype,
                                         device=self.solver.device)
            if self.completed_columns:
                done = np.asarray(self.basis[:, :self.completed_columns]).T
                self.basis_gpu[:self.completed_columns] = torch.from_numpy(
                    np.ascontiguousarray(done)).to(self.solver.device, dev_dtype)
        for start in range(self.completed_columns, self.num_transducers, self.rhs_batch_size):
            stop = min(start + self.rhs_batch_size, self.num_transducers)
            rhs = self.solver.sources.column_rhs(amplitudes, start, stop)
            cols = self.solver.solve_rhs_device(rhs)  # (stop-start, N)
            self.basis_gpu[start:stop] = cols.to(dev_dtype)
            self.basis[:, start:stop] = cols.cpu().numpy().T
            self.basis.flush()
            self.completed_columns = stop
            self._write_metadata()
        return self

    # ----------------------------------------------------------- device copy
    def to_gpu(self):
        self._require_complete()
        if self.basis_gpu is not None:
            return self
        dev = self.solver.device
        required = self.shape[0] * self.shape[1] * (8 if self.device_precision == "complex64" else 16)
        free, _ = torch.cuda.mem_get_info(dev)
        reserve = 256 * 1024 ** 2
        if required + reserve > free:
            raise MemoryError("Insufficient GPU memory for phase response basis: "
                              f"required={required / 1024 ** 3:.2f} GiB, "
                              f"free={free / 1024 ** 3:.2f} GiB")
        dev_dtype, _ = _DEVICE_PRECISION[self.device_precision]
        self.basis_gpu = torch.empty(self.shape[::-1], dtype=dev_dtype, device=dev)
        for start in range(0, self.shape[0], self.voxel_chunk_size):
            stop = min(start + self.voxel_chunk_size, self.shape[0])
            chunk = torch.from_numpy(np.ascontiguousarray(self.basis[start:stop].T))
            self.basis_gpu[:, start:stop] = chunk.to(dev, dev_dtype)
        return self

    def release_gpu(self):
        self.basis_gpu = None

    def _device_basis(self):
        if self.basis_gpu is None:
            self.to_gpu()
        return self.basis_gpu, _DEVICE_PRECISION[self.device_precision][1]

    # ----------------------------------------------------------- queries
    def target_response(self, points):
        """Trilinear complex response (P, M) at physical points (phase_response_basis.py:139-175)."""
        self._require_complete()
        points = np.asarray(points, dtype=float)
        cfg = self.solver.cfg
        shape = np.asarray(cfg.domain.grid_size)
        origin = np.asarray(cfg.domain.origin_m)
        upper = np.asarray(cfg.domain.box_size)
        if (points.ndim != 2 or points.shape[1] != 3 or not np.isfinite(points).all()
                or np.any(points < origin) or np.any(points > origin + upper)):
            raise ValueError("Targets must be finite (N,3) coordinates inside the grid")
        pml = cfg.solver.get("pml", {}) or {}
        cells = int(pml.get("cells", 0))
        if cells:
            faces = pml.get("faces", [f for f in FACES if boundary_type(
                cfg.boundary_conditions.get(f, "reflecting")) == "open"])
            for face in faces:
                axis = "xyz".index(face[1])
                local = points[:, axis] - origin[axis]
                distance = local if face[0] == "-" else upper[axis] - local
                if np.any(distance < cells * cfg.domain.dx):
                    raise ValueError("Target lies in PML; enlarge the physical interior")
        G, prec = self._device_basis()
        dev = self.solver.device
        pts = torch.from_numpy(np.ascontiguousarray(points - origin)).to(dev)
        out = torch.empty((len(points), self.num_transducers), dtype=torch.complex128, device=dev)
        N.check(N.load().usv_basis_target_response(
            N.ptr(G), int(shape[0]), int(shape[1]), int(shape[2]), self.num_transducers, prec,
            N.ptr(pts), len(points), float(cfg.domain.dx), N.ptr(out),
            N.stream_handle(torch, dev)), "target response")
        return out.cpu().numpy()

    def field_device(self, phases: torch.Tensor) -> torch.Tensor:
        """G e^{i phi} as a device vector in Fortran node order."""
        G, prec = self._device_basis()
        ph = torch.as_tensor(phases, dtype=torch.float64, device=G.device).contiguous()
        out = torch.empty(self.shape[0], dtype=torch.complex128, device=G.device)
        N.check(N.load().usv_basis_field(N.ptr(G), self.shape[0], self.num_transducers, prec,
                                         N.ptr(ph), N.ptr(out),
                                         N.stream_handle(torch, G.device)), "basis field")
        return out

    def field(self, phases, return_numpy: bool = True):
        self._require_complete()
        phase_shape = tuple(np.shape(phases))
        if phase_shape != (self.num_transducers,):
            raise ValueError(f"phases must have shape ({self.num_transducers},), got {phase_shape}")
        vec = self.field_device(phases)
        grid = as_grid(vec, self.solver.shape)
        return grid.cpu().numpy() if return_numpy else grid

    def phase_vjp_device(self, cotangent: torch.Tensor, phases) -> torch.Tensor:
        """dL/dphi for dL = Re(g^H du); cotangent is a device vector (Fortran order)."""
        G, prec = self._device_basis()
        dev = G.device
        cot = cotangent.to(device=dev, dtype=torch.complex128).contiguous()
        ph = torch.as_tensor(phases, dtype=torch.float64, device=dev).contiguous()
        grad = torch.empty(self.num_transducers, dtype=torch.float64, device=dev)
        nbytes = C.c_size_t()
        lib = N.load()
        N.check(lib.usv_basis_adjoint_workspace_bytes(self.shape[0], self.num_transducers,
                                                      C.byref(nbytes)), "workspace")
        ws = torch.empty(nbytes.value, dtype=torch.uint8, device=dev)
        N.check(lib.usv_basis_adjoint(N.ptr(G), self.shape[0], self.num_transducers, prec,
                                      N.ptr(cot), N.ptr(ph), None, N.ptr(grad), N.ptr(ws),
                                      nbytes.value, N.stream_handle(torch, dev)), "phase vjp")
        return grad

    def phase_vjp(self, field_cotangent, phases, return_numpy: bool = True):
        """Compute dL/dphase for dL = Re(field_cotangent^H du) (phase_response_basis.py:208-253)."""
        self._require_complete()
        phase_shape = tuple(np.shape(phases))
        if phase_shape != (self.num_transducers,):
            raise ValueError(f"phases must have shape ({self.num_transducers},), got {phase_shape}")
        if isinstance(field_cotangent, torch.Tensor):
            t = field_cotangent
            vec = (t.reshape(-1) if t.dim() == 1 else t.transpose(0, 2).reshape(-1))
        else:
            arr = np.asarray(field_cotangent, dtype=np.complex128).reshape(-1, order="F")
            vec = torch.from_numpy(np.ascontiguousarray(arr))
        if vec.numel() != self.solver.total_dofs:
            raise ValueError("field_cotangent has the wrong size")
        grad = self.phase_vjp_device(vec, phases)
        return grad.cpu().numpy() if return_numpy else grad

    def close(self):
        self.release_gpu()
        if isinstance(self.basis, np.memmap):
            self.basis.flush()
            mm = self.basis._mmap
            self.basis = None
            if mm is not None:
                mm.close()

    # ----------------------------------------------------------- storage
    def _open_or_create_storage(self):
        basis_exists = self.storage_path.exists()
        metadata_exists = self.metadata_path.exists()
        if basis_exists != metadata_exists:
            raise RuntimeError("Phase basis data and metadata must exist together")
        if basis_exists:
            metadata = json.loads(self.metadata_path.read_text(encoding="utf-8"))
            self._validate_metadata(metadata)
            self.basis = np.load(self.storage_path, mmap_mode="r+")
            if self.basis.shape != self.shape:
                raise RuntimeError("Stored phase basis shape mismatch")
            if self.basis.dtype != self.dtype:
                raise RuntimeError("Stored phase basis dtype mismatch")
            self.completed_columns = int(metadata["completed_columns"])
            self._built_fingerprint = metadata["fingerprint"]
            return
        self.storage_path.parent.mkdir(parents=True, exist_ok=True)
        self.basis = np.lib.format.open_memmap(self.storage_path, mode="w+", dtype=self.dtype,
                                               shape=self.shape, fortran_order=False)
        self.completed_columns = 0
        self._write_metadata()

    def _validate_metadata(self, metadata: dict):
        if metadata.get("format_version") != self.FORMAT_VERSION:
            raise RuntimeError("Unsupported phase basis format version")
        if metadata.get("fingerprint") != self._fingerprint():
            raise RuntimeError("Phase basis does not match the current physical scene")
        if metadata.get("shape") != list(self.shape):
            raise RuntimeError(f"Phase basis shape mismatch: {metadata.get('shape')} "
                               f"!= {list(self.shape)}")
        if metadata.get("dtype") != self.dtype.name:
            raise RuntimeError("Phase basis dtype mismatch")
        completed = int(metadata.get("completed_columns", -1))
        if completed < 0 or completed > self.num_transducers:
            raise RuntimeError("Invalid completed column count")

    def _write_metadata(self):
        fingerprint = self._fingerprint()
        metadata = {"format_version": self.FORMAT_VERSION, "fingerprint": fingerprint,
                    "shape": list(self.shape), "dtype": self.dtype.name,
                    "completed_columns": self.completed_columns}
        tmp = Path(f"{self.metadata_path}.tmp")
        tmp.write_text(json.dumps(metadata, indent=2, sort_keys=True), encoding="utf-8")
        tmp.replace(self.metadata_path)
        self._built_fingerprint = fingerprint

    def _fingerprint(self) -> str:
        cfg = self.solver.cfg
        payload = {
            "format_version": self.FORMAT_VERSION,
            "propagation_model": self.solver.MODEL_VERSION,
            "centers_m": self.solver.transducers.centers.tolist(),
            "physics": _as_dict(cfg.physics),
            "transducer_specs": _as_dict(cfg.specs),
            "domain": _as_dict(cfg.domain),
            "boundary_conditions": cfg.boundary_conditions,
            "obstacles": cfg.obstacles,
            "mesh_content_sha256": self._mesh_content_hashes(),
            "amplitudes": self.solver.transducers.amplitudes.tolist(),
            "pde_scene": self.solver.scene_fingerprint(),
        }
        encoded = json.dumps(payload, sort_keys=True, separators=(",", ":")).encode("utf-8")
        return hashlib.sha256(encoded).hexdigest()

    def _mesh_content_hashes(self) -> dict[str, str]:
        hashes = {}
        for obstacle in self.solver.cfg.obstacles:
            if obstacle.get("type", "").lower() != "mesh":
                continue
            path = Path(obstacle["file"])
            digest = hashlib.sha256()
            with path.open("rb") as f:
                for chunk in iter(lambda: f.read(1024 * 1024), b""):
                    digest.update(chunk)
            hashes[str(path)] = digest.hexdigest()
        return hashes

    def _require_complete(self):
        if self.basis is None or not self.is_complete:
            raise RuntimeError("Phase response basis is not complete")
        if self._built_fingerprint is not None and self._fingerprint() != self._built_fingerprint:
            raise RuntimeError("Physical scene changed; rebuild the phase response basis")
