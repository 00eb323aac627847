"""Exact forward solve of the homogeneous-medium FV discretisation (device).

Mirrors HomogeneousSurfaceSolver (src/algorithm/solvers/homogeneous_surface.py:
117-259): for a homogeneous medium the discrete operator separates, so the
x and y axis operators are diagonalised once (host eigen-decomposition, as
the reference does with scipy), the z axis is eliminated by a backward
continued fraction per (x, y) mode (usv_z_transfer, one CUDA thread per
mode), and the sinc_neumann surface flux is solved through the resulting
surface Schur complement. The modal transforms are dense products on the
device. Used by HelmholtzB200Solver.target_response / field_at /
field_at_direct for homogeneous scenes.
"""
from __future__ import annotations

import ctypes as C
import hashlib
from collections import OrderedDict

import numpy as np
import scipy.linalg as la
import torch

from . import _native as N
from .scene import FACES, boundary_type, require_cuda

_EIGEN_CACHE: "OrderedDict[tuple, tuple]" = OrderedDict()


def _eigendecomposition(matrix):
    """(eigenvalues, V, V^-1, ||V||_1 ||V^-1||_1) with a small LRU cache
    (homogeneous_surface.py:20-38: identical axis operators repeat)."""
    a = np.ascontiguousarray(matrix)
    key = (a.shape, a.dtype.str, hashlib.sha256(a.view(np.uint8)).digest())
    hit = _EIGEN_CACHE.get(key)
    if hit is not None:
        _EIGEN_CACHE.move_to_end(key)
        return hit
    w, v = la.eig(a)
    vinv = la.inv(v)
    out = (w, v, vinv, float(la.norm(v, 1) * la.norm(vinv, 1)))
    _EIGEN_CACHE[key] = out
    while len(_EIGEN_CACHE) > 4:
        _EIGEN_CACHE.popitem(last=False)
    return out


def axis_matrix(n, dx, omega, density, sound_speed, faces, pml, axis):
    """1-D FV operator along `axis` of the homogeneous scene and its PML stretch
    (homogeneous_surface.py:88-114): half control volumes at the two ends,
    mid-face stretch, Robin terms of open / impedance ends."""
    lo, hi = FACES[2 * axis], FACES[2 * axis + 1]
    local = {"-": faces.get(lo, "reflecting"), "+": faces.get(hi, "reflecting")}
    if any(boundary_type(v) not in {"open", "reflecting", "impedance"} for v in local.values()):
        raise ValueError("Surface diagnostic supports open/reflecting/impedance faces")
    pml = pml or {}
    cells = int(pml.get("cells", 0))
    strength = float(pml.get("strength", 2.0))
    order = int(pml.get("order", 3))
    if cells < 0 or strength < 0 or not np.isfinite(strength) or order < 1:
        raise ValueError("Invalid PML cells, strength or order")
    pml_faces = pml.get("faces", [f for f in FACES
                                  if boundary_type(faces.get(f, "reflecting")) == "open"])
    active = [side for side, face in (("-", lo), ("+", hi)) if face in pml_faces]
    sigma = np.zeros(n)
    if cells and active:
        if cells * len(active) >= n - 1:
            raise ValueError("PML leaves no physical interior on an axis")
        for side in active:
            if boundary_type(local[side]) != "open":
                raise ValueError("PML may only be placed on open faces")
            d = np.arange(n) if side == "-" else np.arange(n)[::-1]
            sigma += strength * np.maximum(1 - d / cells, 0) ** order
    s = 1 + 1j * sigma
    w = np.ones(n)
    w[[0, -1]] = 0.5
    edge = 1 / (0.5 * (s[:-1] + s[1:]) * dx * dx)
    diagonal = np.zeros(n, complex)
    diagonal[:-1] -= edge
    diagonal[1:] -= edge
    matrix = np.diag(diagonal) + np.diag(edge, 1) + np.diag(edge, -1)
    matrix /= (w * s)[:, None]
    for i, side in ((0, "-"), (-1, "+")):
        kind = boundary_type(local[side])
        if kind in {"open", "impedance"}:
            z = density * sound_speed if kind == "open" else complex(*local[side]["impedance"])
            matrix[i, i] += 1j * omega * density / (z * dx * w[i] * s[i])
    return matrix, s


def _dense(masses, device):
    if hasattr(masses, "toarray"):
        masses = masses.toarray()
    return torch.as_tensor(np.asarray(masses) if not torch.is_tensor(masses) else masses,
                           device=device).to(torch.complex128)


class HomogeneousSurfaceSolver:
    def __init__(self, shape, dx, frequency, sound_speed, density, boundaries, pml=None,
                 device=None):
        if not all(np.ndim(v) == 0 and np.isfinite(v) and v > 0
                   for v in (dx, frequency, sound_speed, density)):
            raise ValueError("This diagnostic requires positive scalar homogeneous materials")
        if set(boundaries) - set(FACES):
            raise ValueError("Unknown boundary face")
        self.shape = tuple(int(v) for v in shape)
        self.dx = float(dx)
        self.device = require_cuda(device)
        self.boundaries = dict(boundaries)
        omega = 2 * np.pi * frequency
        axes = [axis_matrix(n, dx, omega, density, sound_speed, boundaries, pml or {}, a)
                for a, n in enumerate(self.shape)]
        self.axes = [a[0] for a in axes]
        self.surface_pml = ((axes[0][1].imag[:, None] + axes[1][1].imag[None, :]
                             + axes[2][1].imag[0]) > 0)
        ex, vx, ix, cond_x = _eigendecomposition(self.axes[0])
        ey, vy, iy, cond_y = _eigendecomposition(self.axes[1])
        self.eigen_condition = [cond_x, cond_y]
        dev = self.device
        t = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.complex128, device=dev)
        self.vx, self.vy, self.ix, self.iy = t(vx), t(vy), t(ix), t(iy)
        shift = t(ex[:, None] + ey[None, :] + (omega / sound_speed) ** 2)
        z = self.axes[2]
        nx, ny, nz = self.shape
        # H[j] = u[j+1]/u[0] per (x, y) mode, by the backward continued fraction
        self.h = torch.empty((nz - 1, nx, ny), dtype=torch.complex128, device=dev)
        diag, upper, lower = t(np.diag(z)), t(np.diag(z, 1)), t(np.diag(z, -1))
        N.check(N.load().usv_z_transfer(N.ptr(shift), N.ptr(diag), N.ptr(upper), N.ptr(lower),
                                        N.ptr(self.h), nx * ny, nz, N.stream_handle(torch, dev)),
                "z transfer")
        self.schur = shift + complex(z[0, 0]) + complex(z[0, 1]) * self.h[0]
        self.surface_rhs = None

    def _numpy(self, value):
        return value.detach().cpu().numpy() if torch.is_tensor(value) else np.asarray(value)

    def transform(self, plane):
        return self.ix @ plane @ self.iy.T

    def inverse_transform(self, plane):
        return self.vx @ plane @ self.vy.T

    def _validate_flux_masses(self, masses):
        if boundary_type(self.boundaries.get("-z", "reflecting")) != "reflecting":
            raise ValueError("Sinc Neumann source requires a reflecting/baffled bottom")
        m = masses.toarray() if hasattr(masses, "toarray") else self._numpy(masses)
        if (m.ndim != 2 or m.shape[0] != np.prod(self.shape[:2]) or m.shape[1] == 0
                or not np.isfinite(m).all()):
            raise ValueError("Invalid source masses")
        active = np.abs(m).sum(axis=1).reshape(self.shape[:2], order="F") > 0
        if np.any(active & self.surface_pml) or any(np.any(a) for a in
                                                     (active[0], active[-1], active[:, 0],
                                                      active[:, -1])):
            raise ValueError("Flux source overlaps PML or side boundaries")
        return m

    def flux_target_response(self, masses, points):
        """(P, M) responses of the discrete FV PDE at the points (plain
        transposes, no conjugation: p = response @ w), homogeneous_surface.py:185-202."""
        m = self._validate_flux_masses(masses)
        low, frac = self._sample_coordinates(points)
        dev = self.device
        lo = torch.as_tensor(low, device=dev)
        f = torch.as_tensor(frac, device=dev, dtype=torch.float64)
        vx = (1 - f[:, 0, None]) * self.vx[lo[:, 0]] + f[:, 0, None] * self.vx[lo[:, 0] + 1]
        vy = (1 - f[:, 1, None]) * self.vy[lo[:, 1]] + f[:, 1, None] * self.vy[lo[:, 1] + 1]
        ones = torch.ones_like(self.h[0])
        h0 = torch.stack([ones if z == 0 else self.h[z - 1] for z in low[:, 2]])
        h1 = self.h[lo[:, 2]]
        hz = (1 - f[:, 2, None, None]) * h0 + f[:, 2, None, None] * h1
        obs = vx[:, :, None] * vy[:, None, :] * hz / self.schur
        kernel = self.ix.T @ obs @ self.iy                      # (P, nx, ny)
        flat = kernel.transpose(1, 2).reshape(len(low), -1)      # Fortran ravel of each plane
        mt = torch.as_tensor(m, device=dev, dtype=torch.complex128)
        return self._numpy(-4 * np.pi / self.dx ** 3 * (flat @ mt))

    def solve_flux(self, masses, phases, amplitudes=None):
        """Normalised baffled Neumann aperture solve (homogeneous_surface.py:204-224)."""
        m = self._validate_flux_masses(masses)
        phases = np.asarray(phases, dtype=float)
        amplitudes = np.ones_like(phases) if amplitudes is None else np.asarray(amplitudes)
        if (phases.ndim != 1 or amplitudes.shape != phases.shape
                or m.shape != (np.prod(self.shape[:2]), len(phases))
                or not np.isfinite(phases).all() or not np.isfinite(amplitudes).all()):
            raise ValueError("Invalid source masses or phases")
        coeff = torch.as_tensor(amplitudes * np.exp(1j * phases), device=self.device)
        mt = torch.as_tensor(m, device=self.device, dtype=torch.complex128)
        rhs = (-4 * np.pi / self.dx ** 3 * (mt @ coeff))
        self.surface_rhs = rhs.reshape(self.shape[1], self.shape[0]).T  # Fortran reshape
        self.surface_modes = self.transform(self.surface_rhs) / self.schur
        self.surface = self.inverse_transform(self.surface_modes)
        self.diagnostics = {"iterations": 0, "eigenvector_condition": self.eigen_condition,
                            "source_integral_min_max": [float(m.sum(axis=0).min()),
                                                        float(m.sum(axis=0).max())]}
        return self.diagnostics

    def plane(self, index):
        if not 0 <= index < self.shape[2]:
            raise ValueError("z index outside grid")
        if index == 0:
            return self._numpy(self.surface)
        return self._numpy(self.inverse_transform(self.h[index - 1] * self.surface_modes))

    def _sample_coordinates(self, points):
        points = np.asarray(points, float)
        coords = points / self.dx
        if (points.ndim != 2 or points.shape[1] != 3 or not np.isfinite(points).all()
                or np.any(coords < -1e-9)
                or np.any(coords > np.asarray(self.shape) - 1 + 1e-9)):
            raise ValueError("Points must lie inside the local grid")
        coords = np.clip(coords, 0, np.asarray(self.shape) - 1)
        low = np.minimum(np.floor(coords).astype(int), np.asarray(self.shape) - 2)
        return low, coords - low

    def sample(self, points):
        """Trilinear physical-grid interpolation, no target snapping."""
        low, frac = self._sample_coordinates(points)
        result = np.zeros(len(low), complex)
        for z in np.unique(np.concatenate((low[:, 2], low[:, 2] + 1))):
            plane = self.plane(int(z))
            for dz in (0, 1):
                sel = np.flatnonzero(low[:, 2] + dz == z)
                for a in (0, 1):
                    for b in (0, 1):
                        wgt = ((frac[sel, 0] if a else 1 - frac[sel, 0])
                               * (frac[sel, 1] if b else 1 - frac[sel, 1])
                               * (frac[sel, 2] if dz else 1 - frac[sel, 2]))
                        result[sel] += wgt * plane[low[sel, 0] + a, low[sel, 1] + b]
        return result
