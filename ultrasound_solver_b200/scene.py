"""Device-resident scene: materials, matrix-free operator and source columns.

Host code here only validates inputs (with the reference's error messages)
and hands device buffers to the CUDA library; every O(N) step runs on the GPU:

* materials: WarpAssemblyEngine material stage (src/algorithm/physics/warp_utils.py:33-81)
  -> ``usv_materials_blend``
* operator: ConservativeHelmholtz (src/algorithm/physics/conservative_helmholtz.py:18-149)
  -> ``usv_operator_build`` (per-node records, no CSR)
* sources: source_mass_matrix / flux_rhs_columns / assemble_rhs
  (src/algorithm/physics/sinc_aperture.py:19-85, warp_utils.py:95-120)
  -> ``usv_source_masses`` / ``usv_source_rhs``
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch
from numpy.polynomial.legendre import leggauss

from . import _native as N

FACES = ("-x", "+x", "-y", "+y", "-z", "+z")
_KIND = {"reflecting": N.FACE_REFLECTING, "open": N.FACE_OPEN, "soft": N.FACE_SOFT,
         "impedance": N.FACE_IMPEDANCE}


def boundary_type(value):
    """conservative_helmholtz.py:13-14."""
    return value.get("type", "reflecting") if isinstance(value, dict) else value


def require_cuda(device=None) -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("ultrasound_solver_b200 needs a CUDA device (sm_100a); none is visible")
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    if dev.type != "cuda":
        raise ValueError("device must be a CUDA device")
    return dev


def fortran_flat(array, device, dtype=torch.float64) -> torch.Tensor:
    """(nx,ny,nz) host array -> device vector in Fortran node order."""
    a = np.asarray(array)
    return torch.from_numpy(np.ascontiguousarray(a.ravel(order="F"))).to(device=device, dtype=dtype)


def as_grid(vec: torch.Tensor, shape) -> torch.Tensor:
    """Device vector in Fortran order -> (nx,ny,nz) view (no copy)."""
    nx, ny, nz = shape
    return vec.view(*vec.shape[:-1], nz, ny, nx).transpose(-1, -3)


def make_scene(shape, dx, omega, boundaries, pml=None) -> N.Scene:
    """Validate faces / PML like conservative_helmholtz.py:29-103 and pack usv_scene."""
    if len(shape) != 3 or min(shape) < 2:
        raise ValueError("rho and c must have the same 3D grid shape, each dimension >= 2")
    if not np.isfinite(dx) or dx <= 0 or not np.isfinite(omega) or omega <= 0:
        raise ValueError("dx and omega must be finite and positive")
    if set(boundaries) - set(FACES):
        raise ValueError("Unknown boundary face")
    pml = pml or {}
    cells = int(pml.get("cells", 0))
    strength = float(pml.get("strength", 2.0))
    order = int(pml.get("order", 3))
    if cells < 0 or strength < 0 or not np.isfinite(strength) or order < 1:
        raise ValueError("Invalid PML cells, strength or order")
    pml_faces = pml.get("faces", [f for f in FACES
                                  if boundary_type(boundaries.get(f, "reflecting")) == "open"])
    if set(pml_faces) - set(FACES):
        raise ValueError("Unknown PML face")
    s = N.Scene()
    s.nx, s.ny, s.nz = (int(v) for v in shape)
    s.dx, s.omega = float(dx), float(omega)
    for axis, n in enumerate(shape):
        active = [f for f in FACES[2 * axis:2 * axis + 2] if f in pml_faces]
        if cells and active:
            if cells * len(active) >= n - 1:
                raise ValueError("PML leaves no physical interior on an axis")
            for face in active:
                if boundary_type(boundaries.get(face, "reflecting")) != "open":
                    raise ValueError("PML may only be placed on open faces")
    mask = 0
    for f in pml_faces:
        mask |= 1 << FACES.index(f)
    s.pml_cells, s.pml_strength, s.pml_order = cells, strength, order
    s.pml_faces = mask if cells else 0
    for index, face in enumerate(FACES):
        value = boundaries.get(face, "reflecting")
        kind = boundary_type(value)
        if kind not in _KIND:
            raise ValueError(f"Unsupported boundary {face}: {value!r}")
        s.face_kind[index] = _KIND[kind]
        if kind == "impedance":
            if not isinstance(value, dict):
                raise ValueError("impedance requires {type: impedance, impedance: [real, imag]}")
            z = np.asarray(value.get("impedance"), dtype=float)
            if z.shape != (2,) or not np.isfinite(z).all() or z[0] < 0 or not np.any(z):
                raise ValueError("impedance must be finite [real>=0, imag], nonzero, in Pa s/m")
            s.impedance_re[index], s.impedance_im[index] = float(z[0]), float(z[1])
    return s


class DeviceOperator:
    """Matrix-free FV Helmholtz operator resident on one CUDA device.

    ``rho`` and ``c`` are float64 device vectors in Fortran node order. The
    per-node records live in ``self.buffer`` (a torch uint8 tensor).
    """

    def __init__(self, shape, dx, omega, boundaries, rho: torch.Tensor, c: torch.Tensor,
                 pml=None):
        self.shape = tuple(int(v) for v in shape)
        self.n = int(np.prod(self.shape))
        self.scene = make_scene(self.shape, dx, omega, boundaries, pml)
        self.dx, self.omega = float(dx), float(omega)
        self.boundaries, self.pml = boundaries, pml
        if rho.shape != (self.n,) or c.shape != (self.n,):
            raise ValueError("rho and c must have the same 3D grid shape, each dimension >= 2")
        if not (bool(torch.isfinite(rho).all()) and bool(torch.isfinite(c).all())
                and bool((rho > 0).all()) and bool((c > 0).all())):
            raise ValueError("density and sound speed must be finite and positive")
        self.device = rho.device
        self.stencil_kernel = N.STENCIL_AUTO
        self.rho = rho.to(torch.float64).contiguous()
        self.c = c.to(torch.float64).contiguous()
        lib = N.load()
        nbytes = C.c_size_t()
        N.check(lib.usv_operator_bytes(C.byref(self.scene), C.byref(nbytes)), "operator layout")
        self.buffer = torch.empty(nbytes.value, dtype=torch.uint8, device=self.device)
        with torch.cuda.device(self.device):
            N.check(lib.usv_operator_build(C.byref(self.scene), N.ptr(self.rho), N.ptr(self.c),
                                           N.ptr(self.buffer), nbytes.value,
                                           N.stream_handle(torch, self.device)),
                    "operator build")

    @property
    def fixed_mask(self) -> np.ndarray:
        """Soft-face nodes (the reference's fixed DOFs), (nx,ny,nz) bool."""
        m = np.zeros(self.shape, dtype=bool)
        for index, face in enumerate(FACES):
            if self.scene.face_kind[index] == N.FACE_SOFT:
                sel = [slice(None)] * 3
                sel[index // 2] = 0 if index % 2 == 0 else -1
                m[tuple(sel)] = True
        return m

    def fixed_dofs(self) -> np.ndarray:
        return np.flatnonzero(self.fixed_mask.ravel(order="F"))

    def apply(self, x: torch.Tensor, variant: int = N.APPLY_A, precision: int = N.PREC_FP64,
              kernel: int | None = None):
        """y = OP x for x of shape (N,) or (B, N) (complex128; complex64 allowed for K/KH mixed).

        `kernel` selects the complex64 K / K^H stencil (N.STENCIL_*); None
        uses `self.stencil_kernel` (set by autotune.StencilTuner, default auto)."""
        squeeze = x.dim() == 1
        xb = x.reshape(1, -1) if squeeze else x
        if xb.shape[-1] != self.n:
            raise ValueError("vector length does not match the grid")
        want = torch.complex64 if (variant in (N.APPLY_K, N.APPLY_KH)
                                   and precision == N.PREC_MIXED) else torch.complex128
        xb = xb.to(device=self.device, dtype=want).contiguous()
        y = torch.empty_like(xb)
        k = self.stencil_kernel if kernel is None else int(kernel)
        if k == N.STENCIL_RECORD_TILES and xb.shape[0] > 4:
            k = N.STENCIL_AUTO  # the record-tile kernel takes at most 4 right-hand sides
        N.check(N.load().usv_operator_apply_kernel(C.byref(self.scene), N.ptr(self.buffer), variant,
                                                   precision, k, N.ptr(xb), N.ptr(y), xb.shape[0],
                                                   self.n, N.stream_handle(torch, self.device)),
                "apply")
        return y[0] if squeeze else y

    def export(self):
        """diag (complex128), R, s (complex128), R_adj, s_adj as device tensors."""
        diag = torch.empty(self.n, dtype=torch.complex128, device=self.device)
        jac = torch.empty_like(diag)
        jaca = torch.empty_like(diag)
        rs = torch.empty(self.n, dtype=torch.float64, device=self.device)
        rsa = torch.empty_like(rs)
        N.check(N.load().usv_operator_export(C.byref(self.scene), N.ptr(self.buffer), N.ptr(diag),
                                             N.ptr(rs), N.ptr(jac), N.ptr(rsa), N.ptr(jaca),
                                             N.stream_handle(torch, self.device)), "export")
        return diag, rs, jac, rsa, jaca

    def pml_mask(self) -> np.ndarray:
        """Nodes with a positive PML stretch, (nx,ny,nz) bool."""
        m = np.zeros(self.shape, dtype=bool)
        cells = self.scene.pml_cells
        if not cells:
            return m
        for index in range(6):
            if not self.scene.pml_faces & (1 << index):
                continue
            axis, n = index // 2, self.shape[index // 2]
            sel = [slice(None)] * 3
            sel[axis] = slice(0, cells) if index % 2 == 0 else slice(n - cells, n)
            m[tuple(sel)] = True
        return m


def aperture_quadrature(diameter, radial_order=32, angular_order=128):
    """Gauss-Legendre in mu = cos(theta) x uniform angle (sinc_aperture.py:19-33)."""
    if not np.isfinite(diameter) or diameter <= 0:
        raise ValueError("Aperture diameter must be positive")
    if radial_order < 2 or angular_order < 8:
        raise ValueError("Aperture quadrature orders are too small")
    mu, w = leggauss(radial_order)
    mu, w = (mu + 1) / 2, w / 2
    r = diameter / 2 * np.sqrt(1 - mu * mu)
    phi = 2 * np.pi * np.arange(angular_order) / angular_order
    qx = (r[:, None] * np.cos(phi)).ravel()
    qy = (r[:, None] * np.sin(phi)).ravel()
    qw = np.repeat(w / angular_order, angular_order)
    return qx, qy, qw


class SourceColumns:
    """sinc_neumann flux columns B (N x M), stored as the z=0 masses (nx*ny x M)."""

    def __init__(self, op: DeviceOperator, centers, diameter, reference_density,
                 radial_order=64, angular_order=256):
        centers = np.ascontiguousarray(np.asarray(centers, dtype=np.float64))
        nx, ny, _ = op.shape
        if (min(nx, ny) < 3 or centers.ndim != 2 or centers.shape[1] != 3 or not len(centers)
                or not np.isfinite(centers).all() or np.any(centers[:, 2] != 0)):
            raise ValueError("Sources require finite centers on z=0 and a valid xy grid")
        if not np.isfinite(reference_density) or reference_density <= 0:
            raise ValueError("reference_density must be positive")
        qx, qy, qw = aperture_quadrature(diameter, radial_order, angular_order)
        dev = op.device
        self.op, self.m = op, len(centers)
        self.centers = centers
        self.reference_density = float(reference_density)
        self.masses = torch.empty(nx * ny * self.m + 1, dtype=torch.float64, device=dev)
        tq = [torch.from_numpy(a).to(dev) for a in (qx, qy, qw)]
        cdev = torch.from_numpy(centers).to(dev)
        st = N.load().usv_source_masses(
            C.byref(op.scene), N.ptr(op.buffer), centers.ctypes.data_as(C.c_void_p), N.ptr(cdev),
            self.m, float(diameter), N.ptr(tq[0]), N.ptr(tq[1]), N.ptr(tq[2]), len(qx),
            N.ptr(self.masses), N.stream_handle(torch, dev))
        if st == N.USV_ERR_SOURCE_CLEARANCE:
            raise ValueError("Sinc aperture needs one grid cell clearance from side boundaries")
        if st == N.USV_ERR_SOURCE_PML:
            raise ValueError("PML overlaps the deposited sinc aperture")
        if st == N.USV_ERR_SOURCE_SOFT:
            raise ValueError("Sinc flux conflicts with a pressure-release boundary")
        N.check(st, "source masses")

    @property
    def mass_matrix(self) -> torch.Tensor:
        nxy = self.op.shape[0] * self.op.shape[1]
        return self.masses[:nxy * self.m].view(self.m, nxy)

    def coverage(self) -> np.ndarray:
        """Total |mass| per emitter (a zero column means the grid missed it)."""
        return self.mass_matrix.abs().sum(dim=1).cpu().numpy()

    def rhs(self, coefficients: torch.Tensor) -> torch.Tensor:
        """b[:, k] = B @ coefficients[k] for coefficients (K, M) complex128 -> (K, N)."""
        coeff = coefficients.to(device=self.op.device, dtype=torch.complex128).contiguous()
        if coeff.dim() == 1:
            coeff = coeff.view(1, -1)
        if coeff.shape[1] != self.m:
            raise ValueError("coefficient count does not match the emitters")
        out = torch.empty((coeff.shape[0], self.op.n), dtype=torch.complex128, device=self.op.device)
        N.check(N.load().usv_source_rhs(C.byref(self.op.scene), N.ptr(self.masses), self.m,
                                        N.ptr(coeff), self.reference_density, N.ptr(out),
                                        coeff.shape[0], self.op.n,
                                        N.stream_handle(torch, self.op.device)), "source rhs")
        return out

    def phase_rhs(self, amplitudes, phases) -> torch.Tensor:
        """assemble_rhs: B (a e^{i phi}) (warp_utils.py:118-120) -> (N,)."""
        a = torch.as_tensor(np.asarray(amplitudes, dtype=np.float64), device=self.op.device)
        p = torch.as_tensor(np.asarray(phases, dtype=np.float64), device=self.op.device)
        return self.rhs((a * torch.exp(1j * p)).view(1, -1))[0]

    def column_rhs(self, amplitudes, start=0, stop=None) -> torch.Tensor:
        """Single-transducer columns B[:, m] a_m for m in [start, stop) -> (K, N)."""
        stop = self.m if stop is None else stop
        a = np.asarray(amplitudes, dtype=np.float64)
        coeff = np.zeros((stop - start, self.m), dtype=np.complex128)
        coeff[np.arange(stop - start), np.arange(start, stop)] = a[start:stop]
        return self.rhs(torch.from_numpy(coeff))

    def phase_grad(self, lam: torch.Tensor, amplitudes, phases) -> torch.Tensor:
        """dL/dphi_m = Re(conj(a_m (B^H lam)_m) i e^{i phi_m}) for dL = Re(g^H du)."""
        dev = self.op.device
        lam = lam.to(device=dev, dtype=torch.complex128).contiguous()
        ph = torch.as_tensor(np.asarray(phases, dtype=np.float64), device=dev)
        am = torch.as_tensor(np.asarray(amplitudes, dtype=np.float64), device=dev)
        grad = torch.zeros(self.m, dtype=torch.float64, device=dev)
        N.check(N.load().usv_source_phase_grad(C.byref(self.op.scene), N.ptr(self.masses), self.m,
                                               N.ptr(lam), N.ptr(ph), N.ptr(am),
                                               self.reference_density, N.ptr(grad),
                                               N.stream_handle(torch, dev)), "phase grad")
        return grad


def blend_materials(op_shape, dx, device, obstacle, rho0, c0, rho_medium=None, c_medium=None,
                    sdf=None):
    """rho, c (device, Fortran order) from one obstacle over a scalar or array medium."""
    kind = obstacle.get("type", "sphere").lower()
    width = float(obstacle.get("smoothing_width_cells", 1.2)) * dx
    if not np.isfinite(width) or width < 0:
        raise ValueError("smoothing_width_cells must be finite and >= 0")
    material = obstacle.get("material", {})
    rho_o = float(material.get("density", 1250.0))
    c_o = float(material.get("sound_speed", 2200.0))
    scene = N.Scene()
    scene.nx, scene.ny, scene.nz = op_shape
    scene.dx = dx
    n = int(np.prod(op_shape))
    rho = torch.empty(n, dtype=torch.float64, device=device)
    c = torch.empty_like(rho)
    center = None
    sdf_t = None
    if kind == "sphere":
        center = np.asarray(obstacle.get("center", [0.04, 0.04, 0.02]), dtype=np.float64)
        radius = float(obstacle.get("radius", 0.012))
    elif kind in ("mesh", "sdf"):
        if sdf is None:
            raise ValueError("mesh obstacle requires a precomputed SDF (obs_sdf)")
        sdf = np.asarray(sdf, dtype=np.float64)
        if sdf.shape != tuple(op_shape) or not np.isfinite(sdf).all():
            raise ValueError("SDF must be finite and match the grid")
        sdf_t = fortran_flat(sdf, device)
        radius = 0.0
    else:
        raise ValueError(f"Unsupported obstacle type: {kind!r}")
    cptr = center.ctypes.data_as(C.c_void_p) if center is not None else None
    N.check(N.load().usv_materials_blend(
        C.byref(scene), N.ptr(sdf_t) if sdf_t is not None else None, cptr, radius, width, rho_o,
        c_o, N.ptr(rho_medium) if rho_medium is not None else None,
        N.ptr(c_medium) if c_medium is not None else None, float(rho0), float(c0), N.ptr(rho),
        N.ptr(c), N.stream_handle(torch, device)), "materials")
    return rho, c
