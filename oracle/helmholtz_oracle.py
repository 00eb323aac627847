"""CPU oracle for the gpu_iterative Helmholtz path (TEST INFRASTRUCTURE ONLY).

This module is the checker, never the product: only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference arm may
import it. The CUDA path in ``ultrasound_solver_b200`` never calls into it.

It restates, in numpy/scipy, the reference algorithm of Rain-Kotsuzui/
ultrasound_solver for this path. Every function cites the reference file:line
it follows (paths relative to the reference project root):

* material blend and sphere SDF      src/algorithm/physics/warp_utils.py:11-23, 52-77
* PML profiles, face terms, edges,    src/algorithm/physics/conservative_helmholtz.py:18-149
  node-centred FV assembly
* sinc_neumann aperture quadrature,   src/algorithm/physics/sinc_aperture.py:19-85
  bilinear deposition, flux RHS
* transducer centres                  src/algorithm/physics/transducer_array.py:20-44
* row-scaled Jacobi GMRES + gates     src/algorithm/solvers/iterative_solver.py:30-104
* material VJP                        src/algorithm/physics/conservative_helmholtz.py:151-175
* phase basis field / VJP / trilinear src/algorithm/training/phase_response_basis.py:139-253
* focal losses and background mask   src/algorithm/training/phase_adjoint_optimizer.py:142-414
* Adam on the phases (adjoint         src/algorithm/baselines/adjoint/__init__.py:38-83
  baseline, optimizer "adam")

The GMRES arithmetic of the reference lives in a third-party dependency that
the reference does not vendor: ``cupy-cuda12x[ctk]>=14.0.0``
(reference requirements.txt:11), function
``cupyx.scipy.sparse.linalg.gmres``. ``cupyx_gmres`` below restates CuPy's
published algorithm (right preconditioning, one-pass classical Gram-Schmidt,
full restart cycles, convergence checked only on the true residual at each
restart, dense least squares of the (m+1) x m Hessenberg). No golden vector
for that library exists in the reference, so its iteration-level behaviour is
parity-unpinned; the SOLUTION it converges to is pinned by direct solves of
the reference's own assembled matrices (tests/golden).
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla
from numpy.polynomial.legendre import leggauss

FACES = ("-x", "+x", "-y", "+y", "-z", "+z")


def face_kind(value):
    """Boundary value -> kind string (conservative_helmholtz.py:13-14)."""
    return value.get("type", "reflecting") if isinstance(value, dict) else value


# --------------------------------------------------------------------------
# a1: materials (warp_utils.py:11-23, 52-77)
# --------------------------------------------------------------------------
def blend_obstacle_material(h, rho_obstacle, c_obstacle, rho_medium, c_medium):
    """Linear blend of 1/rho and 1/(rho c^2) in h (warp_utils.py:11-23)."""
    inv_rho_o = 1.0 / rho_obstacle
    comp_o = 1.0 / (rho_obstacle * c_obstacle ** 2)
    inv_rho = inv_rho_o + (1.0 / rho_medium - inv_rho_o) * h
    comp = comp_o + (1.0 / (rho_medium * c_medium ** 2) - comp_o) * h
    return 1.0 / inv_rho, np.sqrt(inv_rho / comp)


def sphere_sdf(shape, dx, center, radius):
    """Node-centred sphere SDF, node (i,j,k) at (i,j,k)*dx (warp_utils.py:57-61)."""
    axes = [np.arange(n, dtype=np.float64) * dx - float(center[a])
            for a, n in enumerate(shape)]
    sq = (axes[0][:, None, None] ** 2 + axes[1][None, :, None] ** 2
          + axes[2][None, None, :] ** 2)
    return np.sqrt(sq) - float(radius)


def smoothed_heaviside(sdf, width):
    """h = 0 inside, 1 outside, sine-smoothed over +-width (warp_utils.py:66-73)."""
    if width:
        t = np.clip(sdf / width, -1.0, 1.0)
        return 0.5 * (1.0 + t + np.sin(np.pi * t) / np.pi)
    return (sdf > 0).astype(np.float64)


def obstacle_materials(shape, dx, obstacle, rho0, c0, sdf=None):
    """rho, c for one sphere (or precomputed-SDF) obstacle (warp_utils.py:50-77)."""
    kind = obstacle.get("type", "sphere").lower()
    if kind == "sphere":
        sdf = sphere_sdf(shape, dx, obstacle.get("center", [0.04, 0.04, 0.02]),
                         float(obstacle.get("radius", 0.012)))
    elif sdf is None:
        raise ValueError("mesh obstacle requires a precomputed SDF")
    width = float(obstacle.get("smoothing_width_cells", 1.2)) * dx
    h = smoothed_heaviside(np.asarray(sdf, dtype=np.float64), width)
    material = obstacle.get("material", {})
    return blend_obstacle_material(h, float(material.get("density", 1250.0)),
                                   float(material.get("sound_speed", 2200.0)),
                                   rho0, c0)


# --------------------------------------------------------------------------
# a2: operator assembly (conservative_helmholtz.py:18-149)
# --------------------------------------------------------------------------
def pml_profiles(shape, boundaries, pml):
    """Per-axis half-volume weights and complex stretch (conservative_helmholtz.py:36-66)."""
    pml = pml or {}
    cells = int(pml.get("cells", 0))
    strength = float(pml.get("strength", 2.0))
    order = int(pml.get("order", 3))
    if cells < 0 or strength < 0 or not np.isfinite(strength) or order < 1:
        raise ValueError("Invalid PML cells, strength or order")
    faces = pml.get("faces", [f for f in FACES
                              if face_kind(boundaries.get(f, "reflecting")) == "open"])
    if set(faces) - set(FACES):
        raise ValueError("Unknown PML face")
    weights, stretch = [], []
    for axis, n in enumerate(shape):
        w = np.ones(n)
        w[0] = w[-1] = 0.5
        sigma = np.zeros(n)
        active = [f for f in FACES[2 * axis:2 * axis + 2] if f in faces]
        if cells and active:
            if cells * len(active) >= n - 1:
                raise ValueError("PML leaves no physical interior on an axis")
            for f in active:
                if face_kind(boundaries.get(f, "reflecting")) != "open":
                    raise ValueError("PML may only be placed on open faces")
                dist = np.arange(n) if f[0] == "-" else np.arange(n)[::-1]
                sigma = sigma + strength * np.maximum(1 - dist / cells, 0) ** order
        weights.append(w)
        stretch.append(1 + 1j * sigma)
    return weights, stretch


def _bcast(vec, axis):
    shape = [1, 1, 1]
    shape[axis] = len(vec)
    return vec.reshape(shape)


class Operator:
    """Node-centred FV Helmholtz operator (conservative_helmholtz.py:17-149).

    Holds rho, c, the PML profiles, face terms and the fixed (soft-face) mask,
    and assembles the complex128 CSR matrix with Fortran node order
    idx = i + nx*(j + ny*k).
    """

    def __init__(self, rho, c, dx, omega, boundaries, pml=None, fixed_dofs=()):
        self.rho = np.asarray(rho, dtype=np.float64)
        self.c = np.asarray(c, dtype=np.float64)
        self.shape = self.rho.shape
        if len(self.shape) != 3 or min(self.shape) < 2 or self.c.shape != self.shape:
            raise ValueError("rho and c must have the same 3D grid shape, each dimension >= 2")
        if not (np.isfinite(self.rho).all() and np.isfinite(self.c).all()
                and (self.rho > 0).all() and (self.c > 0).all()):
            raise ValueError("density and sound speed must be finite and positive")
        if not np.isfinite(dx) or dx <= 0 or not np.isfinite(omega) or omega <= 0:
            raise ValueError("dx and omega must be finite and positive")
        if set(boundaries) - set(FACES):
            raise ValueError("Unknown boundary face")
        self.dx, self.omega, self.boundaries = float(dx), float(omega), boundaries
        w, s = pml_profiles(self.shape, boundaries, pml)
        self.w1d, self.s1d = w, s
        self.weights = [_bcast(w[a], a) for a in range(3)]
        self.stretch = [_bcast(s[a], a) for a in range(3)]
        self.mass_weight = (self.weights[0] * self.weights[1] * self.weights[2]
                            * self.stretch[0] * self.stretch[1] * self.stretch[2])
        fixed = np.zeros(self.shape, dtype=bool, order="F")
        fixed.ravel(order="F")[np.asarray(fixed_dofs, dtype=int)] = True
        sources = fixed.copy()
        in_pml = np.broadcast_to(sum(st.imag for st in self.stretch) > 0, self.shape)
        if np.any(fixed & in_pml):
            raise ValueError("PML overlaps a source; enlarge the domain or reduce PML thickness")
        self.face_terms = []
        for index, face in enumerate(FACES):
            axis = index // 2
            sel = [slice(None)] * 3
            sel[axis] = 0 if index % 2 == 0 else -1
            sel = tuple(sel)
            value = boundaries.get(face, "reflecting")
            kind = face_kind(value)
            if kind not in ("reflecting", "open", "soft", "impedance"):
                raise ValueError(f"Unsupported boundary {face}: {value!r}")
            if kind == "soft":
                if np.any(sources[sel]):
                    raise ValueError("A pressure-release face conflicts with a source")
                fixed[sel] = True
            if kind in ("open", "impedance"):
                b, cax = [a for a in range(3) if a != axis]
                area = (self.weights[b] * self.weights[cax]
                        * self.stretch[b] * self.stretch[cax])
                area = np.broadcast_to(area, self.shape)[sel] / dx
                if kind == "open":
                    adm = 1 / (self.rho[sel] * self.c[sel])
                else:
                    if not isinstance(value, dict):
                        raise ValueError("impedance requires {type: impedance, impedance: [real, imag]}")
                    z = np.asarray(value.get("impedance"), dtype=float)
                    if z.shape != (2,) or not np.isfinite(z).all() or z[0] < 0 or not np.any(z):
                        raise ValueError("impedance must be finite [real>=0, imag], nonzero, in Pa s/m")
                    adm = 1 / complex(z[0], z[1])
                self.face_terms.append((sel, kind, 1j * omega * area * adm))
        self.fixed = fixed

    def edges(self):
        """(low, high, factor) per axis (conservative_helmholtz.py:105-117)."""
        for axis in range(3):
            lo, hi = [slice(None)] * 3, [slice(None)] * 3
            lo[axis], hi[axis] = slice(None, -1), slice(1, None)
            lo, hi = tuple(lo), tuple(hi)
            b, cax = [a for a in range(3) if a != axis]
            st = self.stretch[axis]
            mid = 0.5 * (st[lo] + st[hi])
            factor = (self.weights[b] * self.weights[cax] * self.stretch[b]
                      * self.stretch[cax] / mid / self.dx ** 2)
            yield lo, hi, factor

    def diagonal_and_edges(self):
        """Dense diagonal (before the fixed-row override) and per-axis edge arrays."""
        rho, c = self.rho, self.c
        diag = self.mass_weight * self.omega ** 2 / (rho * c * c)
        diag = np.array(np.broadcast_to(diag, self.shape), dtype=np.complex128)
        coefs = []
        for lo, hi, factor in self.edges():
            coef = factor * 2 / (rho[lo] + rho[hi])
            diag[lo] -= coef
            diag[hi] -= coef
            coefs.append((lo, hi, np.array(np.broadcast_to(coef, rho[lo].shape))))
        for sel, _, term in self.face_terms:
            diag[sel] += term
        return diag, coefs

    def assemble(self):
        """COO -> CSR with fixed rows reduced to the identity (conservative_helmholtz.py:119-149)."""
        ids = np.arange(self.rho.size).reshape(self.shape, order="F")
        diag, coefs = self.diagonal_and_edges()
        diag[self.fixed] = 1
        rows, cols, vals = [], [], []
        for lo, hi, coef in coefs:
            for src, dst in ((lo, hi), (hi, lo)):
                keep = ~self.fixed[src]
                rows.append(ids[src][keep])
                cols.append(ids[dst][keep])
                vals.append(coef[keep])
        rows.append(ids.ravel())
        cols.append(ids.ravel())
        vals.append(diag.ravel())
        n = self.rho.size
        A = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                          shape=(n, n)).tocsr()
        A.eliminate_zeros()
        return A

    def material_vjp(self, field, adjoint):
        """dL = -Re(lambda^H dA p) w.r.t. rho and c (conservative_helmholtz.py:151-175)."""
        u = np.asarray(field).reshape(self.shape, order="F")
        lam = np.asarray(adjoint).reshape(self.shape, order="F").copy()
        lam[self.fixed] = 0
        mass = self.mass_weight * self.omega ** 2 / (self.rho * self.c ** 2)
        prod = np.conj(lam) * u * mass
        g_rho = np.real(prod / self.rho)
        g_c = np.real(2 * prod / self.c)
        for lo, hi, factor in self.edges():
            dr = -2 * factor / (self.rho[lo] + self.rho[hi]) ** 2
            contrib = -np.real((np.conj(lam[lo]) - np.conj(lam[hi])) * (u[hi] - u[lo]) * dr)
            g_rho[lo] += contrib
            g_rho[hi] += contrib
        for sel, kind, term in self.face_terms:
            if kind == "open":
                contrib = np.real(np.conj(lam[sel]) * u[sel] * term)
                g_rho[sel] += contrib / self.rho[sel]
                g_c[sel] += contrib / self.c[sel]
        return g_rho, g_c


# --------------------------------------------------------------------------
# a3: sinc_neumann sources (sinc_aperture.py:19-85)
# --------------------------------------------------------------------------
def aperture_quadrature(diameter, radial_order=32, angular_order=128):
    """Gauss-Legendre in mu=cos(theta) x uniform angle (sinc_aperture.py:19-33)."""
    if not np.isfinite(diameter) or diameter <= 0:
        raise ValueError("Aperture diameter must be positive")
    if radial_order < 2 or angular_order < 8:
        raise ValueError("Aperture quadrature orders are too small")
    mu, wr = leggauss(radial_order)
    mu, wr = (mu + 1) / 2, wr / 2
    r = diameter / 2 * np.sqrt(1 - mu * mu)
    ang = 2 * np.pi * np.arange(angular_order) / angular_order
    ox = (r[:, None] * np.cos(ang)).ravel()
    oy = (r[:, None] * np.sin(ang)).ravel()
    return np.column_stack((ox, oy, np.zeros(ox.size))), np.repeat(wr / angular_order, angular_order)


def source_mass_matrix(shape_xy, dx, centers, diameter, radial_order=64, angular_order=256):
    """Bilinear unit-mass deposition per emitter (sinc_aperture.py:36-72)."""
    shape_xy = tuple(shape_xy)
    centers = np.asarray(centers, float)
    if (len(shape_xy) != 2 or min(shape_xy) < 3 or not np.isfinite(dx) or dx <= 0
            or centers.ndim != 2 or centers.shape[1] != 3 or not len(centers)
            or not np.isfinite(centers).all() or np.any(centers[:, 2] != 0)):
        raise ValueError("Sources require finite centers on z=0 and a valid xy grid")
    offsets, wq = aperture_quadrature(diameter, radial_order, angular_order)
    extent = (np.asarray(shape_xy) - 1) * dx
    if (np.any(centers[:, :2] - diameter / 2 < dx)
            or np.any(centers[:, :2] + diameter / 2 > extent - dx)):
        raise ValueError("Sinc aperture needs one grid cell clearance from side boundaries")
    n_xy = shape_xy[0] * shape_xy[1]
    cols = []
    for center in centers:
        coord = (center[:2] + offsets[:, :2]) / dx
        low = np.floor(coord).astype(int)
        frac = coord - low
        rows, mass = [], []
        for a in (0, 1):
            fx = frac[:, 0] if a else 1 - frac[:, 0]
            for b in (0, 1):
                fy = frac[:, 1] if b else 1 - frac[:, 1]
                rows.append(low[:, 0] + a + shape_xy[0] * (low[:, 1] + b))
                mass.append(wq * fx * fy)
        # one bincount over all four corners sums each node in input order
        cols.append(np.bincount(np.concatenate(rows), weights=np.concatenate(mass),
                                minlength=n_xy))
    M = sp.csr_matrix(np.column_stack(cols))
    M.eliminate_zeros()
    return M


def flux_rhs_columns(masses, shape, dx, reference_density):
    """B = -2 pi/(rho_ref dx^3) * masses in the z=0 rows (sinc_aperture.py:75-85)."""
    if not np.isfinite(reference_density) or reference_density <= 0:
        raise ValueError("reference_density must be positive")
    top = -2 * np.pi / (reference_density * dx ** 3) * masses
    rest = sp.csr_matrix((int(np.prod(shape)) - masses.shape[0], masses.shape[1]))
    return sp.vstack((top, rest), format="csr")


def grid_centers(array_n, pitch, lx, ly, origin=(0.0, 0.0, 0.0)):
    """x-major n x n emitter centres on z=0 (transducer_array.py:34-44)."""
    cx, cy = origin[0] + lx * 0.5, origin[1] + ly * 0.5
    half = (array_n - 1) * pitch * 0.5
    return np.array([[cx - half + i * pitch, cy - half + j * pitch, 0.0]
                     for i in range(array_n) for j in range(array_n)], dtype=np.float64)


# --------------------------------------------------------------------------
# a4-a7: GMRES (iterative_solver.py:30-104; CuPy's published gmres)
# --------------------------------------------------------------------------
def cupyx_gmres(matvec, psolve, b, restart=20, maxiter=None, rtol=1e-5, atol=0.0,
                callback=None):
    """Restatement of CuPy's ``cupyx.scipy.sparse.linalg.gmres`` (cupy >= 14).

    Right-preconditioned restarted GMRES(m): one-pass classical Gram-Schmidt,
    every cycle runs all m Arnoldi steps, the restart test uses the true
    residual ||b - A M x||, the (m+1) x m least squares is solved densely.
    Returns (M x, info) like the library.
    """
    n = b.shape[0]
    b_norm = np.linalg.norm(b)
    if b_norm == 0:
        return b, 0
    atol = max(float(atol), rtol * float(b_norm))
    maxiter = n * 10 if maxiter is None else maxiter
    m = min(restart, n)
    V = np.empty((n, m), dtype=b.dtype)
    H = np.zeros((m + 1, m), dtype=b.dtype)
    e = np.zeros(m + 1, dtype=b.dtype)
    x = np.zeros_like(b)
    iters = 0
    while True:
        mx = psolve(x)
        r = b - matvec(mx)
        r_norm = np.linalg.norm(r)
        if callback is not None and iters > 0:
            callback(r_norm / b_norm)
        if r_norm <= atol or iters >= maxiter:
            break
        v = r / r_norm
        V[:, 0] = v
        e[0] = r_norm
        for j in range(m):
            u = matvec(psolve(v))
            h = V[:, :j + 1].conj().T @ u
            H[:j + 1, j] = h
            u = u - V[:, :j + 1] @ h
            H[j + 1, j] = np.linalg.norm(u)
            if j + 1 < m:
                v = u / H[j + 1, j]
                V[:, j + 1] = v
        y = np.linalg.lstsq(H, e, rcond=None)[0]
        x = x + V @ y
        iters += m
    info = iters if (iters == maxiter and not r_norm <= atol) else 0
    return mx, info


def row_scale_and_jacobi(A):
    """R = 1/max|row|, M = diag(R A)^-1 (iterative_solver.py:37-56)."""
    row_max = np.asarray(abs(A).max(axis=1).toarray()).ravel()
    R = np.where(row_max > 0, 1.0 / np.where(row_max > 0, row_max, 1.0), 1.0)
    sd = R * A.diagonal()
    inv_d = np.where(np.abs(sd) > 0, 1.0 / np.where(np.abs(sd) > 0, sd, 1.0), 1.0)
    return R, inv_d


class GmresResult:
    def __init__(self, x, info, iterations, scaled_residual, backward_error, history):
        self.x, self.info, self.iterations = x, info, iterations
        self.scaled_residual, self.backward_error = scaled_residual, backward_error
        self.history = history


def iterative_solve(A, rhs, restart=30, maxiter=3000, rtol=1e-6, backward_error_tol=1e-4,
                    raise_on_failure=True):
    """GpuIterativeSolver.solve restated on the CPU (iterative_solver.py:30-104)."""
    rhs = np.asarray(rhs, dtype=np.complex128)
    if np.linalg.norm(rhs) == 0.0:
        return GmresResult(np.zeros_like(rhs), 0, 0, 0.0, 0.0, [])
    R, inv_d = row_scale_and_jacobi(A)
    b = R * rhs
    hist = []
    x, info = cupyx_gmres(lambda v: R * (A @ v), lambda v: inv_d * v, b,
                          restart=restart, maxiter=maxiter, rtol=rtol, atol=0.0,
                          callback=hist.append)
    scaled = float(np.linalg.norm(R * (A @ x) - b) / np.linalg.norm(b))
    res = A @ x - rhs
    den = abs(A) @ np.abs(x) + np.abs(rhs)
    bwd = float(np.max(np.abs(res) / np.maximum(den, 1e-30)))
    iters = len(hist) * restart
    ok = info == 0 and np.isfinite(x).all() and scaled <= rtol and bwd <= backward_error_tol
    if raise_on_failure and not ok:
        raise RuntimeError(f"info={info}, iterations={iters}, scaled residual={scaled:.3e}, "
                           f"backward error={bwd:.3e}")
    return GmresResult(x, info, iters, scaled, bwd, hist)


def direct_solve(A, rhs):
    """FP64 sparse direct solve (SuperLU), the small-grid oracle."""
    lu = spla.splu(sp.csc_matrix(A))
    rhs = np.asarray(rhs, dtype=np.complex128)
    return lu.solve(rhs) if rhs.ndim == 1 else np.column_stack([lu.solve(rhs[:, k])
                                                                for k in range(rhs.shape[1])])


def backward_error(A, x, b):
    """max |Ax-b| / (|A||x| + |b|) (iterative_solver.py:74-79)."""
    res = A @ x - b
    den = abs(A) @ np.abs(x) + np.abs(b)
    return float(np.max(np.abs(res) / np.maximum(den, 1e-30)))


# --------------------------------------------------------------------------
# a9: phase response basis (phase_response_basis.py:139-253)
# --------------------------------------------------------------------------
def basis_field(G, phases):
    """u = G exp(i phi) (phase_response_basis.py:190-199)."""
    return G @ np.exp(1j * np.asarray(phases, dtype=np.float64))


def basis_phase_vjp(G, cotangent, phases):
    """Re(conj(G^H g) * i e^{i phi}) (phase_response_basis.py:225-253)."""
    resp = G.conj().T @ np.asarray(cotangent, dtype=np.complex128).reshape(-1, order="F")
    w = np.exp(1j * np.asarray(phases, dtype=np.float64))
    return np.real(np.conj(resp) * (1j * w))


def trilinear_rows(points, shape, dx, origin=(0.0, 0.0, 0.0)):
    """Fortran node rows and weights of the 8 trilinear corners (phase_response_basis.py:165-175)."""
    points = np.asarray(points, dtype=float)
    shape = np.asarray(shape)
    pos = (points - np.asarray(origin)) / dx
    low = np.minimum(np.floor(pos).astype(int), shape - 2)
    frac = pos - low
    out = []
    for corner in np.ndindex(2, 2, 2):
        corner = np.asarray(corner)
        idx = low + corner
        w = np.prod(np.where(corner, frac, 1 - frac), axis=1)
        rows = idx[:, 0] + shape[0] * (idx[:, 1] + shape[1] * idx[:, 2])
        out.append((rows, w))
    return out


def basis_target_response(G, points, shape, dx, origin=(0.0, 0.0, 0.0)):
    resp = np.zeros((len(points), G.shape[1]), complex)
    for rows, w in trilinear_rows(points, shape, dx, origin):
        resp += w[:, None] * G[rows]
    return resp


# --------------------------------------------------------------------------
# a10: losses (phase_adjoint_optimizer.py:142-414)
# --------------------------------------------------------------------------
def nearest_index(point, dx, origin=(0.0, 0.0, 0.0)):
    """phase_adjoint_optimizer.py:142-144."""
    return tuple(np.rint((np.asarray(point) - np.asarray(origin)) / dx).astype(int))


def _focal(field, indices, weight, eps):
    """phase_adjoint_optimizer.py:210-223 (grid samples)."""
    idx = tuple(np.asarray(indices, dtype=np.intp).T)
    vals = field[idx]
    amp = np.abs(vals)
    loss = -weight * np.mean(amp)
    cot = np.zeros_like(field, dtype=np.complex128)
    contrib = -weight / len(indices) * vals / (amp + eps)
    np.add.at(cot.real, idx, contrib.real)
    np.add.at(cot.imag, idx, contrib.imag)
    return loss, cot


def focal_pressure_loss(field, indices, target_weight=1.0, background_weight=0.05, eps=1e-12):
    """FocalPressureLoss.evaluate (phase_adjoint_optimizer.py:244-258)."""
    loss, cot = _focal(field, indices, target_weight, eps)
    if background_weight > 0:
        loss += 0.5 * background_weight * float(np.mean(np.abs(field) ** 2))
        cot += background_weight / field.size * field
    return float(loss), cot


def background_mask(shape, box, targets, target_radius, exclusion_layers):
    """_build_background_mask (phase_adjoint_optimizer.py:384-414)."""
    if target_radius <= 0:
        raise ValueError("training.target_radius must be positive")
    xs, ys, zs = (np.linspace(0.0, box[a], shape[a]) for a in range(3))
    mask = np.ones(shape, dtype=bool)
    layers = max(int(exclusion_layers), 0)
    if layers > 0:
        mask[:, :, :layers] = False
    for p in targets:
        r2 = ((xs[:, None, None] - p[0]) ** 2 + (ys[None, :, None] - p[1]) ** 2
              + (zs[None, None, :] - p[2]) ** 2)
        mask[r2 <= target_radius * target_radius] = False
    return mask


def focal_contrast_loss(field, indices, mask, target_weight=1.0, sidelobe_weight=0.05,
                        temperature=25.0, eps=1e-12):
    """FocalContrastLoss.evaluate (phase_adjoint_optimizer.py:312-338)."""
    loss, cot = _focal(field, indices, target_weight, eps)
    amp = np.abs(field)
    bg = amp[mask]
    mx = float(np.max(bg))
    wts = np.exp((bg - mx) / temperature)
    prob = wts / np.sum(wts)
    loss += sidelobe_weight * float(mx + temperature * (np.log(np.sum(wts)) - np.log(bg.size)))
    cot[mask] += sidelobe_weight * prob * field[mask] / (bg + eps)
    return float(loss), cot


# --------------------------------------------------------------------------
# scene: config dict (reference YAML schema) -> rho, c, A, B
# (helmholtz_solver.py:273-369 + warp_utils.py:33-120)
# --------------------------------------------------------------------------
class Scene:
    """Everything the reference's assemble_matrix() produces for one config."""


def grid_dx(domain):
    """Isotropic node spacing L/(N-1) (config.py:67-83)."""
    box = np.asarray(domain["box_size"], dtype=float)
    n = np.asarray(domain["grid_size"], dtype=float)
    d = box / (n - 1)
    if not (np.isclose(d[0], d[1]) and np.isclose(d[0], d[2])):
        raise ValueError("anisotropic grid")
    return float(d[0])


def build_scene(cfg, material_fields=None, phases=None):
    """Assemble one scene the way HelmholtzDirectSolver.assemble_matrix does."""
    dom = cfg["domain"]
    shape = tuple(int(n) for n in dom["grid_size"])
    dx = grid_dx(dom)
    origin = np.asarray(dom.get("origin_m", [0.0, 0.0, 0.0]), dtype=float)
    phys = cfg["physics"]
    c0 = float(phys.get("sound_speed", 343.0))
    rho0 = float(phys.get("medium_density", 1.21))
    spec = cfg["transducer_specs"]
    freq = float(spec.get("frequency", 40000.0))
    omega = 2 * np.pi * freq
    bcs = cfg["boundary_conditions"]
    solver = cfg.get("solver", {})
    pml = solver.get("pml")
    if (c0 / freq) / dx < 6:
        raise ValueError("fewer than 6 points per background wavelength")
    obstacles = cfg.get("obstacles", [])
    if len(obstacles) > 1:
        raise NotImplementedError("one obstacle at a time")
    if material_fields is not None:
        if obstacles:
            raise ValueError("Explicit material fields and obstacle materials are mutually exclusive")
        rho, c = (np.asarray(a, dtype=np.float64) for a in material_fields)
    elif obstacles:
        ob = dict(obstacles[0])
        if ob.get("type", "sphere").lower() == "sphere":
            ob["center"] = (np.asarray(ob.get("center", [0.04, 0.04, 0.02]), float) - origin).tolist()
        rho, c = obstacle_materials(shape, dx, ob, rho0, c0)
    else:
        rho, c = np.full(shape, rho0), np.full(shape, c0)
    n_side = int(spec.get("array_n", 6))
    lx, ly = float(dom["box_size"][0]), float(dom["box_size"][1])
    centers = grid_centers(n_side, float(spec.get("pitch", 0.0105)), lx, ly, origin) - origin
    if face_kind(bcs.get("-z", "reflecting")) != "reflecting":
        raise ValueError("The sinc Neumann source requires a reflecting baffled bottom plane")
    masses = source_mass_matrix(shape[:2], dx, centers, float(spec.get("diameter", 0.0098)),
                                int(spec.get("source_radial_order", 64)),
                                int(spec.get("source_angular_order", 256)))
    B = flux_rhs_columns(masses, shape, dx, rho0)
    op = Operator(rho, c, dx, omega, bcs, pml=pml)
    active = np.asarray(abs(B).sum(axis=1)).ravel() > 0
    in_pml = np.broadcast_to(sum(s.imag for s in op.stretch), shape).ravel(order="F") > 0
    if np.any(active & in_pml):
        raise ValueError("PML overlaps the deposited sinc aperture")
    if np.any(active & op.fixed.ravel(order="F")):
        raise ValueError("Sinc flux conflicts with a pressure-release boundary")
    if c.min() / freq / dx < 6:
        raise ValueError("fewer than 6 points per shortest local wavelength")
    A = op.assemble()
    sc = Scene()
    sc.shape, sc.dx, sc.omega, sc.origin = shape, dx, omega, origin
    sc.rho, sc.c, sc.op, sc.A, sc.B, sc.masses, sc.centers = rho, c, op, A, B, masses, centers
    sc.amplitudes = np.ones(len(centers))
    sc.phases = np.zeros(len(centers)) if phases is None else np.asarray(phases, float)
    sc.rhs = B @ (sc.amplitudes * np.exp(1j * sc.phases))
    return sc


# --------------------------------------------------------------------------
# Adam phase optimisation (src/algorithm/baselines/adjoint/__init__.py:38-83)
# --------------------------------------------------------------------------
def phase_gradient(B, amplitudes, lam, phases):
    """dL/dphi_m = Re(conj((B^H lam)_m) a_m i e^{i phi_m}) for dL = Re(g^H du),
    lam = A^-H g (the basis VJP of phase_response_basis.py:208-253 with
    G = A^-1 B diag(a))."""
    proj = B.conj().T @ lam
    return np.real(np.conj(proj) * np.asarray(amplitudes) * 1j * np.exp(1j * np.asarray(phases)))


def adam_trajectory(A, B, amplitudes, phases0, loss_fn, steps, learning_rate=0.05):
    """Phases and losses of `steps` Adam updates (adjoint/__init__.py:71-83),
    every evaluation a direct forward solve and a direct A^H solve.
    loss_fn(u) -> (loss, cotangent). Returns (phases per evaluation,
    losses per evaluation, gradients per evaluation)."""
    lu = spla.splu(sp.csc_matrix(A))
    amps = np.asarray(amplitudes, dtype=np.float64)

    def evaluate(ph):
        u = lu.solve(B @ (amps * np.exp(1j * ph)))
        loss, cot = loss_fn(u)
        lam = lu.solve(np.asarray(cot, dtype=np.complex128).ravel(), trans="H")
        return loss, phase_gradient(B, amps, lam, ph)

    ph = np.asarray(phases0, dtype=np.float64).copy()
    loss, grad = evaluate(ph)
    phases, losses, grads = [ph.copy()], [loss], [grad]
    first = np.zeros_like(ph)
    second = np.zeros_like(ph)
    for step in range(1, steps + 1):
        first = 0.9 * first + 0.1 * grad
        second = 0.999 * second + 0.001 * grad ** 2
        ph = ph - learning_rate * (first / (1 - 0.9 ** step)) / (
            np.sqrt(second / (1 - 0.999 ** step)) + 1e-8)
        loss, grad = evaluate(ph)
        phases.append(ph.copy())
        losses.append(loss)
        grads.append(grad)
    return phases, losses, grads
