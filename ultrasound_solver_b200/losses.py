"""Focal losses with device cotangents (usv_loss).

Mirrors FocalPressureLoss / FocalContrastLoss of
src/algorithm/training/phase_adjoint_optimizer.py:142-414: same constructor
arguments (cfg, amplitude_target, eps), same targets (nearest grid node of
each cfg.targets point), same background mask, same loss values and
cotangents in the dL = Re(g^H du) convention (which is also the gradient
convention of torch). `evaluate_device` takes and returns device tensors;
`evaluate` accepts numpy arrays. ContrastRatioLoss is the focal-contrast
objective |u_t|^2 / mean_shell |u|^2 (maximised) of the adjoint-gradient
benchmark.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _native as N
from .scene import as_grid


def nearest_grid_index(cfg, point) -> tuple[int, int, int]:
    """phase_adjoint_optimizer.py:142-144."""
    dx = cfg.domain.dx
    return tuple(np.rint((np.asarray(point, float) - np.asarray(cfg.domain.origin_m)) / dx)
                 .astype(int))


def background_mask(cfg, target_points, target_radius, source_exclusion_layers) -> np.ndarray:
    """_build_background_mask (phase_adjoint_optimizer.py:384-414)."""
    if target_radius <= 0.0:
        raise ValueError("training.target_radius must be positive")
    shape = tuple(cfg.domain.grid_size)
    xs, ys, zs = (np.linspace(0.0, L, n) for L, n in zip(cfg.domain.box_size, shape))
    mask = np.ones(shape, dtype=bool)
    layers = max(int(source_exclusion_layers), 0)
    if layers > 0:
        mask[:, :, :layers] = False
    r2max = target_radius * target_radius
    for p in np.asarray(target_points, dtype=float):
        r2 = ((xs[:, None, None] - p[0]) ** 2 + (ys[None, :, None] - p[1]) ** 2
              + (zs[None, None, :] - p[2]) ** 2)
        mask[r2 <= r2max] = False
    return mask


def _flat(shape, idx) -> int:
    return int(idx[0] + shape[0] * (idx[1] + shape[1] * idx[2]))


def _to_device_vector(field, device):
    if isinstance(field, torch.Tensor):
        t = field.to(device=device, dtype=torch.complex128)
        return (t.reshape(-1) if t.dim() == 1 else t.permute(2, 1, 0).reshape(-1)).contiguous()
    a = np.asarray(field, dtype=np.complex128).reshape(-1, order="F")
    return torch.from_numpy(np.ascontiguousarray(a)).to(device)


class _DeviceLoss:
    mode = N.LOSS_FOCAL_PRESSURE

    def __init__(self, cfg, target_indices, mask, target_weight, background_weight,
                 temperature, eps, device=None):
        self.cfg = cfg
        self.shape = tuple(cfg.domain.grid_size)
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None \
            else torch.device(device)
        self.target_indices = [tuple(int(v) for v in t) for t in target_indices]
        if not self.target_indices:
            raise ValueError("phase_optimization requires targets or training.target_field_file")
        flat = [_flat(self.shape, t) for t in self.target_indices]
        self._targets = torch.tensor(flat, dtype=torch.int64, device=self.device)
        self._mask = None if mask is None else torch.from_numpy(
            np.ascontiguousarray(np.asarray(mask, dtype=np.uint8).reshape(-1, order="F"))
        ).to(self.device)
        self.target_weight = float(target_weight)
        self.background_weight = float(background_weight)
        self.temperature = float(temperature)
        self.eps = float(eps)
        n = int(np.prod(self.shape))
        nbytes = C.c_size_t()
        N.check(N.load().usv_loss_workspace_bytes(n, C.byref(nbytes)), "loss workspace")
        self._ws = torch.empty(nbytes.value, dtype=torch.uint8, device=self.device)
        self._value = torch.empty(3, dtype=torch.float64, device=self.device)

    def evaluate_vector(self, u: torch.Tensor, with_cotangent: bool = True):
        """u: device complex128 vector in Fortran order -> (loss 0-d tensor, cotangent vector)."""
        u = u.to(device=self.device, dtype=torch.complex128).contiguous()
        cot = torch.empty_like(u) if with_cotangent else None
        N.check(N.load().usv_loss(
            self.mode, N.ptr(u), u.numel(),
            N.ptr(self._mask) if self._mask is not None else None,
            N.ptr(self._targets), len(self.target_indices), self.target_weight,
            self.background_weight, self.temperature, self.eps, N.ptr(self._value),
            N.ptr(cot) if cot is not None else None, N.ptr(self._ws), self._ws.numel(),
            N.stream_handle(torch, self.device)), "loss")
        return self._value[0].clone(), cot

    def evaluate_device(self, field, with_cotangent: bool = True, focal_field=None):
        if focal_field is not None:
            raise NotImplementedError("external focal samples are not supported on this path")
        vec = _to_device_vector(field, self.device)
        loss, cot = self.evaluate_vector(vec, with_cotangent)
        return loss, (as_grid(cot, self.shape) if cot is not None else None)

    def evaluate(self, field, with_cotangent: bool = True, focal_field=None):
        loss, cot = self.evaluate_device(field, with_cotangent, focal_field)
        return float(loss.item()), (cot.cpu().numpy() if cot is not None else None)


class FocalPressureLoss(_DeviceLoss):
    """-w_t mean |u_t| + 0.5 w_b mean |u|^2 (phase_adjoint_optimizer.py:226-270)."""

    mode = N.LOSS_FOCAL_PRESSURE

    def __init__(self, cfg, amplitude_target=None, eps: float = 1.0e-12, device=None):
        t = cfg.training
        super().__init__(cfg, [nearest_grid_index(cfg, p) for p in cfg.targets], None,
                         t.target_weight, t.background_weight, 1.0, eps, device)


class FocalContrastLoss(_DeviceLoss):
    """-w_t mean |u_t| + w_s softmax_T(|u| on the background) (phase_adjoint_optimizer.py:283-364)."""

    mode = N.LOSS_FOCAL_CONTRAST

    def __init__(self, cfg, amplitude_target=None, eps: float = 1.0e-12, device=None):
        t = cfg.training
        if float(t.sidelobe_temperature) <= 0.0:
            raise ValueError("training.sidelobe_temperature must be positive")
        mask = background_mask(cfg, cfg.targets, float(t.target_radius),
                               int(t.source_exclusion_layers))
        if not np.any(mask):
            raise ValueError("focal_contrast background mask is empty")
        self.background_mask = mask
        super().__init__(cfg, [nearest_grid_index(cfg, p) for p in cfg.targets], mask,
                         t.target_weight, t.background_weight, t.sidelobe_temperature, eps,
                         device)


class ContrastRatioLoss(_DeviceLoss):
    """-|u_t|^2 / mean_shell |u|^2: shell = focal_radius < r <= focal_radius + shell_thickness."""

    mode = N.LOSS_CONTRAST_RATIO

    def __init__(self, cfg, target_point, focal_radius=0.006, shell_thickness=0.010, device=None):
        shape = tuple(cfg.domain.grid_size)
        xs, ys, zs = (np.linspace(0.0, L, n) for L, n in zip(cfg.domain.box_size, shape))
        p = np.asarray(target_point, float) - np.asarray(cfg.domain.origin_m)
        r = np.sqrt((xs[:, None, None] - p[0]) ** 2 + (ys[None, :, None] - p[1]) ** 2
                    + (zs[None, None, :] - p[2]) ** 2)
        mask = (r > focal_radius) & (r <= focal_radius + shell_thickness)
        if not np.any(mask):
            raise ValueError("focal shell is empty")
        self.shell_mask = mask
        super().__init__(cfg, [nearest_grid_index(cfg, target_point)], mask, 1.0, 0.0, 1.0,
                         1e-12, device)
