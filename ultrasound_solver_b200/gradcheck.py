"""Adjoint phase-gradient check on the config-3 scene.

    python -m ultrasound_solver_b200.gradcheck [--grid 128] [--fd 8] [--out result.json]

128^3 config-1 medium with a 16 x 16 array (fit to the PML-free interior),
loss = -|u_t|^2 / mean_shell |u|^2 with the target 80 mm above the array
centre, a 6 mm focal sphere and a 10 mm shell. The gradient w.r.t. all
phases comes from one forward and one adjoint (A^H) solve behind
torch.autograd (PhaseField + LossOfField, mixed precision); it is compared
with central finite differences (step 1e-4 rad) on `--fd` seeded phases and
with the same adjoint computed in complex128. Prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch

from . import workloads as W
from .autograd import loss_of_field, phase_field
from .losses import ContrastRatioLoss


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--grid", type=int, default=128)
    ap.add_argument("--fd", type=int, default=8)
    ap.add_argument("--step", type=float, default=1e-4)
    ap.add_argument("--restart", type=int, default=112)
    ap.add_argument("--rtol", type=float, default=1e-10)
    ap.add_argument("--out", default="")
    args = ap.parse_args(argv)
    torch.cuda.set_device(0)
    cfg = W.config3(n=args.grid)
    solver = W.build_solver(cfg, seed=0)
    solver.assemble_matrix()
    it = solver.iterative_solver
    it.restart, it.rtol, it.maxiter = args.restart, args.rtol, 200000
    centre = (args.grid - 1) * solver.cfg.domain.dx / 2
    target = (centre, centre, 0.080)
    loss = ContrastRatioLoss(solver.cfg, target, focal_radius=0.006, shell_thickness=0.010)
    m = solver.transducers.num_transducers
    phases0 = np.random.default_rng(2).uniform(0, 2 * np.pi, m)

    def gradient(precision):
        it.precision = precision
        ph = torch.tensor(phases0, dtype=torch.float64, device="cuda", requires_grad=True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        L = loss_of_field(phase_field(ph, solver), loss)
        L.backward()
        torch.cuda.synchronize()
        return float(L), ph.grad.cpu().numpy(), time.perf_counter() - t0

    L64, g64, t64 = gradient("fp64")
    L32, g32, t32 = gradient("mixed")

    def value(p):
        with torch.no_grad():
            u = phase_field(torch.tensor(p, dtype=torch.float64, device="cuda"), solver)
            return float(loss.evaluate_vector(u, False)[0])

    it.precision = "mixed"
    idx = np.random.default_rng(3).choice(m, size=min(args.fd, m), replace=False)
    fd = []
    for i in idx:
        e = np.zeros(m)
        e[i] = args.step
        fd.append((value(phases0 + e) - value(phases0 - e)) / (2 * args.step))
    fd = np.asarray(fd)
    scale = np.linalg.norm(g64)
    out = {
        "scene": f"{args.grid}^3 config-3 (16x16 array), contrast-ratio loss",
        "loss_fp64": L64, "loss_mixed": L32,
        "grad_mixed_vs_fp64_rel": float(np.linalg.norm(g32 - g64) / scale),
        "fd_indices": idx.tolist(), "fd": fd.tolist(), "adjoint_mixed": g32[idx].tolist(),
        "fd_vs_adjoint_rel": float(np.linalg.norm(g32[idx] - fd) / np.linalg.norm(fd)),
        "fd_vs_adjoint_max_abs_over_grad_scale": float(np.max(np.abs(g32[idx] - fd)) / scale * np.sqrt(m)),
        "seconds_per_gradient": {"mixed": t32, "fp64": t64},
        "adjoint_grads_per_s": {"mixed": 1.0 / t32, "fp64": 1.0 / t64},
    }
    line = json.dumps(out)
    print(line)
    if args.out:
        with open(args.out, "w") as f:
            f.write(line + "\n")


if __name__ == "__main__":
    main()
