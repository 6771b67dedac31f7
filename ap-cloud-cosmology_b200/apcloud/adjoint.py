"""Gradients through the gravity step: the trajectory vector-Jacobian product of the C ABI
(apc_trajectory_vjp) as a torch.autograd.Function, and the displacement-field loss of
the adjoint workload.

The octree, the selected cells and their particle counts are held fixed, so the cell
fields of a step are constants of the step and the Jacobian of a particle's
acceleration is its cell's Hessian.  The C ABI keeps the state every k steps and
reruns each segment in the backward pass.

    python -m apcloud.adjoint [--side 64] [--steps 32] [--every 8] [--fd 64]

runs the adjoint workload (64^3 EdS Zel'dovich box, 32 steps from a = 0.05 to 0.5,
checkpoints every 8 steps, loss = mean squared distance to a target perturbed from the
forward result by N(0, 0.01 spacing)) and checks the gradient with respect to the FP32
displacement field against central finite differences on random components
(tests/adjoint_c5_cpu_check.py adds the comparison with the FP64 CPU adjoint).
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np

from . import binding, ics


def schedule(n: int, omega0: float, omegal: float, a_start: float, a_end: float, delta_a: float,
             n_steps: int | None = None):
    """The Controller sequence (controller.cpp:88-208 with the README constants) as
    (start_dt, start_c_pos, [(dt, c_dens, c_pot, c_field, c_vel, c_pos), ...])."""
    t = a_start
    start_dt = 0.5 * delta_a
    start_c_pos = ics.drift_factor(t, omega0, omegal)
    t += start_dt
    steps = []
    while t < a_end and (n_steps is None or len(steps) < n_steps):
        dt = delta_a if t + delta_a <= a_end else a_end - t
        steps.append((dt, 1.0 / n, 1.5 * omega0 / t, -1.0, ics.kick_factor(t, omega0, omegal),
                      ics.drift_factor(t + dt / 2, omega0, omegal)))
        t += dt
    return start_dt, start_c_pos, steps


def wrap(d):
    return d - np.round(d)


def run_forward(g: binding.GpuPath, parts: ics.Particles, sched) -> np.ndarray:
    """Final (6, n) state of the trajectory from `parts` (host), on context g."""
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in parts.as_tuple()]
    g._check(g.lib.apc_set_particles(g.h, *[binding._ptr(a) for a in arrs]), "apc_set_particles")
    start_dt, start_c_pos, steps = sched
    g.select()
    g.move_position(start_dt, start_c_pos)
    for q in steps:
        g.step(*q)
    return np.stack(g.particles()[:6])


def trajectory_function():
    """torch.autograd.Function: state0 (6, n) float64 CUDA -> final state (6, n)."""
    import torch

    class Trajectory(torch.autograd.Function):
        @staticmethod
        def forward(ctx, state0, g, sched, every):
            s0 = state0.contiguous()
            out = torch.empty_like(s0)
            zero = torch.zeros_like(s0)
            start_dt, start_c_pos, steps = sched
            # forward only: a zero cotangent through the VJP entry keeps one code path
            g.trajectory_vjp(steps, start_dt, start_c_pos, every, [s0[k].data_ptr() for k in range(6)],
                             [zero[k].data_ptr() for k in range(6)], [out[k].data_ptr() for k in range(6)])
            ctx.save_for_backward(s0)
            ctx.g, ctx.sched, ctx.every = g, sched, every
            return out

        @staticmethod
        def backward(ctx, grad_out):
            (s0,) = ctx.saved_tensors
            cot = grad_out.contiguous().clone()
            start_dt, start_c_pos, steps = ctx.sched
            ctx.g.trajectory_vjp(steps, start_dt, start_c_pos, ctx.every, [s0[k].data_ptr() for k in range(6)],
                                 [cot[k].data_ptr() for k in range(6)])
            return cot, None, None, None

    return Trajectory


def loss_and_grad(g: binding.GpuPath, psi32: np.ndarray, fac: float, target: np.ndarray, sched, every: int):
    """L(psi) = mean_p |wrap(x_p - target_p)|^2 and dL/dpsi (3, n, n, n) through the GPU
    trajectory VJP; x0 = lattice + psi, v0 = fac psi."""
    import torch

    parts = ics.particles_from_field(psi32.astype(np.float64), fac)
    n = parts.n
    s0 = torch.tensor(np.stack(parts.as_tuple()), dtype=torch.float64, device="cuda")
    sf = torch.empty_like(s0)
    zero = torch.zeros_like(s0)
    start_dt, start_c_pos, steps = sched
    g.trajectory_vjp(steps, start_dt, start_c_pos, every, [s0[k].data_ptr() for k in range(6)],
                     [zero[k].data_ptr() for k in range(6)], [sf[k].data_ptr() for k in range(6)])
    d = wrap(sf[:3].cpu().numpy() - target)
    loss = float(np.mean(np.sum(d * d, axis=0)))
    cot = torch.zeros_like(s0)
    cot[:3] = torch.tensor(2.0 * d / n, device="cuda")
    g.trajectory_vjp(steps, start_dt, start_c_pos, every, [s0[k].data_ptr() for k in range(6)],
                     [cot[k].data_ptr() for k in range(6)])
    c = cot.cpu().numpy()
    side = psi32.shape[1]
    grad = (c[:3] + fac * c[3:]).reshape(3, side, side, side)
    return loss, grad, sf.cpu().numpy()


def fd_loss(g, psi64, fac, target, sched) -> float:
    x = run_forward(g, ics.particles_from_field(psi64, fac), sched)
    d = wrap(x[:3] - target)
    return float(np.mean(np.sum(d * d, axis=0)))


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--side", type=int, default=64)
    ap.add_argument("--steps", type=int, default=32)
    ap.add_argument("--every", type=int, default=8)
    ap.add_argument("--fd", type=int, default=64)
    ap.add_argument("--h", type=float, default=1e-4)
    ap.add_argument("--seed", type=int, default=5)
    ap.add_argument("--precision", choices=("fp64", "mixed"), default="mixed")
    args = ap.parse_args(argv)
    side = args.side
    a0, a1 = 0.05, 0.5
    psi, fac = ics.zeldovich_field(side, -2.0, 0.2, a0, 1.0, 0.0, seed=args.seed)
    psi32 = psi.astype(np.float32)
    n = side ** 3
    gfd_c = 1.28 * 8.0 ** (5.0 / 3.0) * side ** -2.0
    sched = schedule(n, 1.0, 0.0, a0, a1, (a1 - a0) / args.steps, args.steps)
    prec = binding.APC_PREC_MIXED if args.precision == "mixed" else binding.APC_PREC_FP64
    g = binding.GpuPath(ics.particles_from_field(psi32.astype(np.float64), fac), 21, gfd_c, precision=prec)
    rng = np.random.default_rng(args.seed + 1)
    fwd = run_forward(g, ics.particles_from_field(psi32.astype(np.float64), fac), sched)
    target = np.mod(fwd[:3] + rng.normal(0.0, 0.01 / side, size=fwd[:3].shape), 1.0)
    t0 = time.perf_counter()
    loss, grad, _ = loss_and_grad(g, psi32, fac, target, sched, args.every)
    t_vjp = time.perf_counter() - t0
    comps = [tuple(int(v) for v in (rng.integers(3), rng.integers(side), rng.integers(side), rng.integers(side)))
             for _ in range(args.fd)]
    fd, ad = [], []
    for c in comps:
        p = psi32.astype(np.float64)
        p[c] += args.h
        lp = fd_loss(g, p, fac, target, sched)
        p[c] -= 2 * args.h
        lm = fd_loss(g, p, fac, target, sched)
        fd.append((lp - lm) / (2 * args.h))
        ad.append(float(grad[c]))
    fd, ad = np.array(fd), np.array(ad)
    scale = float(np.max(np.abs(ad)))
    err = np.abs(fd - ad) / max(scale, 1e-300)
    # A component whose +-h step moves a particle into another cell at some step changes
    # a cell count, so the loss jumps there; such components are redone with h / 100.
    redo = []
    for j in np.nonzero(err >= 1e-3)[0]:
        c, h2 = comps[j], args.h / 100
        p = psi32.astype(np.float64)
        p[c] += h2
        lp = fd_loss(g, p, fac, target, sched)
        p[c] -= 2 * h2
        lm = fd_loss(g, p, fac, target, sched)
        e2 = abs((lp - lm) / (2 * h2) - ad[j]) / max(scale, 1e-300)
        redo.append({"component": list(c), "err_h": float(err[j]), "err_h_over_100": float(e2)})
    out = {"side": side, "steps": len(sched[2]), "checkpoint_every": args.every, "precision": args.precision,
           "loss": loss, "vjp_seconds": t_vjp, "fd_h": args.h, "fd_components": args.fd,
           "fd_max_err_rel_to_max_grad": float(err.max()), "fd_median_err_rel_to_max_grad": float(np.median(err)),
           "fd_within_1e-3": int(np.sum(err < 1e-3)), "fd_redone_with_h_over_100": redo,
           "grad_norm": float(np.linalg.norm(grad))}
    g.close()
    print(json.dumps(out))
    return out, grad, (psi32, fac, gfd_c, sched, target)


if __name__ == "__main__":
    main()
