"""Adjoint of the step sequence: the FP64 CPU adjoint (oracle) against central finite
differences, and on a GPU the trajectory VJP of the C ABI against the CPU adjoint and
against finite differences of the mixed path."""
from __future__ import annotations

import numpy as np
import pytest

from apcloud import ics
from apcloud.adjoint import schedule, wrap


def _case(side=12, steps=4, seed=3):
    a0, a1 = 0.05, 0.5
    psi, fac = ics.zeldovich_field(side, -2.0, 0.2, a0, 1.0, 0.0, seed=seed)
    gfd_c = 1.28 * 8.0 ** (5.0 / 3.0) * side ** -2.0
    sched = schedule(side ** 3, 1.0, 0.0, a0, a1, (a1 - a0) / steps, steps)
    return psi, fac, gfd_c, sched


def _loss_cpu(psi, fac, gfd_c, sched, target):
    import adjoint_ref

    x, _ = adjoint_ref.forward_state(ics.particles_from_field(psi, fac), 21, gfd_c, sched)
    d = wrap(x[:3] - target)
    return float(np.mean(np.sum(d * d, axis=0)))


def test_cpu_adjoint_matches_finite_differences(oracle_lib):
    import adjoint_ref

    psi, fac, gfd_c, sched = _case()
    side = psi.shape[1]
    n = side ** 3
    rng = np.random.default_rng(0)
    x, _ = adjoint_ref.forward_state(ics.particles_from_field(psi, fac), 21, gfd_c, sched)
    target = np.mod(x[:3] + rng.normal(0.0, 0.01 / side, size=x[:3].shape), 1.0)
    d = wrap(x[:3] - target)
    cot = np.zeros((6, n))
    cot[:3] = 2.0 * d / n
    _, c0 = adjoint_ref.trajectory_vjp(ics.particles_from_field(psi, fac), 21, gfd_c, sched, cot)
    grad = (c0[:3] + fac * c0[3:]).reshape(psi.shape)
    h = 1e-7
    errs = []
    for _ in range(6):
        c = (int(rng.integers(3)),) + tuple(int(v) for v in rng.integers(side, size=3))
        p = psi.copy()
        p[c] += h
        lp = _loss_cpu(p, fac, gfd_c, sched, target)
        p[c] -= 2 * h
        lm = _loss_cpu(p, fac, gfd_c, sched, target)
        errs.append(abs((lp - lm) / (2 * h) - grad[c]) / np.abs(grad).max())
    # a component whose particle changes cell within h would jump; allow one
    assert sorted(errs)[-2] < 1e-5, errs


@pytest.mark.gpu
def test_gpu_trajectory_vjp_matches_cpu_adjoint(oracle_lib):
    import torch

    import adjoint_ref
    from apcloud import binding

    psi, fac, gfd_c, sched = _case(side=12, steps=4)
    n = psi.shape[1] ** 3
    parts = ics.particles_from_field(psi, fac)
    rng = np.random.default_rng(1)
    cot = rng.standard_normal((6, n))
    xf_ref, c0_ref = adjoint_ref.trajectory_vjp(parts, 21, gfd_c, sched, cot)
    g = binding.GpuPath(parts, 21, gfd_c, precision=binding.APC_PREC_FP64)
    s0 = torch.tensor(np.stack(parts.as_tuple()), dtype=torch.float64, device="cuda")
    ct = torch.tensor(cot, dtype=torch.float64, device="cuda")
    sf = torch.empty_like(s0)
    start_dt, start_c_pos, steps = sched
    g.trajectory_vjp(steps, start_dt, start_c_pos, 2, [s0[k].data_ptr() for k in range(6)],
                     [ct[k].data_ptr() for k in range(6)], [sf[k].data_ptr() for k in range(6)])
    g.close()
    assert np.abs(wrap(sf.cpu().numpy()[:3] - xf_ref[:3])).max() < 1e-10
    c0 = ct.cpu().numpy()
    assert np.abs(c0 - c0_ref).max() / np.abs(c0_ref).max() < 1e-7


@pytest.mark.gpu
def test_gpu_vjp_finite_differences_mixed():
    from apcloud import binding
    from apcloud.adjoint import fd_loss, loss_and_grad, run_forward

    psi, fac, gfd_c, sched = _case(side=16, steps=6, seed=4)
    side = psi.shape[1]
    psi32 = psi.astype(np.float32)
    g = binding.GpuPath(ics.particles_from_field(psi32.astype(np.float64), fac), 21, gfd_c,
                        precision=binding.APC_PREC_MIXED)
    rng = np.random.default_rng(2)
    x = run_forward(g, ics.particles_from_field(psi32.astype(np.float64), fac), sched)
    target = np.mod(x[:3] + rng.normal(0.0, 0.01 / side, size=x[:3].shape), 1.0)
    _, grad, _ = loss_and_grad(g, psi32, fac, target, sched, every=3)
    h = 1e-6
    errs = []
    for _ in range(8):
        c = (int(rng.integers(3)),) + tuple(int(v) for v in rng.integers(side, size=3))
        p = psi32.astype(np.float64)
        p[c] += h
        lp = fd_loss(g, p, fac, target, sched)
        p[c] -= 2 * h
        lm = fd_loss(g, p, fac, target, sched)
        errs.append(abs((lp - lm) / (2 * h) - grad[c]) / np.abs(grad).max())
    g.close()
    assert sorted(errs)[-2] < 1e-4, errs


@pytest.mark.gpu
def test_solve_vjp_dot_product():
    """<g, J d> = <J^T g, d> for the linear map density rhs -> field derivatives, with J d
    from two re-solves and J^T g from apc_solve_vjp (transposed stencil, GMRES on A2^T
    and A1^T)."""
    import torch

    from apcloud import binding

    psi, fac, gfd_c, sched = _case(side=12, steps=1)
    parts = ics.particles_from_field(psi, fac)
    g = binding.GpuPath(parts, 21, gfd_c, precision=binding.APC_PREC_FP64, rtol=1e-13)
    _, _, steps = sched
    dt, c_dens, c_pot, c_field, c_vel, c_pos = steps[0]
    g.select()
    g.solve(c_dens, c_pot, c_field)
    nc, nv, _, _ = g.counts()
    m = nc + nv
    cells = g.cells()
    rhs0 = cells.count[:m] / cells.h[:m] ** 3 * c_dens
    rng = np.random.default_rng(9)
    d = rng.standard_normal(m) * np.abs(rhs0).mean()
    gbar = rng.standard_normal((m, 9))
    out = []
    for sign in (1.0, -1.0):
        r = torch.tensor(rhs0 + sign * d, dtype=torch.float64, device="cuda")
        g.fields_from_rhs(r.data_ptr())
        out.append(g.fields().deriv.copy())
    jd = 0.5 * (out[0] - out[1])
    gb = torch.tensor(gbar, dtype=torch.float64, device="cuda")
    gr = torch.empty(m, dtype=torch.float64, device="cuda")
    g.solve_vjp(gb.data_ptr(), gr.data_ptr())
    st = g.solve_stats()
    g.close()
    lhs = float(np.sum(gbar * jd))
    rhs = float(np.dot(gr.cpu().numpy(), d))
    assert st["adjoint_potential_reason"] > 0 and st["adjoint_density_reason"] > 0, st
    assert abs(lhs - rhs) <= 1e-7 * abs(lhs), (lhs, rhs)
