"""FP64 CPU adjoint of the step sequence, on the oracle (test infrastructure).

The forward trajectory runs through the oracle's restatement of the reference
(refbind.CpuPath): select, solve, kick, drift per step, with the initial half drift.
After each kick the per-particle Hessians are read from the oracle's cells: the
particle at sorted position j lies in the cell whose particle range holds j
(octree.cpp:3003-3031), and its Hessian is that cell's p_xx..p_yz.  The reverse pass
applies, per step from the last,
    lv <- lv + c_pos dt lx,   lx <- lx + c_vel dt H lv,
then lv <- lv + c_pos(start) dt/2 lx for the half drift.  Everything is in caller order
and FP64.
"""
from __future__ import annotations

import numpy as np

import refbind


def _hessians(r) -> np.ndarray:
    """(6, n) Hessians (xx, yy, zz, xy, xz, yz) of each particle's cell, caller order."""
    _, idx = r.keys()
    cells = r.cells()
    der = r.fields().deriv
    m = der.shape[0]
    cell_of = np.full(idx.shape[0], -1, np.int64)
    for i in range(m):
        f, c = int(cells.first[i]), int(cells.count[i])
        if c > 0:
            cell_of[f:f + c] = i
    assert (cell_of >= 0).all()
    h = np.empty((6, idx.shape[0]))
    h[:, idx] = der[cell_of, 3:9].T
    return h


def _run(parts, depth, gfd_c, sched, tape: list | None):
    r = refbind.CpuPath("oracle", parts, depth, gfd_c)
    r.set_gmres(30, 1e-10, 1e-50, 1e5, 10000)
    start_dt, start_c_pos, steps = sched
    r.select()
    r.move_position(start_dt, start_c_pos)
    for dt, c_dens, c_pot, c_field, c_vel, c_pos in steps:
        r.select()
        r.solve(c_dens, c_pot, c_field)
        r.move_velocity(dt, c_vel)
        if tape is not None:
            tape.append(_hessians(r))
        r.move_position(dt, c_pos)
    state = np.stack(r.particles()[:6])
    r.close()
    return state


def forward_state(parts, depth, gfd_c, sched):
    return _run(parts, depth, gfd_c, sched, None), None


def trajectory_vjp(parts, depth, gfd_c, sched, cot):
    """(final state (6, n), cotangent of the initial state) for the cotangent `cot` (6, n)
    of the final state."""
    tape = []
    state = _run(parts, depth, gfd_c, sched, tape)
    lx, lv = cot[:3].copy(), cot[3:].copy()
    start_dt, start_c_pos, steps = sched
    for (dt, _, _, _, c_vel, c_pos), h in zip(reversed(steps), reversed(tape)):
        lv = lv + (c_pos * dt) * lx
        hxx, hyy, hzz, hxy, hxz, hyz = h
        lx = lx + (c_vel * dt) * np.stack([hxx * lv[0] + hxy * lv[1] + hxz * lv[2],
                                           hxy * lv[0] + hyy * lv[1] + hyz * lv[2],
                                           hxz * lv[0] + hyz * lv[1] + hzz * lv[2]])
    lv = lv + (start_c_pos * start_dt) * lx
    return state, np.concatenate([lx, lv])
