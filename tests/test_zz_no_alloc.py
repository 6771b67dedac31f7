"""GPU test of apc_move_velocity_noalloc, the interpolation + kick entry point for callers
that cannot allocate device memory (their framework owns all device memory, or they
cannot take cudaMalloc's device-wide synchronisation).  It must give what
apc_move_velocity gives on the same state, call after call, while taking its scratch
from the library's fixed array.  Collected last so that a run stopping at the first
failure has already run every other test."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from apcloud import binding, ics

pytestmark = pytest.mark.gpu

RTOL = 1e-12  # the two entry points share arithmetic and rounding; equality is expected
NOALLOC_MAX_PARTICLES = 1 << 20  # APC_NOALLOC_MAX_PARTICLES
APC_ERR_INVALID_ARG = -1


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def test_noalloc_kick_matches_move_velocity_on_two_calls(gpu_lib):
    import torch

    cfg = ics.config("ball32k", n=5000, seed=21)
    p = cfg.particles()
    t = cfg.a_start + 0.5 * cfg.delta_a
    dt, cv = cfg.delta_a, ics.kick_factor(t, cfg.omega0, cfg.omegal)
    gp = binding.GpuPath(p, cfg.depth, cfg.gfd_c)
    gp.select()
    gp.solve(1.0 / p.n, 1.5 * cfg.omega0 / t, -1.0)
    cells = gp.cells()
    fields = gp.fields()
    _, order = gp.keys()  # caller index of each particle in cell (Morton) order
    state0 = gp.particles()

    # reference answer: the context's entry point, twice in a row
    dv_ref, states = [], []
    for _ in range(2):
        dv_ref.append(gp.move_velocity(dt, cv))
        states.append(gp.particles())
    gp.close()

    dev = torch.device("cuda", 0)

    def on_dev(a, dtype=torch.float64):
        return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype).to(dev)

    first = on_dev(cells.first, torch.int32)
    count = on_dev(cells.count, torch.int32)
    cx, cy, cz = on_dev(cells.x), on_dev(cells.y), on_dev(cells.z)
    deriv = on_dev(fields.deriv.reshape(-1))
    x, y, z = (on_dev(a[order]) for a in state0[:3])
    v = [on_dev(a[order]) for a in state0[3:6]]
    acc = [torch.zeros(p.n, dtype=torch.float64, device=dev) for _ in range(3)]
    lib = binding.load_library()

    def call(n):
        d = C.c_double()
        rc = lib.apc_move_velocity_noalloc(
            n, cells.m, first.data_ptr(), count.data_ptr(), cx.data_ptr(), cy.data_ptr(), cz.data_ptr(),
            deriv.data_ptr(), x.data_ptr(), y.data_ptr(), z.data_ptr(), v[0].data_ptr(), v[1].data_ptr(),
            v[2].data_ptr(), acc[0].data_ptr(), acc[1].data_ptr(), acc[2].data_ptr(), dt, cv, C.byref(d), None)
        torch.cuda.synchronize()
        return rc, d.value

    for k in range(2):
        free_before = torch.cuda.mem_get_info(0)[0]
        held_before = torch.cuda.memory_allocated(0)
        rc, dv = call(p.n)
        assert rc == 0
        if k == 1:
            # the first call loaded the library's module (and with it the fixed scratch
            # array); from then on a call leaves the device's free memory unchanged
            assert torch.cuda.mem_get_info(0)[0] == free_before
        assert torch.cuda.memory_allocated(0) == held_before
        assert dv == pytest.approx(dv_ref[k], rel=RTOL)
        for j in range(3):
            assert _rel(v[j].cpu().numpy(), states[k][3 + j][order]) <= RTOL
            assert _rel(acc[j].cpu().numpy(), states[k][6 + j][order]) <= RTOL

    # cell ranges that leave particles uncovered, overlap, or run past the particle count
    # are refused, and the velocities and accelerations are left as they were
    before = [t.clone() for t in v + acc]
    good_first, good_count = first.clone(), count.clone()
    last = int(np.nonzero(cells.count)[0][-1])
    for case, (df, dc) in {"uncovered": (0, -1), "overlap or past the end": (0, 1),
                           "outside [0, n)": (p.n, 0)}.items():
        first.copy_(good_first)
        count.copy_(good_count)
        first[last] += df
        count[last] += dc
        rc, _ = call(p.n)
        assert rc == APC_ERR_INVALID_ARG, case
        for t0, t1 in zip(before, v + acc):
            assert torch.equal(t0, t1), case
    first.copy_(good_first)
    count.copy_(good_count)
    rc, _ = call(p.n)
    assert rc == 0

    # sizes beyond the fixed scratch array are refused before any work is queued
    rc, _ = call(NOALLOC_MAX_PARTICLES + 1)
    assert rc == APC_ERR_INVALID_ARG
