"""Failure detection without a GPU fault.

The solver's persistent kernels wait on one another at a grid barrier whose spin is
bounded: a block that waits too long raises an error flag and an abort flag, every block
leaves, and the host maps the flag to APC_ERR_TIMEOUT.  apc_check_bounded_wait runs that
barrier with a block that never arrives (a flag nothing sets), so the wait must run out;
the test then checks the status and that the device still runs a full step.  Nothing
here traps, faults or hangs the GPU."""
from __future__ import annotations

import numpy as np
import pytest

from apcloud import binding, ics

APC_ERR_INVALID_ARG = -1
APC_ERR_TIMEOUT = -10


def test_bounded_wait_rejects_bad_limits_before_touching_a_device(gpu_lib):
    lib = binding.load_library(gpu_lib)
    assert lib.apc_check_bounded_wait(0, 0) == APC_ERR_INVALID_ARG
    assert lib.apc_check_bounded_wait(0, (1 << 24) + 1) == APC_ERR_INVALID_ARG


@pytest.mark.gpu
def test_bounded_wait_runs_out_and_the_device_stays_usable(gpu_lib):
    import refbind

    lib = binding.load_library(gpu_lib)
    for _ in range(2):  # ~1-2 ms waits that nothing releases
        assert lib.apc_check_bounded_wait(0, 1 << 14) == APC_ERR_TIMEOUT
    cfg = ics.config("ball32k", n=3000, seed=5)
    p = cfg.particles()
    gp = binding.GpuPath(p, cfg.depth, cfg.gfd_c)
    o = refbind.CpuPath("oracle", p, cfg.depth, cfg.gfd_c)
    o.set_gmres(30, 1e-10)
    assert gp.select() == o.select()
    t = cfg.a_start + 0.5 * cfg.delta_a
    gp.solve(1.0 / p.n, 1.5 / t, -1.0)
    o.solve(1.0 / p.n, 1.5 / t, -1.0)
    a, b = gp.fields().potential, o.fields().potential
    assert np.max(np.abs(a - b)) <= 1e-10 * np.max(np.abs(b))
    gp.close()
    o.close()
