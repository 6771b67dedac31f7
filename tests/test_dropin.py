"""The drop-in at the reference's own interfaces: the reference's Controller::solve
(controller.cpp:54-241, compiled unchanged from the reference sources) driving Mover and
Solver whose bodies run on libapcloud_gpu.so (ap-cloud-cosmology_b200/dropin), against the
same controller.cpp over the reference's own Mover / Solver / Octree (oracle/_ref's CPU
twin).  Both are built here from the reference sources (make -C ap-cloud-cosmology_b200/
dropin; make -C oracle dropin) and travel with the tree as built libraries.

The run is the 32,768-particle cold ball (C1) with the reference's macros as shipped:
adaptive time step on (apcloud_macro.h), COSMOLOGY_UNIT off (unit constants, potential
constant 1000), GMRES(30) rtol 1e-10 from the -ksp_* command line; the end time is set
for five steps."""
from __future__ import annotations

import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ORACLE, PKG

from apcloud import binding, ics

GPU_SO = os.path.join(PKG, "dropin", "_build", "libapcdrop_gpu.so")
CPU_SO = os.path.join(ORACLE, "_ref", "libapcdrop_ref.so")
HEADER = os.path.join(os.path.dirname(PKG), "include", "apcloud_gpu.h")


def _load(path):
    if not os.path.exists(path):
        pytest.skip(f"{os.path.relpath(path)} not built (needs the reference sources)")
    lib = C.CDLL(path)
    lib.apc_dropin_run.restype = C.c_int
    lib.apc_dropin_run.argtypes = ([C.c_int] + [C.c_void_p] * 9 + [C.c_double] * 3 +
                                   [C.c_int, C.c_double, C.c_int, C.c_void_p, C.c_int, C.c_double, C.c_int])
    return lib


def _run(lib, cfg, parts, end_a):
    arr = [np.ascontiguousarray(a, dtype=np.float64).copy() for a in parts.as_tuple()] + \
          [np.zeros(parts.n) for _ in range(3)]
    box = np.array([0.0, 1.0, 0.0, 1.0, 0.0, 1.0])
    rc = lib.apc_dropin_run(parts.n, *[a.ctypes.data for a in arr], cfg.a_start, end_a, cfg.delta_a, cfg.depth,
                            cfg.gfd_c, cfg.lm, box.ctypes.data, cfg.restart, cfg.rtol, 10000)
    assert rc == 0
    return arr


def test_gpu_dropin_calls_only_the_c_abi(gpu_lib):
    """The GPU build of Mover / Solver / Controller needs nothing from PETSc, MPI or LAPACK:
    every symbol it leaves to other libraries, apart from the C / C++ / OpenMP runtimes,
    is an entry point of include/apcloud_gpu.h."""
    if not os.path.exists(GPU_SO):
        pytest.skip("drop-in not built (needs the reference sources)")
    out = subprocess.run(["nm", "-D", "--undefined-only", GPU_SO], capture_output=True, text=True,
                         check=True).stdout
    names = [ln.split()[-1] for ln in out.splitlines() if ln.strip().startswith("U ")]
    # symbols of the system runtimes carry their version (GLIBC_, GLIBCXX_, CXXABI_, GCC_, OMP_ ...)
    foreign = [n for n in names if "@" not in n and not n.startswith("apc_")]
    assert not foreign, foreign
    assert not [n for n in names if re.search(r"(?i)petsc|mpi_|lapack|dgels|ksp", n)]
    api = set(re.findall(r"\b(apc_[a-z0-9_]+)\s*\(", re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)))
    called = {n.split("@")[0] for n in names if n.startswith("apc_")}
    assert called and called <= api, called - api


@pytest.mark.gpu
def test_reference_controller_over_gpu_mover_and_solver(gpu_lib, reference_lib):
    import refbind

    binding.load_library(gpu_lib)  # the drop-in resolves the C ABI from the loaded library
    gpu, cpu = _load(GPU_SO), _load(CPU_SO)
    gpu.apc_dropin_set_precision.argtypes = [C.c_int]
    gpu.apc_dropin_kicks.restype = C.c_long
    cfg = ics.config("ball32k")
    parts = cfg.particles()
    # the reference's adaptive step at the start (controller.cpp:146-164), for the end time
    r = refbind.CpuPath("ref", parts, cfg.depth, cfg.gfd_c)
    r.select()
    dt0 = r.adaptive_dt(cfg.delta_a)
    r.close()
    end_a = cfg.a_start + 0.5 * cfg.delta_a + 4.5 * dt0
    gpu.apc_dropin_set_precision(binding.APC_PREC_FP64)
    gpu.apc_dropin_reset_kicks()
    g = _run(gpu, cfg, parts, end_a)
    assert gpu.apc_dropin_kicks() == 5
    c = _run(cpu, cfg, parts, end_a)
    d = np.stack(g[:3]) - np.stack(c[:3])
    d -= np.round(d)
    pos = float(np.max(np.abs(d)))

    def rms(a, b):
        a, b = np.stack(a), np.stack(b)
        return float(np.sqrt(np.mean(np.sum((a - b) ** 2, 0)) / np.mean(np.sum(b ** 2, 0))))

    vel, acc = rms(g[3:6], c[3:6]), rms(g[6:9], c[6:9])
    print("drop-in vs reference: max position difference", pos, "velocity rms", vel, "acceleration rms", acc)
    # FP64 GMRES to rtol 1e-10 on both sides; the fields of two such solutions differ by
    # up to cond(A) 1e-10 (about 1e-9 here), five kicks carry that into the velocities
    assert pos <= 1e-10
    assert vel <= 1e-7 and acc <= 1e-7
    # the mixed path through the same drop-in stays within the force-error bound
    gpu.apc_dropin_set_precision(binding.APC_PREC_MIXED)
    m = _run(gpu, cfg, parts, end_a)
    assert rms(m[6:9], c[6:9]) <= 1e-6
