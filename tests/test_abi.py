"""CPU tests of the C ABI boundary: the library loads, exports every entry point that
include/apcloud_gpu.h declares, and rejects invalid arguments before touching a device."""
from __future__ import annotations

import ctypes as C
import os
import re
import subprocess

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "apcloud_gpu.h")


def declared_functions() -> list[str]:
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(apc_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_phase_entry_points():
    names = declared_functions()
    for n in ("apc_create", "apc_destroy", "apc_set_particles", "apc_select", "apc_solve",
              "apc_move_velocity", "apc_move_position", "apc_get_cells", "apc_get_fields", "apc_step"):
        assert n in names


def test_library_exports_every_declared_symbol(gpu_lib):
    out = subprocess.run(["nm", "-D", "--defined-only", gpu_lib], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (apc_[a-z0-9_]+)\b", out))
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing


def test_binding_covers_every_declared_symbol():
    from apcloud import binding

    assert sorted(binding.EXPORTED) == declared_functions()


def test_library_loads_and_rejects_invalid_config(gpu_lib):
    from apcloud import binding

    lib = binding.load_library(gpu_lib)
    assert lib.apc_status_string(0) == b"ok"
    assert lib.apc_status_string(-5) == b"temp-node budget exceeded"
    cfg = binding.ApcConfig()
    lib.apc_config_default(C.byref(cfg))
    assert (cfg.depth, cfg.lm, cfg.gmres_restart, cfg.maxnc) == (21, 17, 30, 10000)
    assert cfg.gmres_rtol == pytest.approx(1e-10)
    assert cfg.mixed_precond == binding.APC_PRECOND_MULTIGRID
    h = C.c_void_p()
    assert lib.apc_create(None, C.byref(h)) == -1
    for field, bad in (("n_particles", 0), ("depth", 22), ("depth", 0), ("lm", 8), ("lm", 33),
                       ("gmres_restart", 0), ("gmres_restart", 256), ("mixed_restart", 32), ("precision", 7), ("bc", 2)):
        c2 = binding.ApcConfig()
        lib.apc_config_default(C.byref(c2))
        c2.n_particles = 100
        setattr(c2, field, bad)
        assert lib.apc_create(C.byref(c2), C.byref(h)) == -1, field
    c3 = binding.ApcConfig()
    lib.apc_config_default(C.byref(c3))
    c3.n_particles = 100
    c3.box[1] = c3.box[0]  # empty box
    assert lib.apc_create(C.byref(c3), C.byref(h)) == -1
    # phase calls on a null context fail cleanly
    assert lib.apc_select(None, None) == -1
    assert lib.apc_destroy(None) == -1
    assert lib.apc_kernel_launches(None) == 0


def test_build_targets_sm100a_only():
    """The library's nvcc flags name sm_100a and nothing else; the device code the runtime
    actually loads is checked on a B200 by test_device_code_is_sm100."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("apc_build", os.path.join(ROOT, "ap-cloud-cosmology_b200",
                                                                         "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    arch = [f for f in mod.NVCC_FLAGS if "arch=" in f]
    assert arch == ["arch=compute_100a,code=sm_100a"]


@pytest.mark.gpu
def test_device_code_is_sm100(gpu_lib):
    """cudaFuncGetAttributes on a library kernel, as loaded on the device: sm_100."""
    from apcloud import binding

    lib = binding.load_library(gpu_lib)
    bv, pv = C.c_int(), C.c_int()
    assert lib.apc_device_code_version(0, C.byref(bv), C.byref(pv)) == 0
    assert bv.value == 100, (bv.value, pv.value)


def test_petsc_ksp_options(gpu_lib):
    """The reference's run-line options (Makefile:30-32) map onto the GMRES settings."""
    from apcloud import binding

    lib = binding.load_library(gpu_lib)
    cfg = binding.ApcConfig()
    lib.apc_config_default(C.byref(cfg))

    def apply(*args):
        arr = (C.c_char_p * len(args))(*[a.encode() for a in args])
        return lib.apc_config_from_options(C.byref(cfg), len(args), arr)

    assert apply("./run", "parameter.param", "-ksp_gmres_restart", "20", "-ksp_max_it", "1000",
                 "-ksp_atol", "1.e-60", "-ksp_rtol", "1e-8", "-ksp_monitor") == 0
    assert (cfg.gmres_restart, cfg.gmres_max_it) == (20, 1000)
    assert cfg.gmres_atol == pytest.approx(1e-60) and cfg.gmres_rtol == pytest.approx(1e-8)
    # the reference's production run line (restart 200) is accepted; above 255 is not
    assert apply("-ksp_gmres_restart", "200") == 0 and cfg.gmres_restart == 200
    assert apply("-ksp_gmres_restart", "256") == -9  # APC_ERR_UNSUPPORTED
    assert cfg.gmres_restart == 200
    assert apply("-ksp_max_it", "abc") == -1
