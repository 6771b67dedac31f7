"""ctypes binding of libapcloud_gpu.so (include/apcloud_gpu.h).

The GPU path has no fallback: if the library or a CUDA device is missing, construction
raises.  ``GpuPath`` exposes the phase calls of the reference's Mover / Solver
(mover.h:31-43, solver.h:53-62) with host numpy arrays.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "libapcloud_gpu.so")

APC_PREC_FP64 = 0
APC_PREC_MIXED = 1
APC_PREC_FP64_MULTIGRID = 2
APC_PREC_MIXED_VCYCLE = 3
APC_PRECOND_JACOBI = 0
APC_PRECOND_MULTIGRID = 1
APC_BATCH_SOLVE_PER_BOX = 0
APC_BATCH_SOLVE_QUEUED = 1

EXPORTED = [
    "apc_config_default", "apc_status_string", "apc_last_error", "apc_create", "apc_destroy",
    "apc_set_particles", "apc_get_particles", "apc_set_particles_device", "apc_get_particles_device",
    "apc_select", "apc_solve", "apc_move_velocity", "apc_move_position", "apc_step", "apc_synchronize",
    "apc_get_cell_counts", "apc_get_cells", "apc_get_cell_codes", "apc_get_keys", "apc_get_octree_levels",
    "apc_get_fields", "apc_get_stencils", "apc_get_solve_stats", "apc_get_matrix", "apc_kernel_launches",
    "apc_get_phase_times", "apc_get_profile", "apc_reset_profile", "apc_move_velocity_noalloc",
    "apc_batch_create", "apc_batch_destroy", "apc_batch_size", "apc_batch_context", "apc_batch_step",
    "apc_get_hessians_device", "apc_vjp_kick_drift", "apc_trajectory_vjp", "apc_fields_from_rhs",
    "apc_solve_vjp", "apc_max_cell_density", "apc_adaptive_dt", "apc_config_from_options",
    "apc_device_code_version", "apc_check_bounded_wait", "apc_batch_set_solve_mode", "apc_batch_solve_ms",
]


class ApcConfig(C.Structure):
    _fields_ = [
        ("n_particles", C.c_int), ("depth", C.c_int), ("bc", C.c_int), ("box", C.c_double * 6),
        ("gfd_c", C.c_double), ("lm", C.c_int), ("maxnc", C.c_int), ("nmax_cap", C.c_int),
        ("gmres_restart", C.c_int), ("gmres_rtol", C.c_double), ("gmres_atol", C.c_double),
        ("gmres_dtol", C.c_double), ("gmres_max_it", C.c_int), ("precision", C.c_int),
        ("mixed_restart", C.c_int), ("mixed_inner_rtol", C.c_double), ("device", C.c_int),
        ("mixed_precond", C.c_int), ("mg_sweeps", C.c_int), ("mg_omega", C.c_double), ("mg_alpha", C.c_double),
        ("mg_reorth", C.c_int), ("warm_start", C.c_int), ("mixed_solve_graphs", C.c_int),
    ]


class ApcSolveStats(C.Structure):
    _fields_ = [
        ("density_its", C.c_int), ("potential_its", C.c_int),
        ("density_reason", C.c_int), ("potential_reason", C.c_int),
        ("density_rnorm", C.c_double), ("potential_rnorm", C.c_double),
        ("density_refinements", C.c_int), ("potential_refinements", C.c_int), ("mg_levels", C.c_int),
        ("adjoint_density_its", C.c_int), ("adjoint_potential_its", C.c_int),
        ("adjoint_density_reason", C.c_int), ("adjoint_potential_reason", C.c_int),
    ]


class ApcProfile(C.Structure):
    _fields_ = [("krylov_launches", C.c_int64), ("krylov_iterations", C.c_int64), ("krylov_ms", C.c_double),
                ("krylov_bytes", C.c_double), ("select_ms", C.c_double), ("solve_ms", C.c_double),
                ("move_ms", C.c_double), ("steps", C.c_int64), ("step_ms", C.c_double),
                ("gfd_ms", C.c_double), ("mg_build_ms", C.c_double), ("mg_solve_ms", C.c_double),
                ("mg_iterations", C.c_int64), ("assemble_ms", C.c_double), ("density_ms", C.c_double),
                ("potential_ms", C.c_double), ("graph_instantiations", C.c_int64), ("graph_updates", C.c_int64),
                ("sort_retries", C.c_int64), ("mg_bytes", C.c_double)]


class ApcStepParams(C.Structure):
    _fields_ = [("dt", C.c_double), ("c_dens", C.c_double), ("c_pot", C.c_double),
                ("c_field", C.c_double), ("c_vel", C.c_double), ("c_pos", C.c_double)]


class ApcTrajectory(C.Structure):
    _fields_ = [("n_steps", C.c_int), ("steps", C.POINTER(ApcStepParams)), ("start_dt", C.c_double),
                ("start_c_pos", C.c_double), ("checkpoint_every", C.c_int)]


class ApcError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str):
        super().__init__(f"{where}: status {status} ({msg})")
        self.status = status


_lib = None


def load_library(path: str = LIB_PATH):
    """Load the CUDA library; raises if it is missing (no CPU fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is missing: build it with ap-cloud-cosmology_b200/build.py")
    lib = C.CDLL(path)
    vp, ip, dp, u64p = C.c_void_p, C.POINTER(C.c_int), C.c_void_p, C.c_void_p
    sig = {
        "apc_config_default": (None, [C.POINTER(ApcConfig)]),
        "apc_status_string": (C.c_char_p, [C.c_int]),
        "apc_last_error": (C.c_char_p, [vp]),
        "apc_create": (C.c_int, [C.POINTER(ApcConfig), C.POINTER(C.c_void_p)]),
        "apc_destroy": (C.c_int, [vp]),
        "apc_set_particles": (C.c_int, [vp] + [dp] * 6),
        "apc_get_particles": (C.c_int, [vp] + [dp] * 9),
        "apc_set_particles_device": (C.c_int, [vp] + [dp] * 6),
        "apc_get_particles_device": (C.c_int, [vp] + [dp] * 6),
        "apc_select": (C.c_int, [vp, ip]),
        "apc_solve": (C.c_int, [vp, C.c_double, C.c_double, C.c_double]),
        "apc_move_velocity": (C.c_int, [vp, C.c_double, C.c_double, C.POINTER(C.c_double)]),
        "apc_move_position": (C.c_int, [vp, C.c_double, C.c_double, C.POINTER(C.c_double)]),
        "apc_step": (C.c_int, [vp, C.POINTER(ApcStepParams), ip, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
        "apc_synchronize": (C.c_int, [vp]),
        "apc_get_cell_counts": (C.c_int, [vp, ip, ip, ip, ip]),
        "apc_get_cells": (C.c_int, [vp] + [dp] * 4 + [vp] * 6),
        "apc_get_cell_codes": (C.c_int, [vp, u64p]),
        "apc_get_keys": (C.c_int, [vp, u64p, vp]),
        "apc_get_octree_levels": (C.c_int, [vp, vp]),
        "apc_get_fields": (C.c_int, [vp, dp, dp, dp]),
        "apc_get_stencils": (C.c_int, [vp, vp, dp]),
        "apc_get_solve_stats": (C.c_int, [vp, C.POINTER(ApcSolveStats)]),
        "apc_get_matrix": (C.c_int, [vp, C.c_int, ip, ip, vp, vp, vp]),
        "apc_kernel_launches": (C.c_int64, [vp]),
        "apc_get_phase_times": (C.c_int, [vp, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]),
        "apc_get_profile": (C.c_int, [vp, C.POINTER(ApcProfile)]),
        "apc_reset_profile": (C.c_int, [vp]),
        "apc_move_velocity_noalloc": (C.c_int, [C.c_int, C.c_int] + [vp] * 15 + [C.c_double, C.c_double,
                                                                                  C.POINTER(C.c_double), vp]),
        "apc_batch_create": (C.c_int, [C.POINTER(ApcConfig), C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
        "apc_batch_destroy": (C.c_int, [vp]),
        "apc_batch_size": (C.c_int, [vp]),
        "apc_batch_context": (C.c_void_p, [vp, C.c_int]),
        "apc_batch_step": (C.c_int, [vp, C.POINTER(ApcStepParams), ip, vp, vp]),
        "apc_get_hessians_device": (C.c_int, [vp] + [vp] * 6),
        "apc_fields_from_rhs": (C.c_int, [vp, vp]),
        "apc_max_cell_density": (C.c_int, [vp, C.POINTER(C.c_double)]),
        "apc_config_from_options": (C.c_int, [C.POINTER(ApcConfig), C.c_int, C.POINTER(C.c_char_p)]),
        "apc_adaptive_dt": (C.c_int, [vp, C.c_double, C.POINTER(C.c_double)]),
        "apc_solve_vjp": (C.c_int, [vp, vp, vp, vp, vp]),
        "apc_vjp_kick_drift": (C.c_int, [C.c_int, C.POINTER(C.c_void_p), C.c_double, C.c_double,
                                         C.POINTER(C.c_void_p), vp]),
        "apc_trajectory_vjp": (C.c_int, [vp, C.POINTER(ApcTrajectory), C.POINTER(C.c_void_p),
                                         C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]),
        "apc_device_code_version": (C.c_int, [C.c_int, ip, ip]),
        "apc_check_bounded_wait": (C.c_int, [C.c_int, C.c_int]),
        "apc_batch_set_solve_mode": (C.c_int, [vp, C.c_int]),
        "apc_batch_solve_ms": (C.c_float, [vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data


@dataclass
class GpuCells:
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    h: np.ndarray
    first: np.ndarray
    count: np.ndarray
    type: np.ndarray
    firstneigh: np.ndarray
    numneigh: np.ndarray
    neigh24: np.ndarray
    nc: int
    nv: int
    nb: int

    @property
    def m(self) -> int:
        return self.nc + self.nv


@dataclass
class GpuFields:
    density: np.ndarray
    potential: np.ndarray
    deriv: np.ndarray


def make_config(n: int, depth: int, gfd_c: float, lm: int = 17,
                box=(0.0, 1.0, 0.0, 1.0, 0.0, 1.0), bc: int = 1, precision: int = APC_PREC_FP64,
                restart: int = 30, rtol: float = 1e-10, atol: float = 1e-50, dtol: float = 1e5,
                max_it: int = 10000, mixed_restart: int = 0, mixed_inner_rtol: float = 0.0,
                device: int = 0, maxnc: int = 10000, nmax_cap: int = 0, precond: int = APC_PRECOND_MULTIGRID,
                mg_sweeps: int = 0, mg_omega: float = 0.0, mg_alpha: float = 0.0, mg_reorth: int = 0,
                warm_start: int = 0, solve_graphs: int = 1) -> "ApcConfig":
    """An apc_config: the library defaults with the given fields set."""
    lib = load_library()
    cfg = ApcConfig()
    lib.apc_config_default(C.byref(cfg))
    cfg.n_particles = n
    cfg.depth = depth
    cfg.bc = bc
    for k in range(6):
        cfg.box[k] = box[k]
    cfg.gfd_c = gfd_c
    cfg.lm = lm
    cfg.maxnc = maxnc
    cfg.nmax_cap = nmax_cap
    cfg.gmres_restart = restart
    cfg.gmres_rtol = rtol
    cfg.gmres_atol = atol
    cfg.gmres_dtol = dtol
    cfg.gmres_max_it = max_it
    cfg.precision = precision
    cfg.mixed_restart = mixed_restart
    cfg.mixed_inner_rtol = mixed_inner_rtol
    cfg.device = device
    cfg.mixed_precond = precond
    cfg.mg_sweeps = mg_sweeps
    cfg.mg_omega = mg_omega
    cfg.mg_alpha = mg_alpha
    cfg.mg_reorth = mg_reorth
    cfg.warm_start = warm_start
    cfg.mixed_solve_graphs = solve_graphs
    return cfg


class GpuPath:
    """One particle set resident on the GPU, driven phase by phase through the C ABI."""

    def __init__(self, parts, depth: int, gfd_c: float, lm: int = 17, **kw):
        self.lib = load_library()
        cfg = make_config(parts.n, depth, gfd_c, lm, **kw)
        self._owned = True
        self.cfg = cfg
        self.n = parts.n
        self.depth = depth
        self.lm = lm
        h = C.c_void_p()
        self._check(self.lib.apc_create(C.byref(cfg), C.byref(h)), "apc_create", None)
        self.h = h
        self.set_particles(parts)

    def set_particles(self, parts: "ics.Particles") -> None:
        """Replace the particle set (same count) from host arrays; cells and fields are
        invalidated until the next select."""
        if parts.n != self.n:
            raise ValueError(f"particle count {parts.n} != {self.n}")
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in parts.as_tuple()]
        self._check(self.lib.apc_set_particles(self.h, *[_ptr(a) for a in arrs]), "apc_set_particles")

    def _check(self, rc: int, where: str, h="self"):
        if rc != 0:
            msg = self.lib.apc_status_string(rc).decode()
            if h == "self" and getattr(self, "h", None):
                detail = self.lib.apc_last_error(self.h).decode()
                if detail:
                    msg += "; " + detail
            raise ApcError(rc, where, msg)

    @classmethod
    def view(cls, lib, h, cfg: "ApcConfig") -> "GpuPath":
        """A GpuPath over a context owned elsewhere (a batch box); close() leaves it alone."""
        g = cls.__new__(cls)
        g.lib, g.h, g.cfg, g._owned = lib, h, cfg, False
        g.n, g.depth, g.lm = cfg.n_particles, cfg.depth, cfg.lm
        return g

    def close(self):
        if getattr(self, "h", None):
            if getattr(self, "_owned", True):
                self.lib.apc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- phases ----
    def select(self) -> int:
        m = C.c_int()
        self._check(self.lib.apc_select(self.h, C.byref(m)), "apc_select")
        return m.value

    def solve(self, c_dens: float, c_pot: float, c_field: float = -1.0) -> int:
        self._check(self.lib.apc_solve(self.h, c_dens, c_pot, c_field), "apc_solve")
        return 0

    def move_velocity(self, dt: float, c_vel: float) -> float:
        d = C.c_double()
        self._check(self.lib.apc_move_velocity(self.h, dt, c_vel, C.byref(d)), "apc_move_velocity")
        return d.value

    def move_position(self, dt: float, c_pos: float) -> float:
        d = C.c_double()
        self._check(self.lib.apc_move_position(self.h, dt, c_pos, C.byref(d)), "apc_move_position")
        return d.value

    def step(self, dt, c_dens, c_pot, c_field, c_vel, c_pos):
        p = ApcStepParams(dt, c_dens, c_pot, c_field, c_vel, c_pos)
        m, dv, dx = C.c_int(), C.c_double(), C.c_double()
        self._check(self.lib.apc_step(self.h, C.byref(p), C.byref(m), C.byref(dv), C.byref(dx)), "apc_step")
        return m.value, dv.value, dx.value

    def synchronize(self):
        self._check(self.lib.apc_synchronize(self.h), "apc_synchronize")

    # ---- derivatives (device pointers: ints, e.g. torch tensor data_ptr()) ----
    def hessians_device(self, ptrs):
        self._check(self.lib.apc_get_hessians_device(self.h, *[C.c_void_p(p) for p in ptrs]),
                    "apc_get_hessians_device")

    def max_cell_density(self) -> float:
        v = C.c_double()
        self._check(self.lib.apc_max_cell_density(self.h, C.byref(v)), "apc_max_cell_density")
        return v.value

    def adaptive_dt(self, delta_a: float) -> float:
        v = C.c_double()
        self._check(self.lib.apc_adaptive_dt(self.h, delta_a, C.byref(v)), "apc_adaptive_dt")
        return v.value

    def fields_from_rhs(self, rhs_ptr: int):
        self._check(self.lib.apc_fields_from_rhs(self.h, C.c_void_p(rhs_ptr)), "apc_fields_from_rhs")

    def solve_vjp(self, g_deriv_ptr: int, g_rhs_ptr: int, g_rho_ptr: int | None = None, g_phi_ptr: int | None = None):
        self._check(self.lib.apc_solve_vjp(self.h, C.c_void_p(g_deriv_ptr), C.c_void_p(g_rhs_ptr),
                                           C.c_void_p(g_rho_ptr) if g_rho_ptr else None,
                                           C.c_void_p(g_phi_ptr) if g_phi_ptr else None), "apc_solve_vjp")

    def trajectory_vjp(self, steps, start_dt: float, start_c_pos: float, every: int, state0_ptrs, cot_ptrs,
                       statef_ptrs=None):
        """steps: (dt, c_dens, c_pot, c_field, c_vel, c_pos) per step; *_ptrs: 6 device
        pointers each (x, y, z, vx, vy, vz) in caller order; cot is updated in place."""
        k = len(steps)
        arr = (ApcStepParams * max(k, 1))(*[ApcStepParams(*q) for q in steps])
        t = ApcTrajectory(k, arr, start_dt, start_c_pos, every)
        s0 = (C.c_void_p * 6)(*state0_ptrs)
        ct = (C.c_void_p * 6)(*cot_ptrs)
        sf = (C.c_void_p * 6)(*statef_ptrs) if statef_ptrs is not None else None
        self._check(self.lib.apc_trajectory_vjp(self.h, C.byref(t), s0, ct, sf), "apc_trajectory_vjp")

    # ---- results ----
    def counts(self):
        nc, nv, nb, nn = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        self._check(self.lib.apc_get_cell_counts(self.h, C.byref(nc), C.byref(nv), C.byref(nb), C.byref(nn)),
                    "apc_get_cell_counts")
        return nc.value, nv.value, nb.value, nn.value

    def cells(self) -> GpuCells:
        nc, nv, nb, nn = self.counts()
        m = nc + nv
        d = [np.zeros(m) for _ in range(4)]
        i = [np.zeros(m, np.int32) for _ in range(5)]
        nb24 = np.zeros(max(nn, 1), np.int32)
        self._check(self.lib.apc_get_cells(self.h, *[_ptr(a) for a in d], *[_ptr(a) for a in i], _ptr(nb24)),
                    "apc_get_cells")
        return GpuCells(*d, *i, nb24[:nn], nc, nv, nb)

    def codes(self) -> np.ndarray:
        nc, nv, _, _ = self.counts()
        out = np.zeros(nc + nv, np.uint64)
        self._check(self.lib.apc_get_cell_codes(self.h, _ptr(out)), "apc_get_cell_codes")
        return out

    def keys(self):
        k = np.zeros(self.n, np.uint64)
        idx = np.zeros(self.n, np.int32)
        self._check(self.lib.apc_get_keys(self.h, _ptr(k), _ptr(idx)), "apc_get_keys")
        return k, idx

    def octree_levels(self):
        nn = np.zeros(self.depth + 1, np.int32)
        self._check(self.lib.apc_get_octree_levels(self.h, _ptr(nn)), "apc_get_octree_levels")
        return nn

    def fields(self) -> GpuFields:
        nc, nv, _, _ = self.counts()
        m = nc + nv
        rho, phi, der = np.zeros(m), np.zeros(m), np.zeros(9 * m)
        self._check(self.lib.apc_get_fields(self.h, _ptr(rho), _ptr(phi), _ptr(der)), "apc_get_fields")
        return GpuFields(rho, phi, der.reshape(m, 9))

    def stencils(self):
        nc, nv, _, _ = self.counts()
        m = nc + nv
        idx = np.zeros(m * self.lm, np.int32)
        dist = np.zeros(m * self.lm)
        self._check(self.lib.apc_get_stencils(self.h, _ptr(idx), _ptr(dist)), "apc_get_stencils")
        return idx.reshape(m, self.lm), dist.reshape(m, self.lm)

    def solve_stats(self) -> dict:
        st = ApcSolveStats()
        self._check(self.lib.apc_get_solve_stats(self.h, C.byref(st)), "apc_get_solve_stats")
        return {f: getattr(st, f) for f, _ in ApcSolveStats._fields_}

    def matrix(self, which: int):
        n, nnz = C.c_int(), C.c_int()
        self._check(self.lib.apc_get_matrix(self.h, which, C.byref(n), C.byref(nnz), None, None, None),
                    "apc_get_matrix")
        rp = np.zeros(n.value + 1, np.int32)
        ci = np.zeros(max(nnz.value, 1), np.int32)
        v = np.zeros(max(nnz.value, 1))
        self._check(self.lib.apc_get_matrix(self.h, which, None, None, _ptr(rp), _ptr(ci), _ptr(v)),
                    "apc_get_matrix")
        return rp, ci[: nnz.value], v[: nnz.value]

    def particles(self):
        out = [np.zeros(self.n) for _ in range(9)]
        self._check(self.lib.apc_get_particles(self.h, *[_ptr(a) for a in out]), "apc_get_particles")
        return out

    def kernel_launches(self) -> int:
        return int(self.lib.apc_kernel_launches(self.h))

    def profile(self) -> dict:
        pr = ApcProfile()
        self._check(self.lib.apc_get_profile(self.h, C.byref(pr)), "apc_get_profile")
        return {f: getattr(pr, f) for f, _ in ApcProfile._fields_}

    def reset_profile(self):
        self._check(self.lib.apc_reset_profile(self.h), "apc_reset_profile")

    def phase_times(self):
        a, b, c = C.c_double(), C.c_double(), C.c_double()
        self._check(self.lib.apc_get_phase_times(self.h, C.byref(a), C.byref(b), C.byref(c)), "apc_get_phase_times")
        return a.value, b.value, c.value


class BatchPath:
    """Independent boxes stepped together through apc_batch_step (one context each)."""

    def __init__(self, boxes, n_workers: int = 0, solve_mode: int = APC_BATCH_SOLVE_PER_BOX):
        """boxes: sequence of (Particles, dict of make_config keywords incl. depth, gfd_c);
        solve_mode: APC_BATCH_SOLVE_PER_BOX or APC_BATCH_SOLVE_QUEUED (apc_batch_set_solve_mode)."""
        self.lib = load_library()
        n = len(boxes)
        cfgs = (ApcConfig * n)()
        for i, (parts, kw) in enumerate(boxes):
            kw = dict(kw)
            cfgs[i] = make_config(parts.n, kw.pop("depth"), kw.pop("gfd_c"), **kw)
        h = C.c_void_p()
        rc = self.lib.apc_batch_create(cfgs, n, n_workers, C.byref(h))
        if rc != 0:
            raise ApcError(rc, "apc_batch_create", self.lib.apc_status_string(rc).decode())
        self.h = h
        self.cfgs = cfgs
        rc = self.lib.apc_batch_set_solve_mode(h, solve_mode)
        if rc != 0:
            raise ApcError(rc, "apc_batch_set_solve_mode", self.lib.apc_status_string(rc).decode())
        self.boxes = [GpuPath.view(self.lib, C.c_void_p(self.lib.apc_batch_context(h, i)), cfgs[i]) for i in range(n)]
        for g, (parts, _) in zip(self.boxes, boxes):
            arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in parts.as_tuple()]
            g._check(self.lib.apc_set_particles(g.h, *[_ptr(a) for a in arrs]), "apc_set_particles")

    def __len__(self) -> int:
        return len(self.boxes)

    def solve_ms(self) -> float:
        """Device time of the last step's queued solve launches (0 in per-box mode)."""
        return float(self.lib.apc_batch_solve_ms(self.h))

    def step(self, params):
        """params: one (dt, c_dens, c_pot, c_field, c_vel, c_pos) per box."""
        n = len(self.boxes)
        p = (ApcStepParams * n)(*[ApcStepParams(*q) for q in params])
        st = (C.c_int * n)()
        dv = np.zeros(n)
        dx = np.zeros(n)
        rc = self.lib.apc_batch_step(self.h, p, st, _ptr(dv), _ptr(dx))
        if rc != 0:
            bad = [i for i in range(n) if st[i] != 0]
            raise ApcError(rc, "apc_batch_step", f"boxes {bad}: " + self.lib.apc_status_string(rc).decode())
        return dv, dx

    def close(self):
        if getattr(self, "h", None):
            for g in self.boxes:
                g.h = None
            self.lib.apc_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
