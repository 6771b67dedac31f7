"""Test infrastructure: ctypes binding of oracle/_ref/libapcref.so (the reference's
own octree/mover/solver code, built by ``make -C oracle ref``) and of
oracle/liboracle.so (the plain-C restatement).  Only tests, smoke() and the CPU
baseline leg of bench.py load this module."""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "libapcref.so")
ORACLE_SO = os.path.join(HERE, "liboracle.so")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_up = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")


@dataclass
class Cells:
    """Computational_particle arrays (particle.h:23-53)."""
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
class Fields:
    density: np.ndarray
    potential: np.ndarray
    deriv: np.ndarray  # (M, 9): p_x p_y p_z p_xx p_yy p_zz p_xy p_xz p_yz


def _bind_common(lib, prefix):
    f = getattr(lib, prefix + "create")
    f.restype = C.c_void_p
    f.argtypes = [C.c_int, _dp, _dp, _dp, _dp, _dp, _dp, C.c_int, C.c_int, _dp, C.c_double, C.c_int]
    lib_dict = {}
    for name, res, args in [
        ("destroy", None, [C.c_void_p]),
        ("set_gmres", None, [C.c_int, C.c_double, C.c_double, C.c_double, C.c_int]),
        ("set_maxnc", None, [C.c_void_p, C.c_int]),
        ("select", C.c_int, [C.c_void_p]),
        ("cell_counts", C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                  C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        ("get_cells", C.c_int, [C.c_void_p, _dp, _dp, _dp, _dp, _ip, _ip, _ip, _ip, _ip, _ip]),
        ("get_keys", C.c_int, [C.c_void_p, _up, _ip]),
        ("octree_levels", C.c_int, [C.c_void_p, _ip]),
        ("solve", C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double]),
        ("get_fields", C.c_int, [C.c_void_p, _dp, _dp, _dp]),
        ("differentiate", C.c_int, [C.c_void_p, _dp, C.c_double, _dp]),
        ("solve_stats", C.c_int, [C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double),
                                  C.POINTER(C.c_int), C.POINTER(C.c_double)]),
        ("solve_count", C.c_int, []),
        ("reset_solve_stats", None, []),
        ("last_matrix", C.c_int, [C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_void_p,
                                  C.c_void_p, C.c_void_p]),
        ("move_velocity", C.c_double, [C.c_void_p, C.c_double, C.c_double]),
        ("move_position", C.c_double, [C.c_void_p, C.c_double, C.c_double]),
        ("get_particles", C.c_int, [C.c_void_p] + [C.c_void_p] * 9),
        ("phase_times", None, [C.c_void_p, _dp]),
        ("set_threads", None, [C.c_int]),
    ]:
        fn = getattr(lib, prefix + name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
        lib_dict[name] = fn
    lib_dict["create"] = f
    if prefix == "apcref_":
        fn = lib.apcref_get_stencils
        fn.restype, fn.argtypes = C.c_int, [C.c_int, _ip]
    else:
        fn = lib.apcor_get_stencils
        fn.restype, fn.argtypes = C.c_int, [C.c_void_p, _ip, _dp]
    lib_dict["get_stencils"] = fn
    return lib_dict


class CpuPath:
    """One particle set driven through a CPU implementation of the hot path, with the
    phase calls of Mover / Solver (mover.h:31-43, solver.h:53-62)."""

    _libs: dict = {}

    def __init__(self, which: str, parts, depth: int, gfd_c: float, lm: int = 17,
                 box=(0.0, 1.0, 0.0, 1.0, 0.0, 1.0), bc: int = 1):
        so, prefix = (REF_SO, "apcref_") if which == "ref" else (ORACLE_SO, "apcor_")
        if so not in CpuPath._libs:
            if not os.path.exists(so):
                raise FileNotFoundError(f"{so} missing: run `make -C oracle`")
            CpuPath._libs[so] = _bind_common(C.CDLL(so), prefix)
        self.f = CpuPath._libs[so]
        self.n = parts.n
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in parts.as_tuple()]
        self.h = self.f["create"](self.n, *arrs, depth, bc, np.asarray(box, dtype=np.float64), gfd_c, lm)
        self.depth = depth
        self.lm = lm
        self.which = which

    def close(self):
        if self.h:
            self.f["destroy"](self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_gmres(self, restart=30, rtol=1e-10, atol=1e-50, dtol=1e5, max_it=10000):
        self.f["set_gmres"](restart, rtol, atol, dtol, max_it)

    def set_maxnc(self, maxnc: int):
        self.f["set_maxnc"](self.h, maxnc)

    def select(self) -> int:
        return self.f["select"](self.h)

    def cells(self) -> Cells:
        nc, nv, nb, nn = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        m = self.f["cell_counts"](self.h, C.byref(nc), C.byref(nv), C.byref(nb), C.byref(nn))
        d = [np.zeros(m) for _ in range(4)]
        i = [np.zeros(m, np.int32) for _ in range(5)]
        nb24 = np.zeros(max(nn.value, 1), np.int32)
        self.f["get_cells"](self.h, *d, *i, nb24)
        return Cells(*d, *i, nb24[: nn.value], nc.value, nv.value, nb.value)

    def keys(self):
        k = np.zeros(self.n, np.uint64)
        idx = np.zeros(self.n, np.int32)
        self.f["get_keys"](self.h, k, idx)
        return k, idx

    def octree_levels(self):
        nn = np.zeros(self.depth + 1, np.int32)
        self.f["octree_levels"](self.h, nn)
        return nn

    def solve(self, c_dens: float, c_pot: float, c_field: float = -1.0) -> int:
        return self.f["solve"](self.h, c_dens, c_pot, c_field)

    def fields(self) -> Fields:
        nc, nv, nb, nn = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        self.f["cell_counts"](self.h, C.byref(nc), C.byref(nv), C.byref(nb), C.byref(nn))
        m = nc.value + nv.value
        rho, phi, der = np.zeros(m), np.zeros(m), np.zeros(9 * m)
        self.f["get_fields"](self.h, rho, phi, der)
        return Fields(rho, phi, der.reshape(m, 9))

    def differentiate(self, potential: np.ndarray, c_field: float = -1.0) -> np.ndarray:
        """Solver::Differentiate (solver.cpp:295-362) of a given potential on the selected
        cells (the oracle only)."""
        if "differentiate" not in self.f:
            raise NotImplementedError("differentiate: oracle only")
        m = self.cells().m
        d = np.zeros(9 * m)
        rc = self.f["differentiate"](self.h, np.ascontiguousarray(potential, dtype=np.float64), c_field, d)
        if rc != 0:
            raise RuntimeError(f"differentiate failed: {rc}")
        return d.reshape(m, 9)

    def stencils(self) -> np.ndarray:
        """(M, lm) GFD neighbour indices of the last solve, in search order.  For the
        reference they come from the order in which Build_Linear_System inserts row i of
        A1 (solver.cpp:116-125), recorded by the PETSc shim."""
        nc, nv, nb, nn = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        self.f["cell_counts"](self.h, C.byref(nc), C.byref(nv), C.byref(nb), C.byref(nn))
        m = nc.value + nv.value
        idx = np.zeros(m * self.lm, np.int32)
        if self.which == "ref":
            if self.f["get_stencils"](self.lm, idx) != m:
                raise RuntimeError("reference stencils unavailable (no solve since the last select?)")
        else:
            self.f["get_stencils"](self.h, idx, np.zeros(m * self.lm))
        return idx.reshape(m, self.lm)

    def set_threads(self, threads: int):
        """Host threads of the reference's GMRES shim (1 = serial, the pinned order)."""
        self.f["set_threads"](threads)

    def solve_stats(self):
        out = []
        for k in range(self.f["solve_count"]()):
            its, rn, rs, sec = C.c_int(), C.c_double(), C.c_int(), C.c_double()
            self.f["solve_stats"](k, C.byref(its), C.byref(rn), C.byref(rs), C.byref(sec))
            out.append((its.value, rn.value, rs.value, sec.value))
        return out

    def reset_solve_stats(self):
        self.f["reset_solve_stats"]()

    def last_matrix(self, which: int):
        n, nnz = C.c_int(), C.c_int()
        self.f["last_matrix"](which, C.byref(n), C.byref(nnz), None, None, None)
        rp = np.zeros(n.value + 1, np.int32)
        ci = np.zeros(nnz.value, np.int32)
        v = np.zeros(nnz.value)
        self.f["last_matrix"](which, None, None, rp.ctypes.data, ci.ctypes.data, v.ctypes.data)
        return rp, ci, v

    def max_cell_density(self) -> float:
        """max n_p / h / h / h over the cells (controller.cpp:150-156), as the reference."""
        c = self.cells()
        return float(np.max(c.count.astype(np.float64) / c.h / c.h / c.h))

    def adaptive_dt(self, delta_a: float) -> float:
        """controller.cpp:157-162."""
        import math

        v = 0.05 * delta_a * (1.0 / math.pow(self.max_cell_density(), 1.0 / 2))
        return delta_a if v > delta_a else v

    def move_velocity(self, dt: float, c_vel: float) -> float:
        return self.f["move_velocity"](self.h, dt, c_vel)

    def move_position(self, dt: float, c_pos: float) -> float:
        return self.f["move_position"](self.h, dt, c_pos)

    def particles(self):
        out = [np.zeros(self.n) for _ in range(9)]
        self.f["get_particles"](self.h, *[a.ctypes.data for a in out])
        return out

    def phase_times(self):
        t = np.zeros(3)
        self.f["phase_times"](self.h, t)
        return t
