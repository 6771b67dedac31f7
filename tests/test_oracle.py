"""CPU tests of the oracle: the plain-C restatement against the reference's own outputs
(golden fixtures made by running the reference, and a live run of oracle/_ref), plus
known-answer checks of its numerical building blocks."""
from __future__ import annotations

import ctypes as C
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN

import refbind  # noqa: E402  (oracle/refbind.py)
from apcloud import ics  # noqa: E402

CASES = sorted(glob.glob(os.path.join(GOLDEN, "*.npz")))


def _parts(g):
    return ics.Particles(*(g[k].copy() for k in ("x", "y", "z", "vx", "vy", "vz")))


def _run_first_step(which, g):
    p = _parts(g)
    r = refbind.CpuPath(which, p, int(g["depth"]), float(g["gfd_c"]), int(g["lm"]))
    r.set_gmres(int(g["restart"]), float(g["rtol"]))
    r.reset_solve_stats()
    m = r.select()
    out = {"m": m, "cells": r.cells(), "keys": r.keys(), "levels": r.octree_levels()}
    r.solve(float(g["c_dens"]), float(g["c_pot"]), -1.0)
    out["fields"] = r.fields()
    out["its"] = [s[0] for s in r.solve_stats()[-2:]]
    out["dv"] = r.move_velocity(float(g["delta_a"]), float(g["c_vel"]))
    out["dx"] = r.move_position(float(g["delta_a"]), float(g["c_pos"]))
    out["parts"] = r.particles()
    r.close()
    return out


@pytest.mark.parametrize("path", CASES, ids=[os.path.basename(c)[:-4] for c in CASES])
def test_oracle_matches_reference_golden(oracle_lib, path):
    """Bit-exact: keys, octree levels, every cell array incl. Neigh24 in the reference's
    order, GMRES iteration counts; fields and the first step to 1e-13 relative."""
    g = np.load(path)
    o = _run_first_step("oracle", g)
    keys, idx = o["keys"]
    assert np.array_equal(keys, g["keys"])
    # std::sort leaves the order of equal keys unspecified: compare index sets per key
    assert np.array_equal(np.lexsort((idx, keys)), np.lexsort((g["key_index"], g["keys"]))) or \
        np.array_equal(np.sort(idx), np.sort(g["key_index"]))
    assert np.array_equal(o["levels"], g["levels"])
    c = o["cells"]
    assert (c.nc, c.nv, o["m"]) == (int(g["nc"]), int(g["nv"]), int(g["m"]))
    for f, gf in (("x", "cx"), ("y", "cy"), ("z", "cz"), ("h", "ch"), ("count", "ccount"), ("type", "ctype"),
                  ("firstneigh", "firstneigh"), ("numneigh", "numneigh"), ("neigh24", "neigh24")):
        assert np.array_equal(getattr(c, f), g[gf]), f
    assert np.array_equal(c.first, g["cfirst"])
    assert list(o["its"]) == list(g["its"])
    for f in ("density", "potential", "deriv"):
        a, b = getattr(o["fields"], f), g[f]
        assert np.max(np.abs(a - b)) <= 1e-13 * np.max(np.abs(b)), f
    for k, name in enumerate(("step1_x", "step1_y", "step1_z", "step1_vx", "step1_vy", "step1_vz", "ax", "ay", "az")):
        a, b = o["parts"][k], g[name]
        assert np.max(np.abs(a - b)) <= 1e-13 * max(1.0, np.max(np.abs(b))), name
    assert o["dv"] == pytest.approx(float(g["max_dv"]), rel=1e-13)
    assert o["dx"] == pytest.approx(float(g["max_dx"]), rel=1e-13)


def test_oracle_matches_reference_live(oracle_lib, reference_lib):
    """The restatement against the reference code itself on a fresh seed, 2 steps."""
    cfg = ics.config("ball32k", n=1500, seed=99)
    p = cfg.particles()
    runs = {}
    for which in ("ref", "oracle"):
        r = refbind.CpuPath(which, p, cfg.depth, cfg.gfd_c)
        r.set_gmres(30, 1e-10)
        t = cfg.a_start + 0.5 * cfg.delta_a
        for _ in range(2):
            r.select()
            r.solve(1.0 / p.n, 1.5 / t, -1.0)
            r.move_velocity(cfg.delta_a, ics.kick_factor(t, 1.0, 0.0))
            r.move_position(cfg.delta_a, ics.drift_factor(t + cfg.delta_a / 2, 1.0, 0.0))
            t += cfg.delta_a
        runs[which] = (r.cells(), r.fields(), r.particles())
        r.close()
    (ca, fa, pa), (cb, fb, pb) = runs["ref"], runs["oracle"]
    for f in ("x", "y", "z", "h", "first", "count", "type", "firstneigh", "numneigh", "neigh24"):
        assert np.array_equal(getattr(ca, f), getattr(cb, f)), f
    for f in ("density", "potential", "deriv"):
        assert np.array_equal(getattr(fa, f), getattr(fb, f)), f
    for a, b in zip(pa, pb):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("case", ["ball32k", "eds64"])
def test_oracle_stencils_and_matrices_match_reference(oracle_lib, reference_lib, case):
    """The GFD stencils (the reference's: the order in which Build_Linear_System inserts
    row i of A1, solver.cpp:116-125) and both assembled matrices, bit for bit, on reduced
    versions of the ball and the Zel'dovich box (uniform lattice ties included)."""
    cfg = ics.config(case, n=3000 if case == "ball32k" else 16 ** 3, seed=11)
    p = cfg.particles()
    out = {}
    for which in ("ref", "oracle"):
        r = refbind.CpuPath(which, p, cfg.depth, cfg.gfd_c, cfg.lm)
        r.set_gmres(30, 1e-10)
        r.select()
        t = cfg.a_start + 0.5 * cfg.delta_a
        r.solve(1.0 / p.n, 1.5 * cfg.omega0 / t, -1.0)
        out[which] = (r.stencils(), r.last_matrix(0), r.last_matrix(1))
        r.close()
    assert out["ref"][0].shape[1] == cfg.lm
    assert np.array_equal(out["ref"][0], out["oracle"][0])
    for k in (1, 2):
        for a, b in zip(out["ref"][k], out["oracle"][k]):
            assert np.array_equal(a, b)


def test_key64_known_answers(oracle_lib):
    lib = C.CDLL(oracle_lib)
    lib.apcor_key64.restype = C.c_uint64
    lib.apcor_key64.argtypes = [C.c_double] * 3 + [C.POINTER(C.c_double), C.c_int]
    box = (C.c_double * 6)(0, 1, 0, 1, 0, 1)
    # depth 1: one octant digit x->4, y->2, z->1; the midpoint itself goes up (>=)
    assert lib.apcor_key64(0.1, 0.1, 0.1, box, 1) == 0
    assert lib.apcor_key64(0.6, 0.1, 0.9, box, 1) == 5
    assert lib.apcor_key64(0.5, 0.5, 0.5, box, 1) == 7
    # depth 2: (0.3, 0.8, 0.55): level 1 digit 0b011, level 2: x 0.3>=0.25 ->1, y 0.8>=0.75 ->1, z 0.55<0.75 ->0
    assert lib.apcor_key64(0.3, 0.8, 0.55, box, 2) == (0b011 << 3) | 0b110
    # depth 21 uses 63 bits; the far corner is all ones
    assert lib.apcor_key64(1.0, 1.0, 1.0, box, 21) == (1 << 63) - 1
    # non-unit box
    box2 = (C.c_double * 6)(0, 1000, 0, 1000, 0, 1000)
    assert lib.apcor_key64(999.0, 1.0, 501.0, box2, 1) == 0b101


def test_householder_lsq_matches_numpy(oracle_lib):
    lib = C.CDLL(oracle_lib)
    f = lib.oracle_dgels_rowmajor
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int]
    rng = np.random.default_rng(0)
    for m, n, k in ((17, 9, 17), (17, 9, 1), (30, 9, 3)):
        A = rng.standard_normal((m, n))
        B = rng.standard_normal((m, k))
        a, b = A.copy(), B.copy()
        assert f(m, n, k, a.ctypes.data, n, b.ctypes.data, k) == 0
        ref = np.linalg.lstsq(A, B, rcond=None)[0]
        assert np.allclose(b[:n], ref, rtol=1e-12, atol=1e-12)
    # rank deficient: a zero column gives info = column index (1-based)
    A = rng.standard_normal((17, 9))
    A[:, 4] = 0.0
    b = np.ones((17, 1))
    assert f(17, 9, 1, A.ctypes.data, 9, b.ctypes.data, 1) == 5


def test_gmres_petsc_semantics(oracle_lib):
    """GMRES(m)+Jacobi on a small nonsymmetric system reaches rtol on the
    preconditioned residual, restarts correctly, and reports DIVERGED_ITS at max_it."""

    class P(C.Structure):
        _fields_ = [("restart", C.c_int), ("rtol", C.c_double), ("atol", C.c_double), ("dtol", C.c_double),
                    ("max_it", C.c_int), ("its", C.c_int), ("rnorm", C.c_double), ("reason", C.c_int)]

    lib = C.CDLL(oracle_lib)
    lib.oracle_gmres_csr.restype = C.c_int
    lib.oracle_gmres_csr.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.POINTER(P)]
    n = 200
    rng = np.random.default_rng(1)
    A = np.diag(4.0 + rng.random(n)) + np.diag(-1.0 * np.ones(n - 1), 1) + np.diag(-1.3 * np.ones(n - 1), -1)
    rp = np.zeros(n + 1, np.int32)
    ci, vals = [], []
    for i in range(n):
        nz = np.nonzero(A[i])[0]
        ci += list(nz)
        vals += list(A[i, nz])
        rp[i + 1] = len(ci)
    ci = np.array(ci, np.int32)
    vals = np.array(vals)
    b = rng.standard_normal(n)
    x = np.zeros(n)
    p = P(10, 1e-10, 1e-50, 1e5, 10000, 0, 0.0, 0)
    lib.oracle_gmres_csr(n, rp.ctypes.data, ci.ctypes.data, vals.ctypes.data, b.ctypes.data, x.ctypes.data,
                         C.byref(p))
    assert p.reason == 2
    d = np.diag(A)
    assert np.linalg.norm((b - A @ x) / d) <= 1e-10 * np.linalg.norm(b / d) * 1.0001
    assert p.its > 10  # needed at least one restart
    p2 = P(10, 1e-14, 1e-50, 1e5, 7, 0, 0.0, 0)
    x[:] = 0
    lib.oracle_gmres_csr(n, rp.ctypes.data, ci.ctypes.data, vals.ctypes.data, b.ctypes.data, x.ctypes.data,
                         C.byref(p2))
    assert p2.reason == -3 and p2.its == 7


@pytest.mark.parametrize("path", CASES, ids=[os.path.basename(c)[:-4] for c in CASES])
def test_oracle_differentiation_of_a_given_potential(oracle_lib, path):
    """The oracle's Solver::Differentiate applied to a given potential (the checker behind
    the GPU's full-size differentiation test): on the reference's own potential it gives the
    reference's derivatives (golden) to the bit, and on the oracle's potential its solve's
    derivatives to the bit."""
    g = np.load(path)
    r = refbind.CpuPath("oracle", _parts(g), int(g["depth"]), float(g["gfd_c"]), int(g["lm"]))
    r.set_gmres(int(g["restart"]), float(g["rtol"]))
    r.select()
    d_ref = r.differentiate(g["potential"], -1.0)
    assert np.array_equal(d_ref.reshape(-1), g["deriv"].reshape(-1))
    r.solve(float(g["c_dens"]), float(g["c_pot"]), -1.0)
    f = r.fields()
    assert np.array_equal(r.differentiate(f.potential, -1.0), f.deriv)
    r.close()
