"""Generate the golden fixtures of tests/golden/ by running the REFERENCE's own code.

    make -C oracle ref && python tests/golden/make_golden.py

oracle/_ref/libapcref.so is the reference's octree.cpp / mover.cpp / particle.cpp /
solver.cpp compiled from the reference sources with the PETSc / LAPACKE / MPI stand-ins
of oracle/shim.  Each fixture holds:
  - seeded synthetic inputs;
  - the reference's outputs after select (sorted keys, octree levels, cell arrays,
    Neigh24);
  - the outputs after solve (density, potential, derivatives, GMRES iteration counts);
  - the outputs after a full step (particles, accelerations);
  - for the multi-step case, the particles after `steps` steps of the Controller
    sequence (controller.cpp:133-208).
The reference ships no test data or golden vectors; these fixtures pin the oracle and
the CUDA path to the reference's behaviour on the same inputs.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "ap-cloud-cosmology_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from apcloud import ics  # noqa: E402
import refbind  # noqa: E402

CASES = {
    # cold ball, 2048 particles, the uniform-ball config at reduced N
    "ball2k": dict(cfg=("ball32k", dict(n=2048, seed=11)), steps=1),
    # two overlapping balls: strongly uneven refinement and many vacuum (Type -1) cells
    "twoballs3k": dict(cfg=None, steps=1),
    # 16^3 Zel'dovich lattice with large displacement, three steps
    "zel16": dict(cfg=("eds64", dict(n=16 ** 3, rms_spacing=0.6, seed=5, a_start=0.2, a_end=0.5, steps=8)),
                  steps=3),
}


def two_balls(seed=3):
    a = ics.uniform_ball(2048, radius=0.2, center=(0.35, 0.4, 0.45), seed=seed)
    b = ics.uniform_ball(1024, radius=0.08, center=(0.7, 0.62, 0.58), seed=seed + 1)
    cat = [np.concatenate([u, v]) for u, v in zip(a.as_tuple(), b.as_tuple())]
    return ics.Particles(*cat)


def run_case(name: str, spec: dict) -> dict:
    if spec["cfg"] is None:
        cfg = ics.config("ball32k", n=3072)
        parts = two_balls()
    else:
        cfg = ics.config(spec["cfg"][0], **spec["cfg"][1])
        parts = cfg.particles()
    out = {"x": parts.x, "y": parts.y, "z": parts.z, "vx": parts.vx, "vy": parts.vy, "vz": parts.vz,
           "depth": cfg.depth, "gfd_c": cfg.gfd_c, "lm": cfg.lm, "omega0": cfg.omega0, "omegal": cfg.omegal,
           "a_start": cfg.a_start, "delta_a": cfg.delta_a, "restart": cfg.restart, "rtol": cfg.rtol,
           "steps": spec["steps"]}
    r = refbind.CpuPath("ref", parts, cfg.depth, cfg.gfd_c, cfg.lm)
    r.set_gmres(cfg.restart, cfg.rtol)
    t = cfg.a_start + 0.5 * cfg.delta_a
    for step in range(spec["steps"]):
        r.reset_solve_stats()
        m = r.select()
        if step == 0:
            k, idx = r.keys()
            c = r.cells()
            out.update(keys=k, key_index=idx, levels=r.octree_levels(), m=m, nc=c.nc, nv=c.nv,
                       cx=c.x, cy=c.y, cz=c.z, ch=c.h, cfirst=c.first, ccount=c.count, ctype=c.type,
                       firstneigh=c.firstneigh, numneigh=c.numneigh, neigh24=c.neigh24)
        c_dens, c_pot = 1.0 / parts.n, 1.5 * cfg.omega0 / t
        r.solve(c_dens, c_pot, -1.0)
        dt = cfg.delta_a
        cv = ics.kick_factor(t, cfg.omega0, cfg.omegal)
        cp = ics.drift_factor(t + dt / 2, cfg.omega0, cfg.omegal)
        if step == 0:
            f = r.fields()
            st = r.solve_stats()
            out.update(density=f.density, potential=f.potential, deriv=f.deriv, c_dens=c_dens, c_pot=c_pot,
                       its=np.array([s[0] for s in st[-2:]], np.int32), t0=t, c_vel=cv, c_pos=cp)
        dv = r.move_velocity(dt, cv)
        dx = r.move_position(dt, cp)
        p = r.particles()
        if step == 0:
            out.update(ax=p[6], ay=p[7], az=p[8], step1_x=p[0], step1_y=p[1], step1_z=p[2],
                       step1_vx=p[3], step1_vy=p[4], step1_vz=p[5], max_dv=dv, max_dx=dx)
        t += dt
    p = r.particles()
    out.update(final_x=p[0], final_y=p[1], final_z=p[2], final_vx=p[3], final_vy=p[4], final_vz=p[5])
    r.close()
    return out


def main():
    for name, spec in CASES.items():
        out = run_case(name, spec)
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **out)
        print(f"{path}: N={len(out['x'])} cells={out['m']} (nc={out['nc']}, nv={out['nv']}) its={out['its']}")


if __name__ == "__main__":
    main()
