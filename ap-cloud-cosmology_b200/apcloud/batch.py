"""Batched boxes: many independent boxes stepped together on one GPU.

Each box keeps the Controller sequence of controller.cpp:88-208 (initial select and
half drift, then select / solve / kick / drift per step) with its own constants; the
steps of all boxes go through one apc_batch_step call, which runs them concurrently
(one context and stream per box, host worker threads taking boxes largest first).
"""
from __future__ import annotations

import json
import os

from . import binding, ics
from .controller import Controller

TUNED_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuned_b200.json")


def load_tuned(path: str = TUNED_PATH) -> dict | None:
    """The autotuner's table {n_particles: make_config keywords}, if one was saved."""
    try:
        with open(path) as f:
            return {int(k): v for k, v in json.load(f).items()}
    except OSError:
        return None


class BatchRun:
    """A set of RunConfigs stepped together through binding.BatchPath."""

    def __init__(self, cfgs, precision: int = binding.APC_PREC_MIXED, n_workers: int = 0, tuned=None,
                 solve_mode: int = binding.APC_BATCH_SOLVE_PER_BOX, **kw):
        """tuned: optional {n_particles: dict of make_config keywords} from autotune();
        solve_mode: per-box solves, or one queued launch per solve phase for all boxes."""
        self.cfgs = list(cfgs)
        boxes = []
        for c in self.cfgs:
            opts = dict(depth=c.depth, gfd_c=c.gfd_c, lm=c.lm, restart=c.restart, rtol=c.rtol, precision=precision)
            opts.update(kw)
            if tuned and c.n in tuned:
                opts.update(tuned[c.n])
            boxes.append((c.particles(), opts))
        self.path = binding.BatchPath(boxes, n_workers=n_workers, solve_mode=solve_mode)
        self.ctl = [Controller(g, c.n, c.omega0, c.omegal, c.a_start, c.a_end, c.delta_a)
                    for g, c in zip(self.path.boxes, self.cfgs)]

    def start(self):
        for c in self.ctl:
            c.start()

    def done(self) -> bool:
        return all(c.done() for c in self.ctl)

    def params(self):
        out = []
        for c in self.ctl:
            dt = min(c.delta_a, c.end_a - c.t)
            k = c.constants(c.t, dt)
            out.append((dt, k["c_dens"], k["c_pot"], k["c_field"], k["c_vel"], k["c_pos"]))
        return out

    def step(self):
        p = self.params()
        self.path.step(p)
        for c, q in zip(self.ctl, p):
            c.t += q[0]

    def close(self):
        self.path.close()


def autotune(sides=ics.BATCH_SIDES, restarts=(8, 12, 16, 24), sweeps=(1, 2, 3), steps: int = 3,
             seed: int = 7) -> dict:
    """Pick, per box size, the inner restart and the V-cycle sweep count that give the
    fastest mixed step: each candidate runs `steps` steps of one Zel'dovich box of that
    size and is timed by the library's device events (the first step is discarded).
    Returns {n_particles: {"mixed_restart": m, "mg_sweeps": s}}."""
    best = {}
    for side in sides:
        cfg = ics.RunConfig(name=f"tune{side}", kind="zeldovich", n=side ** 3, depth=21,
                            gfd_c=1.28 * 8.0 ** (5.0 / 3.0) * side ** -2.0, omega0=1.0, omegal=0.0,
                            a_start=0.05, a_end=0.5, steps=32, seed=seed, spectral_index=-2.0, rms_spacing=0.2)
        parts = cfg.particles()
        cand = []
        for m in restarts:
            for sw in sweeps:
                g = binding.GpuPath(parts, cfg.depth, cfg.gfd_c, cfg.lm, precision=binding.APC_PREC_MIXED,
                                    mixed_restart=m, mg_sweeps=sw)
                ctl = Controller(g, cfg.n, cfg.omega0, cfg.omegal, cfg.a_start, cfg.a_end, cfg.delta_a)
                ctl.start()
                ctl.step()
                g.reset_profile()
                for _ in range(steps):
                    ctl.step()
                cand.append((g.profile()["step_ms"], m, sw))
                g.close()
        t, m, sw = min(cand)
        best[cfg.n] = {"mixed_restart": m, "mg_sweeps": sw}
    return best


def main():
    """python -m apcloud.batch --autotune [--out PATH]: time the candidates on this GPU
    and save the table that BatchRun and bench.py's batch96 workload load."""
    import argparse

    ap = argparse.ArgumentParser()
    ap.add_argument("--autotune", action="store_true")
    ap.add_argument("--out", default=TUNED_PATH)
    args = ap.parse_args()
    if args.autotune:
        table = autotune()
        with open(args.out, "w") as f:
            json.dump({str(k): v for k, v in table.items()}, f, indent=1)
        print(json.dumps(table))


if __name__ == "__main__":
    main()
