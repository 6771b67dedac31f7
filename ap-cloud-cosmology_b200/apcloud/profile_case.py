"""A short, fixed workload for kernel profiling under ncu.

    python -m apcloud.profile_case [--max-it N] [--precision fp64|mixed] [--workload lcdm128]

Runs one Controller step of the named workload with the GMRES iteration cap lowered to
--max-it, so that each GMRES launch is short enough for a multi-pass ncu capture.  The
density solve is the first GMRES launch of the step and the potential solve the second.
"""
from __future__ import annotations

import argparse
import time

from . import binding, ics
from .controller import for_config


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--max-it", type=int, default=200)
    ap.add_argument("--precision", choices=("fp64", "mixed"), default="fp64")
    ap.add_argument("--workload", default="lcdm128")
    args = ap.parse_args()
    cfg = ics.config(args.workload)
    prec = binding.APC_PREC_FP64 if args.precision == "fp64" else binding.APC_PREC_MIXED
    g = binding.GpuPath(cfg.particles(), cfg.depth, cfg.gfd_c, cfg.lm, precision=prec, max_it=args.max_it)
    ctl = for_config(g, cfg)
    ctl.start()
    g.reset_profile()
    t0 = time.perf_counter()
    rec = ctl.step()
    dt = time.perf_counter() - t0
    pr = g.profile()
    print(f"cells {rec.n_cells} wall {dt * 1e3:.1f} ms  krylov {pr['krylov_ms']:.2f} ms over {pr['krylov_launches']} "
          f"launches, {pr['krylov_iterations']} iterations, {pr['krylov_bytes'] / 1e9:.3f} GB algorithmic; "
          f"stats {g.solve_stats()}")
    print("profile", {k: (round(v, 3) if isinstance(v, float) else v) for k, v in pr.items()})
    g.close()


if __name__ == "__main__":
    main()
