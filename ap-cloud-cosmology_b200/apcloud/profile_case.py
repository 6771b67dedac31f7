"""A short, fixed workload for kernel profiling under ncu.

    python -m apcloud.profile_case [--precision fp64|mixed|fp64mg|vcycle32] [--workload lcdm128]
                                   [--warm K] [--max-it N] [--persistent]

Runs K unprofiled Controller steps of the named workload, then one more step bracketed
by cudaProfilerStart / cudaProfilerStop, so that `ncu --profile-from-start off` sees
exactly one steady-state step.  --max-it lowers the GMRES iteration cap of the FP64
path, so that each of its GMRES launches is short enough for a multi-pass capture.
--persistent runs the multigrid solves as persistent kernels instead of CUDA graphs.
"""
from __future__ import annotations

import argparse
import ctypes
import time

from . import binding, ics
from .controller import for_config


def _cudart():
    for name in ("libcudart.so.12", "libcudart.so"):
        try:
            return ctypes.CDLL(name)
        except OSError:
            continue
    return None


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--max-it", type=int, default=10000)
    ap.add_argument("--precision", choices=("fp64", "mixed", "fp64mg", "vcycle32"), default="mixed")
    ap.add_argument("--persistent", action="store_true")
    ap.add_argument("--workload", default="lcdm128")
    ap.add_argument("--warm", type=int, default=2)
    args = ap.parse_args()
    cfg = ics.config(args.workload)
    prec = {"fp64": binding.APC_PREC_FP64, "mixed": binding.APC_PREC_MIXED,
            "fp64mg": binding.APC_PREC_FP64_MULTIGRID, "vcycle32": binding.APC_PREC_MIXED_VCYCLE}[args.precision]
    g = binding.GpuPath(cfg.particles(), cfg.depth, cfg.gfd_c, cfg.lm, precision=prec, max_it=args.max_it,
                        solve_graphs=0 if args.persistent else 1)
    ctl = for_config(g, cfg)
    ctl.start()
    for _ in range(args.warm):
        ctl.step()
    rt = _cudart()
    g.reset_profile()
    g.synchronize()
    if rt is not None:
        rt.cudaProfilerStart()
    t0 = time.perf_counter()
    rec = ctl.step()
    dt = time.perf_counter() - t0
    if rt is not None:
        rt.cudaProfilerStop()
    pr = g.profile()
    print(f"cells {rec.n_cells} wall {dt * 1e3:.1f} ms; stats {g.solve_stats()}")
    print("profile", {k: (round(v, 3) if isinstance(v, float) else v) for k, v in pr.items()})
    g.close()


if __name__ == "__main__":
    main()
