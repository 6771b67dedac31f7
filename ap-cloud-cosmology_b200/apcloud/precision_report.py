"""Errors of the mixed path against FP64 for each result: potential, acceleration and
final positions.

    python -m apcloud.precision_report [--steps 8]

eds64 (the 64^3 EdS box, where FP64 GMRES(30) reaches rtol 1e-10): both paths run the
same number of Controller steps from the same initial conditions; the last step's cell
potentials (the cell sets are compared first), the particles' accelerations and their
final positions are compared.  lcdm128 (the 128^3 LambdaCDM box, where FP64 GMRES(30)
stops at max_it): on the same state, the mixed solve and the FP64 solve are compared with
a solve converged to rtol 1e-13, and positions after the steps with the mixed path are
compared with positions from the converged solver.
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from . import binding, ics
from .controller import for_config


def _rms(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.sqrt(np.mean((a - b) ** 2) / np.mean(b ** 2)))


def _vec_rms(a, b):
    a, b = np.stack(a), np.stack(b)
    return float(np.sqrt(np.mean(np.sum((a - b) ** 2, 0)) / np.mean(np.sum(b ** 2, 0))))


def _pos_err(a, b, n_side):
    d = np.stack(a) - np.stack(b)
    d -= np.round(d)
    return float(np.sqrt(np.mean(np.sum(d * d, 0))) * n_side)  # in lattice spacings


def run(cfg_name: str, steps: int, ref_kw: dict, test_kw: dict) -> dict:
    cfg = ics.config(cfg_name)
    n_side = round(cfg.n ** (1 / 3))
    out = {}
    runs = {}
    for name, kw in (("ref", ref_kw), ("test", test_kw)):
        g = binding.GpuPath(cfg.particles(), cfg.depth, cfg.gfd_c, cfg.lm, restart=cfg.restart, **kw)
        c = for_config(g, cfg)
        c.start()
        for _ in range(steps):
            c.step()
        runs[name] = dict(codes=np.sort(g.codes()), phi=g.fields().potential, codes_raw=g.codes(),
                          p=g.particles(), stats=g.solve_stats(), a=c.t)
        g.close()
    r, t = runs["ref"], runs["test"]
    out["a"] = r["a"]
    out["same_cells"] = bool(np.array_equal(r["codes"], t["codes"]))
    if out["same_cells"]:
        # align the potentials by cell code
        ir, it = np.argsort(r["codes_raw"]), np.argsort(t["codes_raw"])
        out["potential_rms_rel"] = _rms(t["phi"][it], r["phi"][ir])
    out["acceleration_rms_rel"] = _vec_rms(t["p"][6:9], r["p"][6:9])
    out["position_rms_spacings"] = _pos_err(t["p"][:3], r["p"][:3], n_side)
    out["ref_potential"] = (r["stats"]["potential_its"], r["stats"]["potential_reason"])
    out["test_potential"] = (t["stats"]["potential_its"], t["stats"]["potential_reason"])
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=8)
    args = ap.parse_args()
    rep = {
        "eds64_mixed_vs_fp64": run("eds64", args.steps, dict(precision=binding.APC_PREC_FP64),
                                   dict(precision=binding.APC_PREC_MIXED)),
        "lcdm128_mixed_vs_converged": run("lcdm128", args.steps, dict(precision=binding.APC_PREC_MIXED, rtol=1e-13),
                                          dict(precision=binding.APC_PREC_MIXED)),
        "lcdm128_fp64_vs_converged": run("lcdm128", 2, dict(precision=binding.APC_PREC_MIXED, rtol=1e-13),
                                         dict(precision=binding.APC_PREC_FP64)),
    }
    print(json.dumps(rep))


if __name__ == "__main__":
    main()
