"""The C5 workload's gradient against the FP64 CPU adjoint (a script, not collected by
pytest: minutes of host time at 64^3 x 32 steps).

    python tests/adjoint_c5_cpu_check.py [--side 64 --steps 32 --every 8] > c5.json

Runs apcloud.adjoint (the GPU trajectory VJP with its finite-difference check), then the
FP64 CPU adjoint of oracle/adjoint_ref.py on the oracle's forward trajectory from the same
initial displacement field, and adds the largest difference between the two gradients,
relative to the largest CPU gradient component, to the last JSON line."""
from __future__ import annotations

import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "ap-cloud-cosmology_b200"), os.path.join(ROOT, "oracle")):
    sys.path.insert(0, p)

import numpy as np  # noqa: E402

import adjoint_ref  # noqa: E402  (the FP64 CPU adjoint: the checker)
from apcloud import adjoint, ics  # noqa: E402


def main():
    out, grad, (psi32, fac, gfd_c, sched, target) = adjoint.main(sys.argv[1:])
    side = psi32.shape[-1]
    n = side ** 3
    t1 = time.perf_counter()
    parts = ics.particles_from_field(psi32.astype(np.float64), fac)
    xf, _ = adjoint_ref.forward_state(parts, 21, gfd_c, sched)
    d = adjoint.wrap(xf[:3] - target)
    cot = np.zeros((6, n))
    cot[:3] = 2.0 * d / n
    _, c0 = adjoint_ref.trajectory_vjp(parts, 21, gfd_c, sched, cot)
    gref = (c0[:3] + fac * c0[3:]).reshape(3, side, side, side)
    out["cpu_ref_seconds"] = time.perf_counter() - t1
    out["cpu_ref_max_rel_err"] = float(np.max(np.abs(gref - grad)) / np.max(np.abs(gref)))
    print(json.dumps(out))


if __name__ == "__main__":
    main()
