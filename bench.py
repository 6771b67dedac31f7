#!/usr/bin/env python
"""Benchmark: particle-steps/s of the AP-Cloud gravity step on one or more B200s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (default): the 128^3 LambdaCDM Zel'dovich box.
  - 2,097,152 particles, P(k) ~ k^-1.5, rms displacement 0.3 lattice spacings at
    a = 0.02; Omega0 = 0.3, OmegaL = 0.7;
  - 128 leapfrog steps to a = 1, depth 21, c = 6.2e-3, lm = 17;
  - GMRES(30), rtol 1e-10, max_it 10000.
A step is one pass of the Controller sequence (select; solve; kick; drift) over the
whole particle set.  The timed arm is a mixed-precision path (--precision):
  - vcycle32 (default): FP64 FGMRES with FP64 Krylov vectors, right-preconditioned by an
    FP32 octree-multigrid V-cycle (APC_PREC_MIXED_VCYCLE);
  - mixed: FP32 FGMRES corrections inside FP64 iterative refinement (APC_PREC_MIXED).
GFD moments and the leapfrog are FP64 in both.  The plain FP64 GPU path (the same
multigrid FGMRES solver with FP64 vectors, operators and V-cycle) is timed beside it from
the same state.  Every arm's force error is measured against one FP64 solve converged to
rtol 1e-13, together with that of the reference-semantics FP64 GMRES(30)+Jacobi, which at
this size stops at max_it.  `full_run` times the whole configured run (every step to
a = 1) on a fresh context.

Timing: W warm-up steps, then K steps.
  - Each step is timed on the device with the library's CUDA events, on its own stream.
  - L2 is flushed (a 512 MiB write) before each timed step.
  - Ranks run independent replicas; the time is the max over ranks.
  - `e2e` repeats K steps through the public API from pinned host buffers (particles
    copied in, step, particles and accelerations copied out) and times them on the host.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

# 32 hardware work queues instead of CUDA's default 8, read when the CUDA context is
# created: the batched workload keeps one stream per box in flight, and with 8 queues
# streams share queues and wait on one another's kernels.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "ap-cloud-cosmology_b200")
sys.path.insert(0, PKG)

import numpy as np  # noqa: E402

from apcloud import binding as _b, ics  # noqa: E402

METRIC = "particle-steps/s at 128^3: mixed-prec vs FP64 GPU path at equal force error"
UNIT = "particle-steps/s"
WORKLOAD = "lcdm128"
# the timed arm's choices: (apc_precision, solver, arithmetic types)
PRECISIONS = {
    "vcycle32": (_b.APC_PREC_MIXED_VCYCLE, "FP64 FGMRES(16) with FP64 Krylov vectors, right-preconditioned by an "
                 "FP32 octree-multigrid V-cycle; density by FP32 GMRES(16) corrections in FP64 refinement",
                 "f64 Krylov / f32 multigrid V-cycle; f64 GFD moments and leapfrog"),
    "mixed": (_b.APC_PREC_MIXED, "FP64 iterative refinement around FP32 FGMRES(16) corrections with the FP32 "
              "V-cycle; density by FP32 GMRES(16) corrections",
              "f32 Krylov / f64 refinement, GFD moments and leapfrog"),
}


def workload_desc(cfg) -> str:
    return (f"{cfg.name}: {round(cfg.n ** (1 / 3))}^3={cfg.n} particles, LambdaCDM Zel'dovich "
            f"(Omega0={cfg.omega0}, OmegaL={cfg.omegal}, P(k)~k^{cfg.spectral_index}, rms {cfg.rms_spacing} "
            f"spacing at a={cfg.a_start}), {cfg.steps} steps to a={cfg.a_end}, depth {cfg.depth}, "
            f"c={cfg.gfd_c}, lm={cfg.lm}, GMRES({cfg.restart}) rtol {cfg.rtol}")


# ------------------------------------------------------------------ helpers

def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class Dist:
    """Rank plumbing: NCCL on GPUs for the bench, gloo on CPU for the tests.  Only
    barriers and a max over ranks cross ranks; the step itself has no collective."""

    def __init__(self, device: int, backend: str = "nccl"):
        self.ws, self.rank, self.local = dist_env()
        self.pg = None
        self.dev = "cuda" if backend == "nccl" else "cpu"
        if self.ws > 1:
            import datetime

            import torch
            import torch.distributed as td

            if backend == "nccl":
                torch.cuda.set_device(device)
            td.init_process_group(backend, timeout=datetime.timedelta(seconds=900 if backend == "nccl" else 60))
            self.pg = td

    def barrier(self):
        if self.pg:
            import torch

            t = torch.zeros(1, device=self.dev)
            self.pg.all_reduce(t)
            if self.dev == "cuda":
                torch.cuda.synchronize()

    def max(self, v: float) -> float:
        if not self.pg:
            return v
        import torch

        t = torch.tensor([v], dtype=torch.float64, device=self.dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def sum(self, v: float) -> float:
        if not self.pg:
            return v
        import torch

        t = torch.tensor([v], dtype=torch.float64, device=self.dev)
        self.pg.all_reduce(t)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled during the timed region.

    NVML is polled every 5 ms from a thread, so that a region of a few hundred ms still gets
    dozens of samples; the device is found by its PCI bus id (CUDA and NVML may number GPUs
    differently).  Without NVML, nvidia-smi is run at its 200 ms minimum.  Only reads."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, device: int, period_s: float = 0.005):
        self.device = device
        self.period = period_s
        self.proc = None
        self.nvml = None
        self.stop = threading.Event()
        self.samples: list[tuple[float, float, set]] = []
        self.lines: list[str] = []

    def _nvml_handle(self):
        import pynvml
        import torch

        pynvml.nvmlInit()
        try:
            pr = torch.cuda.get_device_properties(self.device)
            bus = "%08X:%02X:%02X.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.device)

    def __enter__(self):
        try:
            nv, h = self._nvml_handle()
            self.nvml = (nv, h, nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self.bits = [nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                         nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap]
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.device)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _poll(self):
        nv, h, mx = self.nvml
        while not self.stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append((float(sm), float(mx), {n for n, b in zip(self.NAMES, self.bits) if r & b}))
            except Exception:
                return
            self.stop.wait(self.period)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        self.stop.set()
        if self.nvml:
            self.thread.join(timeout=5)
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], 0.0, set()
        for f, m, r in self.samples:
            sm.append(f)
            mx = max(mx, m)
            reasons |= r
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for k, nm in enumerate(self.NAMES):
                if parts[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm),
                "source": "nvml 5 ms" if self.samples else "nvidia-smi 200 ms"}


def measured_peaks() -> tuple[float, str]:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# Algorithmic bytes of the GFD kernel per cell: gather of 17 neighbours (position +
# index, 17 x (24 + 4) = 476), two matrix rows of 18 entries (value + column,
# 2 x 18 x 12 = 432), one rhs value (8).
GFD_BYTES_PER_CELL = 476 + 432 + 8


def step_algorithmic_bytes(n: int, cells: int, potential_bytes: float, density_its: float) -> float:
    """Bytes a step must move: 160 per particle (keys, sort, interpolation, kick, drift),
    1.2 KB per cell (selection, GFD, differentiation), the potential solve's bytes from the
    library's model (apc_profile.mg_bytes: Krylov passes, every V-cycle level, refinement),
    and per FP64 density iteration per row an 18-wide SpMV (18 x 12), and the dots and
    Gram-Schmidt update over a mean basis of 5 (15 x 8): 336 B."""
    return 160.0 * n + 1200.0 * cells + potential_bytes + 336.0 * cells * density_its


def ncu_traffic_per_unit(kernel: str) -> float | None:
    """DRAM bytes per unit of `kernel` from the committed ncu summary, if present: per cell
    for the GFD assembly, per algorithmic byte for the solve."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    try:
        for ln in open(path):
            ln = ln.strip()
            if ln.startswith(kernel + ":"):
                return float(ln.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


def batch_shard(cfgs, ws: int, rank: int) -> list:
    """The boxes of `rank`: longest-processing-time partition by particle-steps, the
    same on every rank, so the ranks share no data and need no collective."""
    return ics.lpt_partition([c.n * c.steps for c in cfgs], ws)[rank]


# ------------------------------------------------------------------ our arm

def run_ours(args) -> dict:
    import torch

    from apcloud import binding
    from apcloud.controller import for_config

    ws, rank, local = dist_env()
    dev = local
    torch.cuda.set_device(dev)
    dist = Dist(dev)
    cfg = ics.config(args.workload)
    parts = cfg.particles()
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def make(prec, p):
        return binding.GpuPath(p, cfg.depth, cfg.gfd_c, cfg.lm, restart=cfg.restart, rtol=cfg.rtol,
                               precision=prec, device=dev, mixed_restart=args.mixed_restart,
                               mixed_inner_rtol=args.inner_rtol, solve_graphs=0 if args.persistent else 1)

    head_prec = PRECISIONS[args.precision][0]
    # ---- warm-up on the timed path ----
    mx = make(head_prec, parts)
    ctl = for_config(mx, cfg)
    ctl.start()
    for _ in range(args.warmup):
        ctl.step()
    state = mx.particles()
    state_parts = ics.Particles(*state[:6])
    t_state = ctl.t

    # ---- force error on the same state.  Arms: both mixed paths (one of them the timed
    #      headline), the plain FP64 GPU path (the same multigrid FGMRES solver with every
    #      vector and operator in FP64), and the reference-semantics FP64 GMRES(30)+Jacobi, all
    #      to rtol 1e-10.  Each is measured against one independent FP64 solve converged to
    #      rtol 1e-13 ----
    arms = (("mixed_vcycle", binding.APC_PREC_MIXED_VCYCLE, cfg.rtol), ("mixed", binding.APC_PREC_MIXED, cfg.rtol),
            ("fp64", binding.APC_PREC_FP64_MULTIGRID, cfg.rtol), ("fp64_gmres", binding.APC_PREC_FP64, cfg.rtol),
            ("converged", binding.APC_PREC_FP64_MULTIGRID, 1e-13))
    acc = {}
    for name, prec, rtol in arms:
        g = binding.GpuPath(state_parts, cfg.depth, cfg.gfd_c, cfg.lm, restart=cfg.restart, rtol=rtol,
                            precision=prec, device=dev, mixed_restart=args.mixed_restart,
                            mixed_inner_rtol=args.inner_rtol, solve_graphs=0 if args.persistent else 1)
        c2 = for_config(g, cfg)
        c2.t = t_state
        k = c2.constants(c2.t, cfg.delta_a)
        g.select()
        g.solve(k["c_dens"], k["c_pot"], k["c_field"])
        g.move_velocity(cfg.delta_a, k["c_vel"])
        acc[name] = (np.stack(g.particles()[6:9]), g.solve_stats(), g.fields().potential)
        g.close()

    def rms(a, b):
        return float(np.sqrt(np.mean(np.sum((a - b) ** 2, 0)) / np.mean(np.sum(b ** 2, 0))))

    aref, pref = acc["converged"][0], acc["converged"][2]
    force = {name: {"acc_rms_vs_converged": rms(acc[name][0], aref),
                    "potential_rms_vs_converged": float(np.sqrt(np.mean((acc[name][2] - pref) ** 2) /
                                                                np.mean(pref ** 2))),
                    "potential_its": acc[name][1]["potential_its"],
                    "potential_reason": acc[name][1]["potential_reason"],
                    "potential_refinements": acc[name][1]["potential_refinements"]}
             for name in ("mixed_vcycle", "mixed", "fp64", "fp64_gmres")}

    def timed(g, c):
        dist.barrier()
        torch.cuda.synchronize()
        g.reset_profile()
        l0 = g.kernel_launches()
        with ClockSampler(dev) as clk:
            for _ in range(args.steps):
                flush.zero_()
                torch.cuda.synchronize()
                c.step()
        dist.barrier()
        pr = g.profile()
        return pr, g.kernel_launches() - l0, clk.summary()

    prof, launches, clocks = timed(mx, ctl)
    step_ms = dist.max(prof["step_ms"])
    value = ws * cfg.n * args.steps / (step_ms / 1e3)

    # ---- the whole configured run: a fresh context from the initial state through every
    #      step to a_end, each step timed on the device (no L2 flush: a real run) ----
    full = None
    if not args.no_full_run:
        gf = make(head_prec, parts)
        cf = for_config(gf, cfg)
        dist.barrier()
        t0 = time.perf_counter()
        cf.start()
        per = []
        while not cf.done():
            gf.reset_profile()
            cf.step()
            per.append(gf.profile()["step_ms"])
        wall = time.perf_counter() - t0
        gf.close()
        dev_s = dist.max(sum(per) / 1e3)
        wall = dist.max(wall)
        q = len(per) // 4
        full = {"steps": len(per), "a_end": round(cf.t, 6), "value": ws * cfg.n * len(per) / dev_s,
                "unit": UNIT, "seconds_device": dev_s, "seconds_wall": wall,
                "value_wall": ws * cfg.n * len(per) / wall,
                "ms_first_quarter": statistics.mean(per[:q]), "ms_last_quarter": statistics.mean(per[-q:]),
                "ms_max": max(per), "ms_min": min(per),
                "timing": "device events per step (select to drift), summed; seconds_wall = host clock around "
                          "the whole run incl. the initial select + half drift"}

    # ---- the plain FP64 GPU path over the same steps (the same initial state and warm-up
    #      steps, so that both arms' timed steps start from warm contexts), timed the same way ----
    fp64 = None
    if not args.no_fp64:
        g64 = make(binding.APC_PREC_FP64_MULTIGRID, parts)
        c64 = for_config(g64, cfg)
        c64.start()
        for _ in range(args.warmup):
            c64.step()
        p64, l64, clk64 = timed(g64, c64)
        fp64_ms = dist.max(p64["step_ms"])
        st64 = g64.solve_stats()
        g64.close()
        fv = ws * cfg.n * args.steps / (fp64_ms / 1e3)
        fp64 = {"value": fv, "ms_per_step": fp64_ms / args.steps, "speedup_timed_arm_over_fp64": value / fv,
                "solver": "FP64 multigrid FGMRES (APC_PREC_FP64_MULTIGRID): the mixed path's solver with FP64 "
                          "vectors and operators, restarted from the true FP64 residual, rtol 1e-10",
                "phases_ms_per_step": {k2: p64[k2 + "_ms"] / args.steps for k2 in
                                       ("select", "solve", "assemble", "gfd", "density", "potential", "move")},
                "potential_iterations_per_step": p64["mg_iterations"] / args.steps,
                "potential_reason": st64["potential_reason"], "gpu_launches": l64, "clocks": clk64}

    # ---- end to end through the public API with host buffers ----
    e2e = None
    if not args.no_e2e:
        pin = [torch.empty(cfg.n, dtype=torch.float64).pin_memory().numpy() for _ in range(9)]
        cur = mx.particles()
        for a, b in zip(pin[:6], cur[:6]):
            a[:] = b
        lib = mx.lib
        dist.barrier()
        tot = 0.0
        t = ctl.t
        per_step = []
        for _ in range(args.steps):
            k = ctl.constants(t, cfg.delta_a)
            t0 = time.perf_counter()
            mx._check(lib.apc_set_particles(mx.h, *[a.ctypes.data for a in pin[:6]]), "apc_set_particles")
            mx.step(cfg.delta_a, k["c_dens"], k["c_pot"], k["c_field"], k["c_vel"], k["c_pos"])
            mx._check(lib.apc_get_particles(mx.h, *[a.ctypes.data for a in pin]), "apc_get_particles")
            dt = time.perf_counter() - t0
            per_step.append(round(dt * 1e3, 2))
            tot += dt
            t += cfg.delta_a
        tot = dist.max(tot)
        e2e = {"value": ws * cfg.n * args.steps / tot, "unit": UNIT, "h2d_bytes_per_step": 6 * 8 * cfg.n,
               "d2h_bytes_per_step": 9 * 8 * cfg.n, "timing": "host wall clock per step, max over ranks",
               "ms_per_step": per_step}

    peak, peak_kind = measured_peaks()
    # ---- roofline of the dominant kernel: gfd_stencil, one launch per step over the M
    #      computational + vacuum cells (neighbour search, least squares, both matrix rows) ----
    nc, nv, _, _ = mx.counts()
    cells = nc + nv
    gfd_ms = prof["gfd_ms"] / args.steps
    gfd_bytes = GFD_BYTES_PER_CELL * cells
    gfd_achieved = gfd_bytes / (gfd_ms / 1e3) / 1e9 if gfd_ms > 0 else 0.0
    traffic_per_cell = ncu_traffic_per_unit("gfd")
    gfd_roof = {"kernel": "GFD assembly: gfd_search + gfd_lsq<false> + gfd_lsq<true> (neighbour search and "
                          "sort; Cholesky least squares, Householder for the cells it queues, X, A1/A2 rows), "
                          "one launch each per step, timed together",
                "bound": "hbm", "achieved": gfd_achieved, "peak": peak, "unit": "GB/s",
                "frac": gfd_achieved / peak, "peak_kind": peak_kind,
                "traffic": (traffic_per_cell * cells) if traffic_per_cell else None,
                "algorithmic_bytes_per_launch": gfd_bytes, "bytes_per_cell": GFD_BYTES_PER_CELL,
                "cells": cells, "ms_per_launch": gfd_ms,
                "note": "latency- and issue-bound (the exact per-cell neighbour search and sort, the FP64 "
                        "least squares); the HBM fraction is low by nature of the kernels"}
    # ---- roofline of the potential solve (one graph, or one persistent kernel, per step): its
    #      algorithmic bytes from the library's model (apc_profile.mg_bytes) over its CUDA-event
    #      time ----
    mg_ms = prof["mg_solve_ms"] / args.steps
    mg_bytes = prof["mg_bytes"] / args.steps
    mg_achieved = mg_bytes / (mg_ms / 1e3) / 1e9 if mg_ms > 0 else 0.0
    mg_traffic = ncu_traffic_per_unit("mg_solve")
    solve_roof = {"kernel": "potential solve: ir_solve_persistent (FP64 refinement, FGMRES(16) cycles, "
                            "octree-multigrid V-cycles; one cooperative launch per step)"
                            if args.persistent and args.precision == "mixed" else
                            "potential solve: one CUDA graph per step (" + PRECISIONS[args.precision][1] +
                            "; ~20 kernels per iteration), timed as a unit",
                  "bound": "hbm", "achieved": mg_achieved, "peak": peak, "unit": "GB/s",
                  "frac": mg_achieved / peak, "peak_kind": peak_kind,
                  "traffic": (mg_traffic * mg_bytes) if mg_traffic else None,
                  "algorithmic_bytes_per_launch": mg_bytes, "ms_per_launch": mg_ms,
                  "iterations_per_launch": prof["mg_iterations"] / args.steps,
                  "note": "the working set (~80 MB in FP32, ~130 MB with FP64 Krylov vectors at 128^3) stays "
                          "largely in the 126 MB L2 between phases; the peak is the HBM copy bandwidth"}
    roofs = sorted([gfd_roof, solve_roof], key=lambda r: -r["ms_per_launch"])
    # ---- whole-step algorithmic bytes (particles, cells, Krylov rows), for context ----
    st = mx.solve_stats()
    step_bytes = step_algorithmic_bytes(cfg.n, cells, mg_bytes, st["density_its"])
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": step_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": PRECISIONS[args.precision][2], "data": "synthetic",
        "config": {"workload": workload_desc(cfg), "precision": args.precision,
                   "solver": PRECISIONS[args.precision][1], "parallelism": f"replicas x{ws}",
                   "l2": "flushed (512 MiB write) before every timed step",
                   "start_a": round(t_state, 6),
                   "timed_steps": f"steps {args.warmup + 1}-{args.warmup + args.steps} of {cfg.steps} "
                                  f"(a = {t_state:.4f} onwards); the whole run is in full_run",
                   "mixed_restart": args.mixed_restart or 16,
                   "inner_rtol": args.inner_rtol or 1e-3,
                   "solve": "one persistent cooperative kernel per solve" if args.persistent else
                            "one CUDA graph of per-phase kernels per solve"},
        "fp64": fp64,
        "force_error": dict(force, bound=1e-6,
                            measure="RMS relative error of the accelerations (and potentials) of one step on the "
                                    "same state, against an FP64 multigrid solve converged to rtol 1e-13",
                            equal_force_error=bool(force["mixed_vcycle"]["acc_rms_vs_converged"] <= 1e-6 and
                                                   force["mixed"]["acc_rms_vs_converged"] <= 1e-6 and
                                                   force["fp64"]["acc_rms_vs_converged"] <= 1e-6)),
        "phases_ms_per_step": {k: prof[k + "_ms"] / args.steps for k in
                               ("select", "solve", "assemble", "gfd", "density", "potential", "mg_build",
                                "mg_solve", "move")},
        "solve": {"potential_its": st["potential_its"], "potential_refinements": st["potential_refinements"],
                  "potential_reason": st["potential_reason"], "density_its": st["density_its"],
                  "potential_iterations_per_step": prof["mg_iterations"] / args.steps},
        "roofline": dict(roofs[0], dominant="the kernel (set) with the longest device time per step"),
        "roofline_next": roofs[1],
        "step_roofline": {"algorithmic_bytes": step_bytes, "achieved_gbs": step_bytes / (step_ms / args.steps / 1e3) / 1e9,
                          "frac": step_bytes / (step_ms / args.steps / 1e3) / 1e9 / peak},
        "full_run": full,
        "gpu_launches": launches,
        "clocks": clocks,
        "e2e": e2e,
    }
    mx.close()
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(cfg, args)
    dist.close()
    return out if rank == 0 else None


# ------------------------------------------------------------- batched boxes

def run_batch(args) -> dict | None:
    """96 independent boxes (16^3..64^3 balls and Zel'dovich lattices), each rank taking
    a longest-processing-time share; every step of every box goes through one
    apc_batch_step call per rank.  Two forms of the step are timed from the same start:
    per-box (the headline: each box's step whole in its fiber, its solves its own CUDA
    graphs; results equal single contexts bit for bit) and queued (all boxes' density
    solves, then all potential solves, in one cooperative launch each, block groups pulling
    boxes from a device work queue).
    Timed on the host around whole batch steps, with the device synchronised on both
    sides (the boxes run on many streams); max over ranks."""
    import torch

    from apcloud import binding
    from apcloud.batch import BatchRun, load_tuned

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = Dist(local)
    cfgs = ics.batch_boxes()
    mine = [cfgs[i] for i in batch_shard(cfgs, ws, rank)]
    total = sum(c.n for c in cfgs)

    def timed(mode):
        # per box: FP64 FGMRES over the FP32 V-cycle (the fastest at equal force error); the
        # queued launches run the persistent solve body, built for the FP32-Krylov path
        prec = binding.APC_PREC_MIXED_VCYCLE if mode == binding.APC_BATCH_SOLVE_PER_BOX else binding.APC_PREC_MIXED
        br = BatchRun(mine, precision=prec, n_workers=args.batch_workers, tuned=load_tuned(), solve_mode=mode)
        br.start()
        for _ in range(args.warmup):
            br.step()
        for g in br.path.boxes:
            g.reset_profile()
        dist.barrier()
        torch.cuda.synchronize()
        per, solve = [], []
        t0 = time.perf_counter()
        for _ in range(args.steps):
            t1 = time.perf_counter()
            br.step()
            torch.cuda.synchronize()
            per.append(round(1e3 * (time.perf_counter() - t1), 2))
            solve.append(round(br.path.solve_ms(), 2))
        dt = time.perf_counter() - t0
        dist.barrier()
        dt = dist.max(dt)
        launches = sum(g.kernel_launches() for g in br.path.boxes)
        br.close()
        return dt, per, solve, launches

    dt_q, per_q, solve_q, launches_q = timed(binding.APC_BATCH_SOLVE_QUEUED)
    dt_b, per_b, _, launches_b = timed(binding.APC_BATCH_SOLVE_PER_BOX)
    value = total * args.steps / dt_b
    dist.close()
    if rank != 0:
        return None
    return {"metric": "particle-steps/s over 96 batched boxes (16^3..64^3, mixed precision)", "value": value,
            "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * dt_b / args.steps, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": PRECISIONS["vcycle32"][2],
            "data": "synthetic",
            "config": {"workload": f"batch96: {len(cfgs)} boxes, {total} particles, a 0.05->0.5 in 32 steps",
                       "solves": "per box: each box's solves its own CUDA graphs, boxes as fibers; "
                                 + PRECISIONS["vcycle32"][1],
                       "parallelism": f"boxes sharded over {ws} ranks by LPT; {args.batch_workers or 16} "
                                      f"host workers per rank",
                       "timing": "host clock around whole batch steps, device synchronised, max over ranks"},
            "ms_per_step_each": per_b,
            "queued": {"value": total * args.steps / dt_q, "ms_per_step": 1e3 * dt_q / args.steps,
                       "ms_per_step_each": per_q, "solve_launches_ms_each": solve_q, "gpu_launches": launches_q,
                       "solves": "one cooperative launch per solve phase for all boxes, block groups pulling "
                                 "boxes from a device work queue, largest first; " + PRECISIONS["mixed"][1]},
            "rank0": {"boxes": len(mine)},
            "gpu_launches": launches_b}


# ------------------------------------------------------------- CPU reference

# The reference's own run lines cap GMRES at 1000 iterations (-ksp_max_it 1000,
# Makefile:30-32).  At 128^3 GMRES(30)+Jacobi reaches neither 1000 nor 10000 iterations'
# worth of rtol 1e-10, and a 10000-iteration step (~20-110 s on the host) cannot be
# repeated K + W times within minutes, so the CPU arms run the reference's production cap.
REF_MAX_IT = 1000


def reference_threads() -> int:
    """All the host cores this process may use (OpenMP regions of the reference and the
    GMRES shim, which spreads its loops as PETSc spreads them over MPI ranks)."""
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


class ReferenceRun:
    """The reference's own code (oracle/_ref: octree.cpp, mover.cpp, particle.cpp,
    solver.cpp) driven through the Controller step sequence from the workload's initial
    state: select + half drift, then whole steps (select; solve; kick; drift), each timed
    in full on the host clock."""

    def __init__(self, cfg, threads: int):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import refbind  # test infrastructure: only the CPU arms of the bench load it

        from apcloud.controller import for_config

        self.r = refbind.CpuPath("ref", cfg.particles(), cfg.depth, cfg.gfd_c, cfg.lm)
        self.r.set_gmres(cfg.restart, cfg.rtol, 1e-50, 1e5, REF_MAX_IT)
        self.r.set_threads(threads)
        self.ctl = for_config(self.r, cfg)
        self.ctl.start()

    def step(self) -> tuple[float, list]:
        self.r.reset_solve_stats()
        t0 = time.perf_counter()
        self.ctl.step()
        dt = time.perf_counter() - t0
        return dt, [(s[0], s[2]) for s in self.r.solve_stats()]

    def close(self):
        self.r.close()


def ref_sample_text(cfg, threads: int, k: int, first_step: int, its) -> str:
    return (f"{k} whole 128^3 step(s) of the reference code (oracle/_ref), steps {first_step}-{first_step + k - 1} "
            f"of the run from its initial state: select, GFD assembly, density and potential GMRES({cfg.restart}) "
            f"rtol {cfg.rtol} capped at {REF_MAX_IT} iterations as in the reference's run lines (Makefile:30-32), "
            f"differentiation, kick, drift; each timed in full (no scaling); OpenMP regions and the GMRES loops on "
            f"{threads} host threads, selection and assembly serial as in the reference; (its, reason) of the "
            f"last step's solves {its}")


def cpu_baseline(cfg, args) -> dict:
    """The reference on the host, bounded: the first whole step of the run."""
    th = reference_threads()
    rr = ReferenceRun(cfg, th)
    sec, its = rr.step()
    rr.close()
    return {"value": cfg.n / sec, "unit": UNIT, "cores": th, "kind": "reference",
            "sample": ref_sample_text(cfg, th, 1, 1, its), "seconds_per_step": sec}


def run_reference(args) -> dict | None:
    ws, rank, _ = dist_env()
    if rank != 0:
        return None
    cfg = ics.config(args.workload)
    ref_so = os.path.join(ROOT, "oracle", "_ref", "libapcref.so")
    if not os.path.exists(ref_so):
        return {"impl": "reference", "unavailable": "oracle/_ref/libapcref.so not built (make -C oracle ref)"}
    th = reference_threads()
    rr = ReferenceRun(cfg, th)
    for _ in range(args.warmup):
        rr.step()
    secs = []
    its = None
    for _ in range(args.steps):
        sec, its = rr.step()
        secs.append(sec)
    rr.close()
    total = sum(secs)
    value = cfg.n * args.steps / total
    sample = ref_sample_text(cfg, th, args.steps, args.warmup + 1, its)
    return {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": workload_desc(cfg), "precision": "fp64 (reference CPU path)",
                       "gmres_max_it": REF_MAX_IT, "timed_steps": f"{args.warmup + 1}-{args.warmup + args.steps}",
                       "timing": "host clock around each whole step"},
            "impl": "reference",
            "seconds_per_step": [round(x, 3) for x in secs],
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": th, "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--workload", default=WORKLOAD)
    ap.add_argument("--precision", choices=tuple(PRECISIONS), default="vcycle32",
                    help="the timed arm's solver precision")
    ap.add_argument("--mixed-restart", type=int, default=0)
    ap.add_argument("--inner-rtol", type=float, default=0.0)
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-full-run", action="store_true")
    ap.add_argument("--persistent", action="store_true",
                    help="run the multigrid solves as one persistent cooperative kernel each instead of CUDA "
                         "graphs of per-phase kernels")
    ap.add_argument("--batch-workers", type=int, default=0, help="host worker threads per rank (batch96)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        out = run_reference(args)
    elif args.workload == "batch96":
        out = run_batch(args)
    else:
        out = run_ours(args)
    if out is not None:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
