"""The step sequence of Controller::solve (controller.cpp:54-241) over any backend that
has the phase calls select / solve / move_velocity / move_position.

The reference's call sequence is kept:
  - an initial select and a half drift;
  - per step: select, solve, kick(t), drift(t + dt/2), t += dt, with dt clipped to end_a;
  - adaptive time stepping (ADAPTIVE_TIME_STEP, apcloud_macro.h:25-27) off unless asked
    for, and viewer output off.
The constants follow the equations of the reference README (README.md:28-34):
  - drift F(a)/a^2 and kick F(a), F(a) = (Omega0/a + OmegaL a^2)^(-1/2);
  - C_pot = 3 Omega0 / (2a) and C_field = -1;
  - C_dens = V/N, so that rho is in units of the mean density.
"""
from __future__ import annotations

from dataclasses import dataclass, field

from . import ics


@dataclass
class StepLog:
    t: float
    dt: float
    n_cells: int
    max_dv: float
    max_dx: float


@dataclass
class Controller:
    backend: object
    n: int
    omega0: float
    omegal: float
    start_a: float
    end_a: float
    delta_a: float
    box_volume: float = 1.0
    adaptive: bool = False  # ADAPTIVE_TIME_STEP (controller.cpp:146-164)
    output_dir: str | None = None  # VTK snapshots (viewer.cpp) every write_interval steps
    write_interval: int = 0
    fused: bool = True  # use the backend's whole-step call when it has one (fixed dt)
    t: float = field(init=False)
    log: list = field(default_factory=list)

    def __post_init__(self):
        self.t = self.start_a

    def constants(self, t: float, dt: float) -> dict:
        return dict(c_dens=self.box_volume / self.n, c_pot=1.5 * self.omega0 / t, c_field=-1.0,
                    c_vel=ics.kick_factor(t, self.omega0, self.omegal),
                    c_pos=ics.drift_factor(t + dt / 2, self.omega0, self.omegal))

    def start(self) -> None:
        """controller.cpp:88-111: select, then drift half a step with C_pos(start)."""
        self.backend.select()
        self.backend.move_position(0.5 * self.delta_a, ics.drift_factor(self.t, self.omega0, self.omegal))
        self.t += 0.5 * self.delta_a

    def done(self) -> bool:
        return not (self.t < self.end_a)

    def step(self) -> StepLog:
        """One pass of controller.cpp:133-208: select, the step size (adaptive: from the
        densest cell, controller.cpp:146-164), solve, kick, drift.  With an output
        directory, snapshots are written first every write_interval steps
        (controller.cpp:136-146)."""
        if self.output_dir and self.write_interval > 0 and len(self.log) % self.write_interval == 0:
            self.snapshot()
        if not self.adaptive and self.fused and hasattr(self.backend, "step"):
            # the whole step in one library call, kick and drift fused (apc_step)
            dt = self.delta_a
            if self.t + dt > self.end_a:
                dt = self.end_a - self.t
            k = self.constants(self.t, dt)
            m, dv, dx = self.backend.step(dt, k["c_dens"], k["c_pot"], k["c_field"], k["c_vel"], k["c_pos"])
            rec = StepLog(self.t, dt, m, dv, dx)
            self.log.append(rec)
            self.t += dt
            return rec
        m = self.backend.select()
        dt = self.backend.adaptive_dt(self.delta_a) if self.adaptive else self.delta_a
        if self.t + dt > self.end_a:
            dt = self.end_a - self.t
        k = self.constants(self.t, dt)
        self.backend.solve(k["c_dens"], k["c_pot"], k["c_field"])
        dv = self.backend.move_velocity(dt, k["c_vel"])
        dx = self.backend.move_position(dt, k["c_pos"])
        rec = StepLog(self.t, dt, m, dv, dx)
        self.log.append(rec)
        self.t += dt
        return rec


    def snapshot(self) -> None:
        """physical_<t>.vtk, and computational_<t>.vtk once a solve has run (viewer.cpp)."""
        from . import vtk

        p = self.backend.particles()
        vtk.write_physical(self.output_dir, self.t, *p[:9])
        if self.log:
            vtk.write_computational(self.output_dir, self.t, self.backend.cells(), self.backend.fields())


def for_config(backend, cfg: "ics.RunConfig", adaptive: bool = False) -> Controller:
    return Controller(backend, cfg.n, cfg.omega0, cfg.omegal, cfg.a_start, cfg.a_end, cfg.delta_a,
                      adaptive=adaptive)
