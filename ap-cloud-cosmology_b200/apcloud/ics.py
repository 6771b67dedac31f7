"""Seeded synthetic initial conditions for the gravity-step workloads.

The reference reads its initial conditions from legacy-VTK files produced elsewhere
(initialization.cpp:4-101; the IC files named in ball.param:15 / parameter.param:15
are not part of the reference).  These generators make seeded particle sets with the
shapes and distributions of the benchmark configurations instead:

* ``uniform_ball``: equal-mass particles uniform in a sphere, at rest (cold collapse).
* ``zeldovich``: a cubic lattice displaced by the Zel'dovich approximation from a
  Gaussian random field with a power-law spectrum P(k) ~ k^n and a Gaussian cutoff
  at half the Nyquist wavenumber, normalised to a given rms displacement (in lattice
  spacings) at the start time, with growing-mode momenta.

Units follow the equations in the reference README (README.md:28-34):
dp/da = -F(a) grad(phi), dx/da = F(a) p / a^2, F(a) = (Omega0/a + OmegaL a^2)^(-1/2),
laplacian(phi) = 3 Omega0 / (2a) (rho - 1); the box is [0,1]^3 and rho is in units of
the mean.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


@dataclass
class Particles:
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    vx: np.ndarray
    vy: np.ndarray
    vz: np.ndarray

    @property
    def n(self) -> int:
        return int(self.x.shape[0])

    def copy(self) -> "Particles":
        return Particles(*(a.copy() for a in (self.x, self.y, self.z, self.vx, self.vy, self.vz)))

    def as_tuple(self):
        return (self.x, self.y, self.z, self.vx, self.vy, self.vz)


def uniform_ball(n: int, radius: float = 0.25, center=(0.5, 0.5, 0.5), seed: int = 0) -> Particles:
    """n points uniform in a sphere, zero velocity."""
    rng = np.random.default_rng(seed)
    d = rng.standard_normal((n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = radius * rng.random(n) ** (1.0 / 3.0)
    p = d * r[:, None] + np.asarray(center, dtype=np.float64)[None, :]
    z = np.zeros(n)
    return Particles(p[:, 0].copy(), p[:, 1].copy(), p[:, 2].copy(), z.copy(), z.copy(), z.copy())


def hubble(a: float, omega0: float, omegal: float) -> float:
    return math.sqrt(omega0 / a ** 3 + omegal)


def growth(a: float, omega0: float, omegal: float) -> tuple[float, float]:
    """Linear growth D(a) (unnormalised) and dD/da for a flat background.

    D = H(a) * int_0^a da' / (a' H(a'))^3 ; dD/da = H'(a) I + 1 / (a^3 H^2).
    """
    from scipy.integrate import quad

    integral, _ = quad(lambda s: (s * hubble(s, omega0, omegal)) ** -3.0, 0.0, a, limit=200)
    h = hubble(a, omega0, omegal)
    dh = -1.5 * omega0 / a ** 4 / h
    return h * integral, dh * integral + 1.0 / (a ** 3 * h * h)


def kick_factor(a: float, omega0: float, omegal: float) -> float:
    """F(a) = (Omega0/a + OmegaL a^2)^(-1/2): dp/da = -F grad(phi) (README.md:30)."""
    return 1.0 / math.sqrt(omega0 / a + omegal * a * a)


def drift_factor(a: float, omega0: float, omegal: float) -> float:
    """F(a)/a^2: dx/da = F p / a^2 (README.md:30)."""
    return kick_factor(a, omega0, omegal) / (a * a)


def zeldovich_field(n_side: int, spectral_index: float, rms_spacing: float, a_start: float,
                    omega0: float, omegal: float, seed: int = 0):
    """The Zel'dovich displacement field psi (3, n, n, n), in box units at a_start, and the
    growing-mode factor fac with momenta p = fac psi."""
    rng = np.random.default_rng(seed)
    n = n_side
    white = rng.standard_normal((n, n, n))
    wk = np.fft.rfftn(white)
    kx = 2.0 * np.pi * np.fft.fftfreq(n, d=1.0 / n)
    kz = 2.0 * np.pi * np.fft.rfftfreq(n, d=1.0 / n)
    KX, KY, KZ = np.meshgrid(kx, kx, kz, indexing="ij")
    k2 = KX ** 2 + KY ** 2 + KZ ** 2
    k = np.sqrt(k2)
    k_nyq = np.pi * n
    kc = 0.5 * k_nyq
    with np.errstate(divide="ignore", invalid="ignore"):
        amp = np.where(k > 0, k ** (0.5 * spectral_index) * np.exp(-0.5 * (k / kc) ** 2), 0.0)
        dk = wk * amp
        inv = np.where(k2 > 0, 1.0 / k2, 0.0)
    # psi_k = i k / k^2 delta_k  (delta = -div psi)
    psi = [np.fft.irfftn(1j * K * inv * dk, s=(n, n, n), axes=(0, 1, 2)) for K in (KX, KY, KZ)]
    rms = math.sqrt(float(np.mean(psi[0] ** 2 + psi[1] ** 2 + psi[2] ** 2)))
    scale = rms_spacing / n / rms
    psi = np.stack([p * scale for p in psi])
    d, dd = growth(a_start, omega0, omegal)
    # p = a^2 dx/da / F(a),  dx/da = (D'/D) psi
    fac = a_start * a_start * (dd / d) / kick_factor(a_start, omega0, omegal)
    return psi, fac


def particles_from_field(psi, fac: float) -> Particles:
    """Lattice q = (i + 1/2)/n displaced by psi (3, n, n, n), wrapped into [0, 1)."""
    n = psi.shape[1]
    psi = np.asarray(psi, dtype=np.float64)
    q = (np.arange(n, dtype=np.float64) + 0.5) / n
    QX, QY, QZ = np.meshgrid(q, q, q, indexing="ij")
    pos = [np.mod(Q + P, 1.0).ravel() for Q, P in zip((QX, QY, QZ), psi)]
    for p in pos:
        p[p >= 1.0] -= 1.0
    vel = [(fac * P).ravel() for P in psi]
    return Particles(pos[0], pos[1], pos[2], vel[0], vel[1], vel[2])


def zeldovich(n_side: int, spectral_index: float, rms_spacing: float, a_start: float,
              omega0: float, omegal: float, seed: int = 0) -> Particles:
    """Lattice + Zel'dovich displacement with growing-mode momenta."""
    psi, fac = zeldovich_field(n_side, spectral_index, rms_spacing, a_start, omega0, omegal, seed)
    return particles_from_field(psi, fac)


@dataclass
class RunConfig:
    """One workload: particle set recipe + method parameters + time integration."""
    name: str
    kind: str  # "ball" | "zeldovich"
    n: int
    depth: int
    gfd_c: float
    omega0: float
    omegal: float
    a_start: float
    a_end: float
    steps: int
    lm: int = 17
    restart: int = 30
    rtol: float = 1e-10
    seed: int = 0
    radius: float = 0.25
    spectral_index: float = -2.0
    rms_spacing: float = 0.2

    @property
    def delta_a(self) -> float:
        return (self.a_end - self.a_start) / self.steps

    def particles(self) -> Particles:
        if self.kind == "ball":
            return uniform_ball(self.n, self.radius, seed=self.seed)
        n_side = round(self.n ** (1.0 / 3.0))
        assert n_side ** 3 == self.n
        return zeldovich(n_side, self.spectral_index, self.rms_spacing, self.a_start,
                         self.omega0, self.omegal, seed=self.seed)


def config(name: str, **over) -> RunConfig:
    """Named workloads.  gfd_c maps a target particles-per-cell to the refinement
    constant of octree.cpp:1176-1183 (n h^2 > c): c = cap^(5/3) rho^(-2/3)."""
    base = {
        # cold uniform-ball collapse, N = 32,768, a 0.1 -> 0.3 in 20 steps
        "ball32k": dict(kind="ball", n=32768, depth=21, gfd_c=5.08e-3, omega0=1.0, omegal=0.0,
                        a_start=0.1, a_end=0.3, steps=20, radius=0.25),
        # Einstein-de Sitter Zel'dovich box, 64^3, P ~ k^-2, rms 0.2 spacing at a = 0.02
        "eds64": dict(kind="zeldovich", n=64 ** 3, depth=21, gfd_c=1.0e-2, omega0=1.0, omegal=0.0,
                      a_start=0.02, a_end=1.0, steps=64, spectral_index=-2.0, rms_spacing=0.2),
        # LambdaCDM Zel'dovich box, 128^3, P ~ k^-1.5, rms 0.3 spacing at a = 0.02
        "lcdm128": dict(kind="zeldovich", n=128 ** 3, depth=21, gfd_c=6.2e-3, omega0=0.3, omegal=0.7,
                        a_start=0.02, a_end=1.0, steps=128, spectral_index=-1.5, rms_spacing=0.3),
    }[name]
    base.update(over)
    return RunConfig(name=name, **base)


# ---------------------------------------------------------------- batched boxes

BATCH_SIDES = (16, 24, 32, 48, 64)


def batch_boxes(n_boxes: int = 96, seed: int = 2024, a_start: float = 0.05, a_end: float = 0.5,
                steps: int = 32, sides=BATCH_SIDES) -> list:
    """Independent periodic EdS boxes of uneven size, each with its own seed.

    Particle counts are drawn uniformly from sides^3.  Even-numbered boxes are cold
    uniform-ball collapses (radius uniform in [0.15, 0.35], zero velocity); odd ones
    are Zel'dovich lattices with P(k) ~ k^-2 and rms displacement uniform in [0.1, 0.3]
    spacings at a_start.  Refinement constants follow c = cap^(5/3) rho^(-2/3) with a
    cap of 8 particles per cell (rho the mean density inside the ball, or N for a
    lattice box, scaled by 1.28 as for the 64^3 box)."""
    rng = np.random.default_rng(seed)
    out = []
    for b in range(n_boxes):
        side = int(rng.choice(sides))
        n = side ** 3
        box_seed = int(rng.integers(1, 2 ** 31 - 1))
        if b % 2 == 0:
            radius = float(rng.uniform(0.15, 0.35))
            rho = n / (4.0 / 3.0 * math.pi * radius ** 3)
            out.append(RunConfig(name=f"box{b}-ball{side}", kind="ball", n=n, depth=21,
                                 gfd_c=8.0 ** (5.0 / 3.0) * rho ** (-2.0 / 3.0), omega0=1.0, omegal=0.0,
                                 a_start=a_start, a_end=a_end, steps=steps, seed=box_seed, radius=radius))
        else:
            rms = float(rng.uniform(0.1, 0.3))
            out.append(RunConfig(name=f"box{b}-zel{side}", kind="zeldovich", n=n, depth=21,
                                 gfd_c=1.28 * 8.0 ** (5.0 / 3.0) * n ** (-2.0 / 3.0), omega0=1.0, omegal=0.0,
                                 a_start=a_start, a_end=a_end, steps=steps, seed=box_seed,
                                 spectral_index=-2.0, rms_spacing=rms))
    return out


def lpt_partition(costs, parts: int) -> list:
    """Longest-processing-time assignment of items to `parts` bins: items by decreasing
    cost (ties by index), each to the currently lightest bin (ties by bin index).
    Deterministic, so every rank computes the same assignment."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * parts
    bins = [[] for _ in range(parts)]
    for i in order:
        k = min(range(parts), key=lambda j: (load[j], j))
        bins[k].append(i)
        load[k] += costs[i]
    return [sorted(b) for b in bins]
