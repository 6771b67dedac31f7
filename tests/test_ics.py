"""CPU tests of the seeded initial-condition generators."""
from __future__ import annotations

import math

import numpy as np
import pytest

from apcloud import ics


def test_ball_is_seeded_uniform_and_inside():
    a = ics.uniform_ball(5000, radius=0.25, seed=4)
    b = ics.uniform_ball(5000, radius=0.25, seed=4)
    assert np.array_equal(a.x, b.x)
    r = np.sqrt((a.x - 0.5) ** 2 + (a.y - 0.5) ** 2 + (a.z - 0.5) ** 2)
    assert r.max() <= 0.25
    # uniform in volume: P(r < R/2) = 1/8
    assert abs(np.mean(r < 0.125) - 0.125) < 0.02
    assert not a.vx.any()


def test_zeldovich_rms_displacement_and_growing_mode():
    n = 16
    p = ics.zeldovich(n, -2.0, 0.2, 0.02, 1.0, 0.0, seed=1)
    q = (np.arange(n) + 0.5) / n
    Q = np.stack(np.meshgrid(q, q, q, indexing="ij")).reshape(3, -1)
    d = np.stack([p.x, p.y, p.z]) - Q
    d -= np.round(d)  # periodic
    rms = math.sqrt(np.mean(np.sum(d ** 2, axis=0)))
    assert rms == pytest.approx(0.2 / n, rel=1e-6)
    # EdS growing mode: p = a^(1/2) psi(a_start)
    v = np.stack([p.vx, p.vy, p.vz])
    assert np.allclose(v, math.sqrt(0.02) * d, rtol=1e-6, atol=1e-12)
    assert (p.x >= 0).all() and (p.x < 1).all()


def test_growth_factor_matches_eds_analytic():
    d, dd = ics.growth(0.5, 1.0, 0.0)
    assert dd / d == pytest.approx(1.0 / 0.5, rel=1e-8)
    # LambdaCDM growth is slower than EdS at late times
    d1, dd1 = ics.growth(0.9, 0.3, 0.7)
    assert dd1 / d1 < 1.0 / 0.9


def test_factors_follow_readme_equations():
    a, om, ol = 0.3, 0.3, 0.7
    F = (om / a + ol * a * a) ** -0.5
    assert ics.kick_factor(a, om, ol) == pytest.approx(F)
    assert ics.drift_factor(a, om, ol) == pytest.approx(F / (a * a))


def test_named_configs():
    c = ics.config("lcdm128")
    assert (c.n, c.steps, c.omega0, c.omegal) == (128 ** 3, 128, 0.3, 0.7)
    assert c.delta_a == pytest.approx(0.98 / 128)
    assert ics.config("ball32k").n == 32768
