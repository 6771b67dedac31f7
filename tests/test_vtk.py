"""Legacy-VTK IC and snapshot files in the reference's layouts (initialization.cpp:21-101,
viewer.cpp:12-116)."""
from __future__ import annotations

import numpy as np

from apcloud import ics, vtk


def test_ic_round_trip(tmp_path):
    p = ics.config("ball32k", n=500, seed=4).particles()
    p.vx[:] = np.linspace(-1, 1, p.n)
    ids = np.arange(p.n)[::-1].copy()
    f = tmp_path / "ic.vtk"
    vtk.write_ic(str(f), p, ids)
    q, qid = vtk.read_ic(str(f), unit_velocity=2.0)
    assert np.array_equal(q.x, p.x) and np.array_equal(q.z, p.z)
    assert np.array_equal(q.vx, p.vx / 2.0)
    assert np.array_equal(qid, ids)
    r, _ = vtk.read_ic(str(f), redshift=3.0)
    assert np.allclose(r.vy, p.vy / 4.0 / 2.0, rtol=0, atol=1e-15)


def test_reader_accepts_the_reference_line_layout(tmp_path):
    """A file laid out line by line as the reference's reader expects it."""
    lines = ["# vtk DataFile Version 3.0", "ICs", "ASCII", "DATASET POLYDATA", "POINTS 3 double",
             "0.1 0.2 0.3", "0.4 0.5 0.6", "0.7 0.8 0.9", "", "POINT_DATA 3",
             "SCALARS v_x double", "LOOKUP_TABLE default", "1", "2", "3", "",
             "SCALARS v_y double", "LOOKUP_TABLE default", "4", "5", "6", "",
             "SCALARS v_z double", "LOOKUP_TABLE default", "7", "8", "9", "",
             "SCALARS ID int", "LOOKUP_TABLE default", "10", "11", "12"]
    f = tmp_path / "ref.vtk"
    f.write_text("\n".join(lines) + "\n")
    p, ids = vtk.read_ic(str(f))
    assert np.allclose(p.y, [0.2, 0.5, 0.8]) and np.allclose(p.vz, [7, 8, 9])
    assert list(ids) == [10, 11, 12]


def test_physical_and_computational_snapshots(tmp_path):
    from types import SimpleNamespace

    n, m = 50, 7
    rng = np.random.default_rng(0)
    arr = [rng.random(n) for _ in range(9)]
    path = vtk.write_physical(str(tmp_path), 0.25, *arr)
    assert path.endswith("physical_0.250000.vtk")
    sc = vtk.read_scalars(path)
    assert set(sc) == {"v_x", "v_y", "v_z", "a_x", "a_y", "a_z"}
    assert np.allclose(sc["a_z"], arr[8], rtol=1e-6)
    cells = SimpleNamespace(x=rng.random(m), y=rng.random(m), z=rng.random(m), count=np.arange(m),
                            type=np.zeros(m, int), first=np.arange(m) * 3)
    fields = SimpleNamespace(density=rng.random(m), potential=rng.random(m), deriv=rng.random((m, 9)))
    cpath = vtk.write_computational(str(tmp_path), 0.25, cells, fields)
    cs = vtk.read_scalars(cpath)
    assert list(cs["n_p"]) == list(range(m)) and list(cs["first_id"]) == list(cells.first)
    assert np.allclose(cs["p_y"], fields.deriv[:, 1], rtol=1e-6)


def test_controller_writes_snapshots(tmp_path, oracle_lib):
    """The Controller's viewer output on the oracle backend: one physical file per interval,
    computational files once fields exist."""
    import refbind
    from apcloud.controller import for_config

    cfg = ics.config("ball32k", n=800, seed=2, steps=20)
    o = refbind.CpuPath("oracle", cfg.particles(), cfg.depth, cfg.gfd_c)
    o.set_gmres(30, 1e-10)
    c = for_config(o, cfg)
    c.output_dir, c.write_interval = str(tmp_path), 2
    c.start()
    for _ in range(3):
        c.step()
    o.close()
    names = sorted(f.name for f in tmp_path.iterdir())
    assert sum(nm.startswith("physical_") for nm in names) == 2
    assert sum(nm.startswith("computational_") for nm in names) == 1
