"""Legacy-VTK particle files in the reference's layouts.

* Initial conditions (initialization.cpp:21-101, ICFileType 1): an ASCII POLYDATA file with
  POINTS N (x y z per point), then POINT_DATA scalars v_x, v_y, v_z (one value per
  line) and the integer particle IDs.  Velocities are divided by UnitVelocity_in_cm_per_s
  and, with COSMOLOGY_UNIT, by (1 + z)^(3/2).
* Snapshots (viewer.cpp:12-116): physical_<t>.vtk with positions (%f), the velocity and
  acceleration vectors and their components (%e); computational_<t>.vtk with the cell
  centres and n_p, type, first_id, density, potential, p_x, p_y, p_z.

The reader follows the sections by their keywords rather than by counting lines, so it
reads the files the writer makes and the reference's ICs alike.
"""
from __future__ import annotations

import io
import os

import numpy as np

from .ics import Particles


def _tokens(path):
    with open(path) as f:
        return f.read().split()


def read_ic(path: str, unit_velocity: float = 1.0, redshift: float | None = None):
    """(Particles, ids) from an IC file; redshift: apply the COSMOLOGY_UNIT scaling."""
    tok = _tokens(path)
    i = tok.index("POINTS")
    n = int(tok[i + 1])
    j = i + 3  # POINTS N <type>
    pos = np.array(tok[j:j + 3 * n], dtype=np.float64).reshape(n, 3)
    j += 3 * n
    cols = []
    while len(cols) < 4:
        k = tok.index("LOOKUP_TABLE", j)
        j = k + 2
        dtype = np.int64 if len(cols) == 3 else np.float64
        cols.append(np.array(tok[j:j + n], dtype=dtype))
        j += n
    vx, vy, vz, ids = cols
    vel = [v * (1.0 / unit_velocity) for v in (vx, vy, vz)]
    if redshift is not None:
        f = 1.0 / (1.0 + redshift) / np.sqrt(1.0 + redshift)
        vel = [v * f for v in vel]
    return Particles(pos[:, 0].copy(), pos[:, 1].copy(), pos[:, 2].copy(), *vel), ids.astype(np.int32)


def write_ic(path: str, parts: Particles, ids=None):
    """An IC file the reference's reader accepts (the layout of a physical snapshot's
    header, positions, v_x/v_y/v_z scalars and the IDs)."""
    n = parts.n
    ids = np.arange(n) if ids is None else np.asarray(ids)
    out = io.StringIO()
    out.write("# vtk DataFile Version 3.0\nInitial conditions\nASCII\nDATASET POLYDATA\n")
    out.write(f"POINTS {n} double\n")
    np.savetxt(out, np.stack([parts.x, parts.y, parts.z], 1), fmt="%.17g")
    out.write(f"\nPOINT_DATA {n}\n")
    for name, v in (("v_x", parts.vx), ("v_y", parts.vy), ("v_z", parts.vz)):
        out.write(f"SCALARS {name} double\nLOOKUP_TABLE default\n")
        np.savetxt(out, v, fmt="%.17g")
        out.write("\n")
    out.write("SCALARS ID int\nLOOKUP_TABLE default\n")
    np.savetxt(out, ids, fmt="%d")
    with open(path, "w") as f:
        f.write(out.getvalue())


def _scalar(out, name, kind, v, fmt):
    out.write(f"\nSCALARS {name} {kind}\nLOOKUP_TABLE default\n")
    np.savetxt(out, v, fmt=fmt)


def write_physical(directory: str, t: float, x, y, z, vx, vy, vz, ax, ay, az) -> str:
    """viewer.cpp:12-61: <directory>/physical_<t>.vtk; returns the path."""
    n = len(x)
    out = io.StringIO()
    out.write("# vtk DataFile Version 3.0\nData on physical particles for cosmology problem\nASCII\n")
    out.write(f"DATASET POLYDATA\nPOINTS {n} double\n\n")
    np.savetxt(out, np.stack([x, y, z], 1), fmt="%f")
    out.write(f"\nPOINT_DATA {n}")
    out.write("\nVECTORS velocity double\n")
    np.savetxt(out, np.stack([vx, vy, vz], 1), fmt="%e")
    for name, v in (("v_x", vx), ("v_y", vy), ("v_z", vz)):
        _scalar(out, name, "double", v, "%e")
    out.write("\nVECTORS acceleration double\n")
    np.savetxt(out, np.stack([ax, ay, az], 1), fmt="%e")
    for name, v in (("a_x", ax), ("a_y", ay), ("a_z", az)):
        _scalar(out, name, "double", v, "%e")
    path = os.path.join(directory, "physical_%f.vtk" % t)
    with open(path, "w") as f:
        f.write(out.getvalue())
    return path


def write_computational(directory: str, t: float, cells, fields) -> str:
    """viewer.cpp:63-116: <directory>/computational_<t>.vtk from GpuPath.cells() and
    GpuPath.fields() (or the oracle's); returns the path."""
    m = len(fields.density)
    out = io.StringIO()
    out.write("# vtk DataFile Version 3.0\nData on computational particles for cosmology problem\nASCII\n")
    out.write(f"DATASET POLYDATA\nPOINTS {m} double\n\n")
    np.savetxt(out, np.stack([cells.x[:m], cells.y[:m], cells.z[:m]], 1), fmt="%f")
    out.write(f"\nPOINT_DATA {m}\n")
    out.write("SCALARS n_p int\nLOOKUP_TABLE default\n")
    np.savetxt(out, cells.count[:m], fmt="%d")
    _scalar(out, "type", "int", cells.type[:m], "%d")
    _scalar(out, "first_id", "int", cells.first[:m], "%d")
    _scalar(out, "density", "double", fields.density, "%e")
    _scalar(out, "potential", "double", fields.potential, "%e")
    for k, name in enumerate(("p_x", "p_y", "p_z")):
        _scalar(out, name, "double", fields.deriv[:, k], "%e")
    path = os.path.join(directory, "computational_%f.vtk" % t)
    with open(path, "w") as f:
        f.write(out.getvalue())
    return path


def read_scalars(path: str) -> dict:
    """name -> array of every SCALARS section of a snapshot (for checks and tools)."""
    tok = _tokens(path)
    n = int(tok[tok.index("POINT_DATA") + 1])
    out = {}
    j = 0
    while True:
        try:
            k = tok.index("SCALARS", j)
        except ValueError:
            return out
        name, kind = tok[k + 1], tok[k + 2]
        s = tok.index("LOOKUP_TABLE", k) + 2
        out[name] = np.array(tok[s:s + n], dtype=np.int64 if kind == "int" else np.float64)
        j = s + n
