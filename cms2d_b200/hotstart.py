"""Hot-start files in the SMS generic ASCII dataset format.

The reference writes an ASCII hot start as a super file and one dataset file
per field (write_hotstart_sup, source/hot_start/hot_start.F90:1625-1736): the
water pressure, the water level, the current velocity and the wet flags, each
through write_scal_dat_file / write_vec_dat_file (source/output/
out_lib.f90:252-605):

    DATASET / OBJTYPE "scat2d" / BEGSCL (BEGVEC + VECTYPE 0) / OBJID 17255 /
    ND n / NC n / NAME "..." / RT_JULIAN t0 / TIMEUNITS hours /
    TS 0 <hours> / one value per active cell (1pe12.5; NaN as -999) / ENDDS

and it reads initial conditions back with hot_read_dat (hot_start.F90:
596-690): the water level (Water_Elevation and its aliases; p = g eta) and
the current velocity (Current_Velocity and its aliases), on the full grid of
the grid file (land cells included), mapped to the active cells; with wet
flags in the dataset the velocity of a dry cell is zeroed.  The reference's
writer writes the active cells only (ncells values) while its reader asks for
the full grid (ncellsfull values); read_hot_start accepts both.

write_hot_start / read_hot_start produce and consume these files;
hot_start_fields turns what was read into the arguments of
FlowModel.init_hot (pressure and velocities of all ncellsD cells, dummies
taking their cell's values).
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field

import numpy as np

GRAV = 9.81  # grav, source/flow/flow.F90:34
OBJID = 17255

SCALAR_NAMES = ("Water_Elevation", "Water_Surface_Elevation", "Water_Level", "wse", "WSE")
VECTOR_NAMES = ("Current_Velocity", "Water_Velocity", "Depth-Averaged_Current_Velocity", "Depth-Averaged_Velocity")


@dataclass
class Dataset:
    name: str
    vector: bool
    nd: int
    times: list = field(default_factory=list)   # hours
    values: list = field(default_factory=list)  # [nd] or [nd, 2] per time step
    status: list = field(default_factory=list)  # [nd] flags per time step, or None


def _fmt(v: float) -> str:
    """Fortran 1pe12.5 (NaN written as -999., as the reference does)."""
    if not np.isfinite(v):
        return f"{-999.0:11.0f}."  # F12.0
    s = f"{v:.5E}"
    mant, ex = s.split("E")
    return f"{mant}E{int(ex):+03d}".rjust(12)


def _write_dataset(path, name: str, values, time_hours: float, reftime: float, vector: bool):
    values = np.asarray(values, dtype=np.float64)
    n = values.shape[0]
    with open(path, "w") as f:
        f.write("DATASET\nOBJTYPE \"scat2d\"\n")
        f.write("BEGVEC\nVECTYPE 0\n" if vector else "BEGSCL\n")
        f.write(f"OBJID {OBJID:5d}\nND {n:6d}\nNC {n:6d}\nNAME \"{name}\"\n")
        f.write(f"RT_JULIAN {reftime:15.3f}\nTIMEUNITS hours\n")
        f.write(f"TS 0 {time_hours:12.4f}\n")
        for row in values:
            f.write((_fmt(row[0]) + " " + _fmt(row[1]) if vector else _fmt(row)) + "\n")
        f.write("ENDDS\n")


def write_hot_start(prefix, p, eta, u, v, iwet, ncells: int, time_hours: float = 0.0, reftime: float = 0.0,
                    sediment=None, salinity=None, heat=None):
    """prefix.sup plus prefix_p.dat, _eta.dat, _vel.dat, _wet.dat (and the
    optional transport fields) over the first ncells (active) cells."""
    prefix = str(prefix)
    files = []

    def scal(label, suffix, arr):
        fn = f"{prefix}_{suffix}.dat"
        _write_dataset(fn, label, np.asarray(arr, dtype=np.float64)[:ncells], time_hours, reftime, False)
        files.append(fn)

    scal("Water_Pressure", "p", p)
    scal("Water_Elevation", "eta", eta)
    fn = f"{prefix}_vel.dat"
    _write_dataset(fn, "Current_Velocity", np.stack([np.asarray(u)[:ncells], np.asarray(v)[:ncells]], axis=1),
                   time_hours, reftime, True)
    files.append(fn)
    scal("Wet", "wet", np.asarray(iwet, dtype=np.float64))
    if sediment is not None:
        scal("Concentration", "conc", sediment)
    if salinity is not None:
        scal("Salinity", "sal", salinity)
    if heat is not None:
        scal("Heat", "heat", heat)
    with open(prefix + ".sup", "w") as f:
        f.write("SUPER\n")
        for fn in files:
            f.write(f"DATA    \"{os.path.basename(fn)}\"\n")
    return files


def read_datasets(path) -> list:
    """Every dataset block of an SMS generic ASCII dataset file."""
    with open(path) as f:
        lines = [ln.strip() for ln in f]
    out, cur, q = [], None, 0
    while q < len(lines):
        ln = lines[q]
        q += 1
        if not ln:
            continue
        card = ln.split()[0]
        if card in ("BEGSCL", "BEGVEC"):
            cur = Dataset(name="", vector=card == "BEGVEC", nd=0)
        elif cur is None:
            continue
        elif card == "ND":
            cur.nd = int(ln.split()[1])
        elif card == "NAME":
            cur.name = ln.split(None, 1)[1].strip().strip('"')
        elif card == "TS":
            parts = ln.split()
            istat, t = int(parts[1]), float(parts[2])
            stat = None
            if istat:
                stat = np.array([float(lines[q + k].split()[0]) for k in range(cur.nd)])
                q += cur.nd
            rows = [lines[q + k].split() for k in range(cur.nd)]
            q += cur.nd
            vals = np.array([[float(x) for x in r[:2]] for r in rows]) if cur.vector else \
                np.array([float(r[0]) for r in rows])
            cur.times.append(t)
            cur.values.append(vals)
            cur.status.append(stat)
        elif card == "ENDDS":
            out.append(cur)
            cur = None
    return out


def read_hot_start(sup_path) -> list:
    """The datasets of every file a super file lists."""
    base = os.path.dirname(os.path.abspath(sup_path))
    out = []
    with open(sup_path) as f:
        for ln in f:
            parts = ln.split(None, 1)
            if len(parts) == 2 and parts[0] == "DATA":
                out += read_datasets(os.path.join(base, parts[1].strip().strip('"')))
    return out


def _to_active(vals, gf):
    """Full-grid values (ncellsfull, by file row / cell id) or active-cell
    values (ncells) to the active cells."""
    n = gf.grid.ncells
    vals = np.asarray(vals)
    if vals.shape[0] == n:
        return vals
    if vals.shape[0] >= int(np.max(gf.mapid)):
        return vals[np.asarray(gf.mapid, dtype=np.int64) - 1]
    raise ValueError(f"dataset of {vals.shape[0]} values does not match the grid ({n} active cells)")


def _with_dummies(g, act):
    out = np.zeros(g.ncellsD)
    out[: g.ncells] = act
    for k in range(g.nmaxfaces):
        c = g.cell2cell[g.ncells:, k]
        m = c > 0
        out[g.ncells:][m] = act[c[m] - 1]
    return out


def hot_start_fields(datasets, gf, grav: float = GRAV, hmin: float = 0.05):
    """p, u, v (ncellsD each) and the time (hours) of the last record, as
    hot_read_dat reads the water level and the current velocity.  A water
    level, not a pressure, was read, so a cell that hot_init finds dry
    (h < hmin + 1e-5) gets p = (hmin + zb - 1e-4) g (hot_start.F90:1171-1173)."""
    eta = u = v = None
    t = 0.0
    for d in datasets:
        if not d.vector and d.name in SCALAR_NAMES:
            eta = _to_active(d.values[-1], gf)
            t = d.times[-1]
            break
    for d in datasets:
        if d.vector and d.name in VECTOR_NAMES:
            uv = _to_active(d.values[-1], gf)
            u, v = uv[:, 0].copy(), uv[:, 1].copy()
            if d.status[-1] is not None:
                w = _to_active(d.status[-1], gf)
                u *= w
                v *= w
            t = d.times[-1]
            break
    if eta is None or u is None:
        raise ValueError("the hot start needs a water level and a current velocity dataset")
    g = gf.grid
    p = _with_dummies(g, eta * grav)
    zb = np.asarray(gf.zb, dtype=np.float64)
    h = p * (1.0 / grav) - zb
    dry = h < hmin + 1.0e-5
    p[dry] = (hmin + zb[dry] - 1.0e-4) * grav
    return p, _with_dummies(g, u), _with_dummies(g, v), t
