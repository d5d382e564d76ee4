"""Readers and writers of the reference's ASCII grid files.

* ``.tel`` telescoping grid: ``read_tel`` follows source/geospatial/
  geospatial.F90:403-795 (read_tel): one header line; ``angle x0 y0 ncellsfull``;
  then one row per cell ``id x y dx dy n1 n2 e1 e2 s1 s2 w1 w2 depth`` (list-
  directed, so a row may wrap), land cells with depth -999, neighbour entries
  naming file rows (0: none).  Active cells are numbered in file order, dummy
  cells as read_tel numbers them (``grid.assemble``); zb = -depth, and a dummy
  takes the bed of the cell it hangs off.  Cells whose first four faces all
  lead to dummies are isolated and rejected (geospatial.F90:745-790).
* ``.cart`` Cartesian grid: ``read_cart`` follows read_grid_cart
  (geospatial.F90:2553-2706) and geo_cart (2709-2960): cards
  GRID_NUMBER_CELLS_X/Y, GRID_RESOLUTION_X/Y_BEGIN (one spacing per line,
  accumulated) or GRID_COORDS_I/J_BEGIN (cumulative coordinates),
  GRID_DEPTHS_BEGIN and GRID_ACTIVITY_BEGIN blocks (maxcol*maxrow values, i
  fastest), GRID_ANGLE, GRID_ORIGIN_X/Y, GRID_TYPE.  Cells are numbered
  id = i + (j-1)*maxcol over the active ones; every missing or inactive
  neighbour becomes a full-size dummy, N, E, S, W in turn per cell.

The writers produce files these readers (and the reference) accept: the
telescoping writer from a parent-level map, the Cartesian one from column and
row spacings.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import grid as G

LAND = -999.0


@dataclass
class GridFile:
    grid: G.Grid
    zb: np.ndarray        # [ncellsD] bed elevation (-depth), dummies copy their cell's
    angle: float          # grid angle as written in the file (degrees)
    xorigin: float
    yorigin: float
    mapid: np.ndarray     # [ncells] file row (1-based) of each active cell


def parse_tel(path):
    """(angle, x0, y0, rows) of a .tel file: rows[ncellsfull][14] holds each
    cell's ``id x y dx dy n1 n2 e1 e2 s1 s2 w1 w2 depth`` as read."""
    with open(path) as f:
        lines = f.read().splitlines()
    if len(lines) < 2:
        raise ValueError(f"{path}: not a telescoping grid file")
    head = lines[1].replace(",", " ").split()
    angle, x0, y0 = (float(v) for v in head[:3])
    nfull = int(float(head[3]))
    rows = np.empty((nfull, 14))
    q = 2
    for r in range(nfull):
        # one list-directed READ of 14 items per cell: it starts on a new
        # record, may continue over records, and drops what is left of the
        # record where the 14th item was found
        vals = []
        while len(vals) < 14:
            if q >= len(lines):
                raise ValueError(f"{path}: {nfull} cells announced, fewer rows found")
            vals.extend(lines[q].replace(",", " ").split())
            q += 1
        rows[r] = [float(v) for v in vals[:14]]
    return angle, x0, y0, rows


def read_tel(path) -> GridFile:
    angle, x0, y0, rows = parse_tel(path)
    return tel_grid(rows, angle, x0, y0, str(path))


def tel_grid(rows: np.ndarray, angle: float = 0.0, x0: float = 0.0, y0: float = 0.0, name: str = "grid") -> GridFile:
    """The grid of a .tel file's cell rows (parse_tel), as read_tel builds it."""
    path = name
    nfull = rows.shape[0]
    xt, yt, dxt, dyt = rows[:, 1], rows[:, 2], rows[:, 3], rows[:, 4]
    loct = rows[:, 5:13].astype(np.int64)
    zt = rows[:, 13]
    land = np.abs(zt - LAND) < 1.0e-15  # abs(ztemp - fnan) < small
    if np.any((loct < 0) | (loct > nfull)):
        raise ValueError(f"{path}: neighbour entry outside 0..{nfull}")
    idmap = np.zeros(nfull + 1, dtype=np.int64)  # file row -> active id (0: land)
    act = np.nonzero(~land)[0]
    if act.size == 0:
        raise ValueError(f"{path}: no active cells")
    idmap[act + 1] = np.arange(1, act.size + 1)
    island = np.concatenate([[False], land])
    # neighbour slots as active ids, -1 for land, 0 for none (read_tel's first pass)
    loc = np.where(loct == 0, 0, np.where(island[loct], -1, idmap[loct]))[act]
    dxc, dyc = dxt[act], dyt[act]
    # refinement level relative to the coarsest cell (informative only)
    dmin = np.maximum(np.minimum(dxc, dyc), 1e-300)
    lev = (np.rint(np.log2(dmin.max() / dmin)).astype(np.int8) if act.size else np.zeros(0, np.int8))
    tele = bool(np.any(loc[:, 1::2] != 0))
    g = G.assemble(loc, xt[act], yt[act], dxc, dyc, nmaxfaces=6, level=lev, telescoping=tele)
    n = g.ncells
    c = g.cell2cell[:n, :4]
    iso = np.all(c > n, axis=1)
    if np.any(iso):
        raise ValueError(f"{path}: {int(iso.sum())} isolated ocean cells (first file row "
                         f"{int(act[np.nonzero(iso)[0][0]]) + 1})")
    zb = _bed_with_dummies(g, -zt[act])
    return GridFile(g, zb, angle, x0, y0, act + 1)


def _bed_with_dummies(g: G.Grid, zb_active: np.ndarray) -> np.ndarray:
    zb = np.zeros(g.ncellsD)
    zb[: g.ncells] = zb_active
    owner = np.zeros(g.ncellsD, dtype=np.int64)
    for k in range(g.nmaxfaces):
        c = g.cell2cell[g.ncells:, k]
        m = c > 0
        owner[g.ncells:][m] = c[m] - 1
    zb[g.ncells:] = zb[owner[g.ncells:]]
    return zb


def write_tel(path, level: np.ndarray, dx0: float, depth, active=None, angle: float = 0.0, xorigin: float = 0.0,
              yorigin: float = 0.0, header: str = "CMS telescoping grid"):
    """Writes the telescoping grid of a parent-level map (every leaf one row,
    row-major, land leaves with depth -999).  depth: callable (xc, yc) -> depth
    of the active leaves, or an array over all leaves.  Reading the file back
    gives grid.telescoping_grid(level, dx0, active)."""
    fx, fy, fs, lmax, R, W, H = G._leaves(level)
    h = dx0 / R
    xc = (fx + 0.5 * fs) * h
    yc = (fy + 0.5 * fs) * h
    keep = np.ones(fx.size, dtype=bool) if active is None else np.asarray(active(xc, yc, fs * h), dtype=bool)
    ids = np.arange(1, fx.size + 1, dtype=np.int64)
    loc = G._neighbour_slots(G._owner_lookup(fx, fy, fs, ids, W, H), fx, fy, fs)
    dep = np.asarray(depth(xc, yc) if callable(depth) else depth, dtype=np.float64)
    dep = np.where(keep, dep, LAND)
    size = fs * h
    with open(path, "w") as f:
        f.write(header + "\n")
        f.write(f"{angle:.6f} {xorigin:.6f} {yorigin:.6f} {fx.size}\n")
        for r in range(fx.size):
            nb = " ".join(str(int(v)) for v in loc[r])
            f.write(f"{r + 1} {float(xc[r])!r} {float(yc[r])!r} {float(size[r])!r} {float(size[r])!r} {nb} "
                    f"{float(dep[r])!r}\n")


# ---------------------------------------------------------------------------
# Cartesian grid file

def read_cart(path) -> GridFile:
    with open(path) as f:
        lines = f.read().splitlines()
    maxcol = maxrow = 0
    angle = x0 = y0 = 0.0
    dxx = dyy = z = cell_type = None
    q = 0

    def block(count, one_per_line):
        nonlocal q
        vals = []
        if one_per_line:  # read(kunit,*) dxx(i), one record per value
            for _ in range(count):
                vals.append(float(lines[q].replace(",", " ").split()[0]))
                q += 1
        else:  # one list-directed read of count values across records
            while len(vals) < count:
                vals.extend(float(t) for t in lines[q].replace(",", " ").split())
                q += 1
            vals = vals[:count]
        q += 1  # the end card
        return np.array(vals)

    while q < len(lines):
        parts = lines[q].replace(",", " ").split()
        q += 1
        if not parts:
            continue
        card = parts[0]
        if card == "GRID_ANGLE":
            angle = float(parts[1])
        elif card == "GRID_ORIGIN_X":
            x0 = float(parts[1])
        elif card == "GRID_ORIGIN_Y":
            y0 = float(parts[1])
        elif card == "GRID_NUMBER_CELLS_X":
            maxcol = int(parts[1])
        elif card == "GRID_NUMBER_CELLS_Y":
            maxrow = int(parts[1])
        elif card == "GRID_RESOLUTION_X_BEGIN":
            dxx = np.cumsum(block(maxcol, True))
        elif card == "GRID_RESOLUTION_Y_BEGIN":
            dyy = np.cumsum(block(maxrow, True))
        elif card in ("GRID_COORDSI_BEGIN", "GRID_COORDS_I_BEGIN"):
            dxx = block(maxcol, False)
        elif card in ("GRID_COORDSJ_BEGIN", "GRID_COORDS_J_BEGIN"):
            dyy = block(maxrow, False)
        elif card == "GRID_DEPTHS_BEGIN":
            z = block(maxcol * maxrow, False)
        elif card in ("GRID_ACTIVITY_BEGIN", "GRID_ACTIVE_BEGIN"):
            cell_type = block(maxcol * maxrow, False).astype(np.int64)
    if maxcol <= 0 or maxrow <= 0 or dxx is None or dyy is None or z is None:
        raise ValueError(f"{path}: incomplete Cartesian grid file")
    if cell_type is None:
        # read_grid_cart assigns the whole array inside its per-cell loop
        # (geospatial.F90:2690-2698), so the last cell's depth decides for all
        cell_type = np.full(z.size, 0 if abs(z[-1] + 999.0) < 1.0 else 1, dtype=np.int64)
    return _cart_grid(dxx, dyy, z, cell_type, angle, x0, y0)


def _cart_grid(dxx, dyy, z, cell_type, angle, x0, y0) -> GridFile:
    maxcol, maxrow = dxx.size, dyy.size
    ct = cell_type.reshape(maxrow, maxcol)
    zz = z.reshape(maxrow, maxcol)
    jj, ii = np.nonzero(ct >= 1)  # row-major: j outer, i inner
    n = ii.size
    if n == 0:
        raise ValueError("no active cells")
    idmap = np.zeros((maxrow, maxcol), dtype=np.int64)
    idmap[jj, ii] = np.arange(1, n + 1)
    dxc = np.where(ii == 0, dxx[ii], dxx[ii] - dxx[np.maximum(ii - 1, 0)])
    dyc = np.where(jj == 0, dyy[jj], dyy[jj] - dyy[np.maximum(jj - 1, 0)])
    xc = dxx[ii] - 0.5 * dxc
    yc = dyy[jj] - 0.5 * dyc

    def nb(dj, di):
        j2, i2 = jj + dj, ii + di
        ok = (j2 >= 0) & (j2 < maxrow) & (i2 >= 0) & (i2 < maxcol)
        out = np.zeros(n, dtype=np.int64)
        out[ok] = idmap[j2[ok], i2[ok]]
        return out  # 0: outside or inactive -> dummy

    loc = np.zeros((n, 8), dtype=np.int64)
    for q, (dj, di) in enumerate(((1, 0), (0, 1), (-1, 0), (0, -1))):
        loc[:, 2 * q] = nb(dj, di)
    g = G.assemble(loc, xc, yc, dxc, dyc, nmaxfaces=4)
    g.idirface[g.ncells:] = 0
    if np.any(np.all(g.cell2cell[:n, :4] > n, axis=1)):
        raise ValueError("invalid ocean cell: all four neighbours are dummies")
    zb = _bed_with_dummies(g, -zz[jj, ii])
    return GridFile(g, zb, angle, x0, y0, (ii + 1 + jj * maxcol).astype(np.int64))


def write_cart(path, dx_cols, dy_rows, depth, active=None, angle: float = 0.0, xorigin: float = 0.0,
               yorigin: float = 0.0, coords: bool = False):
    """Writes a Cartesian grid file: column widths dx_cols [maxcol], row
    heights dy_rows [maxrow], depth [maxrow, maxcol] (i fastest), active mask
    of the same shape (None: all active).  coords=True writes cumulative
    coordinate blocks instead of the resolution blocks."""
    dx_cols = np.asarray(dx_cols, dtype=np.float64)
    dy_rows = np.asarray(dy_rows, dtype=np.float64)
    depth = np.asarray(depth, dtype=np.float64)
    maxcol, maxrow = dx_cols.size, dy_rows.size
    act = np.ones((maxrow, maxcol), dtype=np.int64) if active is None else np.asarray(active).astype(np.int64)
    with open(path, "w") as f:
        f.write("CMS_GRID_FILE\n")
        f.write("GRID_TYPE REGULAR\n")
        f.write(f"GRID_ANGLE {float(angle)!r}\nGRID_ORIGIN_X {float(xorigin)!r}\nGRID_ORIGIN_Y {float(yorigin)!r}\n")
        f.write(f"GRID_NUMBER_CELLS_X {maxcol}\nGRID_NUMBER_CELLS_Y {maxrow}\n")
        if coords:
            f.write("GRID_COORDS_I_BEGIN\n" + " ".join(repr(float(v)) for v in np.cumsum(dx_cols)) + "\nGRID_COORDS_I_END\n")
            f.write("GRID_COORDS_J_BEGIN\n" + " ".join(repr(float(v)) for v in np.cumsum(dy_rows)) + "\nGRID_COORDS_J_END\n")
        else:
            f.write("GRID_RESOLUTION_X_BEGIN\n" + "".join(f"{float(v)!r}\n" for v in dx_cols) + "GRID_RESOLUTION_X_END\n")
            f.write("GRID_RESOLUTION_Y_BEGIN\n" + "".join(f"{float(v)!r}\n" for v in dy_rows) + "GRID_RESOLUTION_Y_END\n")
        f.write("GRID_DEPTHS_BEGIN\n")
        for j in range(maxrow):
            f.write(" ".join(repr(float(v)) for v in depth[j]) + "\n")
        f.write("GRID_DEPTHS_END\nGRID_ACTIVITY_BEGIN\n")
        for j in range(maxrow):
            f.write(" ".join(str(int(v)) for v in act[j]) + "\n")
        f.write("GRID_ACTIVITY_END\n")
