"""Seeded synthetic flow cases with the shapes of the benchmark configurations.

tidal_basin:  rectangular basin on a uniform Cartesian grid (default 200 x 100
              cells at 20 m), depth a linear slope from 2 m at the shore to
              10 m offshore plus seeded Gaussian bumps (0.2 m standard
              deviation), an M2 water level (0.5 m, 12.42 h) on the open
              offshore (north) edge, walls elsewhere, Manning n = 0.025.
tidal_inlet:  three-level telescoping grid (40/20/10 m) of about 1.0M active
              cells: ocean to the north, a barrier strip (inactive land) cut by
              a 300 m wide, 8 m deep inlet channel, an ebb shoal of 2-6 m in
              front of it and a back bay; lognormal Manning n (median 0.025,
              sigma_log 0.2); M2 + K1 water level (0.6 m / 0.2 m) on the north
              edge.
tidal_flat:   intertidal flat that wets and dries over the tide: bed from 1 m
              above mean sea level at the south shore to 3 m depth at the open
              north edge, seeded bumps, a one-cell-wide creek cut into the flat
              and a depression on the upper flat that is cut off at low water;
              M2 tide of 1 m.  Cartesian, or telescoping with a refined zone
              around the creek.

gauges:       seeded water-level gauge cells of a case (the misfit of the
              adjoint gradient and the fixtures of the parity tests).

from_grid_file: a case on a grid read from a .tel or .cart file
              (cms2d_b200.gridio), with a water-level string on its open north
              edge, a tide and a uniform Manning n.

A case carries the grid (cms2d_b200.grid.Grid), bed elevation zb (= -depth,
ncellsD values; dummies copy their parent cell), coefman (ncells), the
water-level string (1-based cells and faces of the open edge) and the tide.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import grid as G

M2_HOURS = 12.42
K1_HOURS = 23.93


@dataclass
class Case:
    name: str
    grid: G.Grid
    zb: np.ndarray
    coefman: np.ndarray
    th_cells: np.ndarray
    th_faces: np.ndarray
    tide: list  # [(amplitude m, period h)]
    dt: float
    nsteps: int
    t0: float = 0.0  # tide phase: the water level at time t is the tide at t0 + t (seconds)
    th_offset: np.ndarray = None  # per string cell: a constant added to the tide (a head difference)

    def wse(self, t_seconds: float) -> float:
        th = (t_seconds + self.t0) / 3600.0
        return float(sum(a * np.cos(2.0 * np.pi * th / T) for a, T in self.tide))

    def wsebnd(self, t_seconds: float) -> np.ndarray:
        out = np.full(self.th_cells.size, self.wse(t_seconds))
        return out if self.th_offset is None else out + self.th_offset


def _smooth_field(shape, corr_cells: float, rng) -> np.ndarray:
    """Unit-variance Gaussian random field with a Gaussian correlation (FFT filter)."""
    ny, nx = shape
    w = rng.standard_normal(shape)
    ky = np.fft.fftfreq(ny)[:, None]
    kx = np.fft.fftfreq(nx)[None, :]
    filt = np.exp(-2.0 * (np.pi * corr_cells) ** 2 * (kx ** 2 + ky ** 2))
    f = np.real(np.fft.ifft2(np.fft.fft2(w) * filt))
    s = f.std()
    return f / s if s > 0 else f


def _north_string(g: G.Grid):
    """Active cells whose north face leads to a dummy, with that face (1-based)."""
    return _edge_string(g, G.N_)


def _edge_string(g: G.Grid, direction: int):
    """Active cells whose face of the given direction (1-4 = N, E, S, W)
    leads to a dummy, with that face (1-based)."""
    n = g.ncells
    cells, faces = [], []
    for k in range(g.nmaxfaces):
        c = g.cell2cell[:n, k]
        m = (k < g.ncface[:n]) & (c > n) & (g.idirface[:n, k] == direction)
        idx = np.nonzero(m)[0]
        cells.append(idx + 1); faces.append(np.full(idx.size, k + 1))
    cells = np.concatenate(cells); faces = np.concatenate(faces)
    o = np.argsort(cells, kind="stable")
    return cells[o].astype(np.int32), faces[o].astype(np.int32)


def _fill_dummies(g: G.Grid, vals_active: np.ndarray) -> np.ndarray:
    """Extends a cell field to the dummies (each copies the cell it hangs off)."""
    out = np.zeros(g.ncellsD)
    out[: g.ncells] = vals_active
    parent = np.zeros(g.ncellsD, np.int64)
    for k in range(g.nmaxfaces):
        c = g.cell2cell[g.ncells:, k]
        m = c > 0
        parent[g.ncells:][m] = c[m] - 1
    out[g.ncells:] = vals_active[parent[g.ncells:]]
    return out


def tidal_basin(nx: int = 200, ny: int = 100, dx: float = 20.0, seed: int = 0, amp: float = 0.5,
                manning: float = 0.025, dt: float = 600.0, hours: float = 24.0, depth_shore: float = 2.0,
                depth_off: float = 10.0) -> Case:
    rng = np.random.default_rng(seed)
    g = G.cartesian_grid(nx, ny, dx)
    n = g.ncells
    jrow = (g.y[:n] / dx - 0.5)  # 0 .. ny-1
    depth = depth_shore + (depth_off - depth_shore) * jrow / max(ny - 1, 1)
    bumps = _smooth_field((ny, nx), 6.0, rng) * 0.2
    depth = depth + bumps.ravel()  # natural order is row-major (y then x)
    zb = _fill_dummies(g, -depth)
    th_cells, th_faces = _north_string(g)
    return Case("tidal_basin", g, zb, np.full(n, manning), th_cells, th_faces, [(amp, M2_HOURS)], dt,
                int(round(hours * 3600.0 / dt)))


def from_grid_file(gf, tide=((0.5, M2_HOURS),), manning: float = 0.025, dt: float = 600.0, hours: float = 24.0,
                   name: str = "grid_file") -> Case:
    """A case on a grid read by gridio.read_tel / read_cart: the bed from the
    file, the water-level string on every north face that leads to a dummy."""
    g = gf.grid
    th_cells, th_faces = _north_string(g)
    return Case(name, g, np.asarray(gf.zb, dtype=np.float64), np.full(g.ncells, manning), th_cells, th_faces,
                [tuple(t) for t in tide], dt, int(round(hours * 3600.0 / dt)))


def through_flow(gf, head: float, manning: float = 0.025, dt: float = 60.0, steps: int = 10,
                 name: str = "through_flow") -> Case:
    """A case on a grid file (a flume or basin) driven by a water-level
    difference: strings on the west (level +head/2) and east (-head/2) edges,
    walls elsewhere, cold start at level 0 -- a steady through-flow after a few
    steps, as the reference's flume test cases carry an inflow."""
    g = gf.grid
    wc, wf = _edge_string(g, G.W_)
    ec, ef = _edge_string(g, G.E_)
    cells = np.concatenate([wc, ec]); faces = np.concatenate([wf, ef])
    off = np.concatenate([np.full(wc.size, 0.5 * head), np.full(ec.size, -0.5 * head)])
    o = np.argsort(cells, kind="stable")
    return Case(name, g, np.asarray(gf.zb, dtype=np.float64), np.full(g.ncells, manning), cells[o].astype(np.int32),
                faces[o].astype(np.int32), [(0.0, M2_HOURS)], dt, steps, th_offset=off[o])


def ensemble_specs(nmembers: int = 64, seed: int = 0, nmin: int = 50_000, nmax: int = 400_000) -> list:
    """The members of ensemble_basins without building them: one dict of
    tidal_basin arguments per member (nx, ny and the member's seed, M2
    amplitude, Manning n and depth profile), drawn in member order."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(nmembers):
        ncell = rng.uniform(nmin, nmax)
        aspect = rng.uniform(1.0, 4.0)
        long_side = int(round(np.sqrt(ncell * aspect)))
        short_side = max(4, int(round(ncell / long_side)))
        nx, ny = (long_side, short_side) if rng.random() < 0.5 else (short_side, long_side)
        out.append(dict(nx=nx, ny=ny, seed=int(rng.integers(1 << 30)), amp=float(rng.uniform(0.3, 1.0)),
                        manning=float(rng.uniform(0.015, 0.035)), depth_shore=float(rng.uniform(1.5, 3.0)),
                        depth_off=float(rng.uniform(6.0, 14.0)), name=f"basin{k:02d}"))
    return out


def basin_from_spec(spec: dict, dt: float = 600.0, steps: int = 24) -> Case:
    c = tidal_basin(spec["nx"], spec["ny"], 20.0, seed=spec["seed"], amp=spec["amp"], manning=spec["manning"], dt=dt,
                    hours=steps * dt / 3600.0, depth_shore=spec["depth_shore"], depth_off=spec["depth_off"])
    c.name = spec["name"]
    return c


def ensemble_basins(nmembers: int = 64, seed: int = 0, nmin: int = 50_000, nmax: int = 400_000,
                    dt: float = 600.0, steps: int = 24, members=None) -> list:
    """Independent tidal basins of uneven size: uniform Cartesian grids at
    20 m with nmin..nmax cells and aspect ratios 1:1 to 4:1, each with its own
    M2 amplitude (0.3-1.0 m), Manning n (0.015-0.035) and depth profile
    (shore 1.5-3 m, offshore 6-14 m, its own seeded bumps).  members: the
    indices to build (default all), e.g. one rank's share of the ensemble."""
    specs = ensemble_specs(nmembers, seed, nmin, nmax)
    idx = range(nmembers) if members is None else members
    return [basin_from_spec(specs[k], dt, steps) for k in idx]


def tidal_inlet(target_cells: int = 1_000_000, seed: int = 0, dt: float = 300.0, nsteps: int = 48) -> Case:
    """Three-level telescoping tidal inlet of about target_cells active cells."""
    rng = np.random.default_rng(seed)
    dx0 = 40.0
    # parent lattice scaled so that the active count lands near the target
    # (the refined zones roughly double the parent count)
    P = target_cells / 2.07
    ny = int(round(np.sqrt(P / 1.7)))
    nx = int(round(1.7 * ny))
    xc = nx // 2
    yb0 = int(0.45 * ny)                 # barrier strip rows [yb0, yb1)
    yb1 = yb0 + max(4, ny // 60)
    lev = np.zeros((ny, nx), dtype=np.int64)
    # level 1: wide zone around the inlet; level 2: the channel and ebb shoal core
    w1x, w1y = int(0.22 * nx), int(0.30 * ny)
    w2x, w2y = int(0.06 * nx), int(0.12 * ny)
    lev[max(0, (yb0 + yb1) // 2 - w1y): min(ny, (yb0 + yb1) // 2 + w1y), max(0, xc - w1x): min(nx, xc + w1x)] = 1
    lev[max(0, (yb0 + yb1) // 2 - w2y): min(ny, (yb0 + yb1) // 2 + w2y), max(0, xc - w2x): min(nx, xc + w2x)] = 2
    x_in = (xc + 0.5) * dx0  # inlet centre x
    half_w = 150.0           # 300 m channel

    def active(x, y, s):
        in_barrier = (y > yb0 * dx0) & (y < yb1 * dx0)
        in_gap = np.abs(x - x_in) < half_w
        return ~(in_barrier & ~in_gap)

    g = G.telescoping_grid(lev, dx0, active=active, nmaxfaces=6)
    n = g.ncells
    x, y = g.x[:n], g.y[:n]
    yb = 0.5 * (yb0 + yb1) * dx0
    Ly = ny * dx0
    # depth: bay 3 m, ocean 5 m near the barrier rising to 14 m offshore,
    # ebb shoal mound (2 m crest) in front of the inlet, 8 m channel in the gap
    off = np.clip((y - yb) / (Ly - yb), 0.0, 1.0)
    depth = np.where(y < yb, 3.0, 5.0 + 9.0 * off)
    r2 = ((x - x_in) / 1200.0) ** 2 + ((y - (yb + 900.0)) / 700.0) ** 2
    shoal = np.exp(-r2)
    depth = np.where(y >= yb, depth - (depth - 2.0) * shoal, depth)
    chan = (np.abs(x - x_in) < half_w) & (np.abs(y - yb) < (yb1 - yb0) * dx0)
    depth = np.where(chan, 8.0, depth)
    depth = np.maximum(depth, 2.0)
    zb = _fill_dummies(g, -depth)
    # lognormal Manning n on a smooth field (correlation ~12 parents)
    fld = _smooth_field((ny, nx), 12.0, rng)
    pi = np.clip((x / dx0).astype(np.int64), 0, nx - 1)
    pj = np.clip((y / dx0).astype(np.int64), 0, ny - 1)
    coefman = 0.025 * np.exp(0.2 * fld[pj, pi])
    th_cells, th_faces = _north_string(g)
    return Case("tidal_inlet", g, zb, coefman, th_cells, th_faces, [(0.6, M2_HOURS), (0.2, K1_HOURS)], dt, nsteps)


def tidal_flat(nx: int = 60, ny: int = 40, dx: float = 20.0, seed: int = 0, amp: float = 1.0, dt: float = 300.0,
               hours: float = 12.42, t0_hours: float = 0.0, refine: bool = False, manning: float = 0.025) -> Case:
    """Intertidal flat (see the module docstring).  With refine=True the grid is
    telescoping: parents of 2 dx with a refined (dx) zone around the creek, so
    that wet/dry fronts cross refinement interfaces."""
    rng = np.random.default_rng(seed)
    if refine:
        pnx, pny = max(4, nx // 2), max(4, ny // 2)
        lev = np.zeros((pny, pnx), dtype=np.int64)
        cx = pnx // 3
        lev[: max(2, (2 * pny) // 3), max(0, cx - pnx // 6): min(pnx, cx + pnx // 6 + 1)] = 1
        g = G.telescoping_grid(lev, 2.0 * dx, nmaxfaces=6)
    else:
        g = G.cartesian_grid(nx, ny, dx)
    n = g.ncells
    x, y = g.x[:n], g.y[:n]
    Lx, Ly = nx * dx, ny * dx
    depth = -1.0 + 4.0 * np.clip(y / Ly, 0.0, 1.0)
    fld = _smooth_field((ny, nx), 4.0, rng) * 0.15
    ii = np.clip((x / dx).astype(np.int64), 0, nx - 1)
    jj = np.clip((y / dx).astype(np.int64), 0, ny - 1)
    depth = depth + fld[jj, ii]
    # one-cell-wide creek from the shore to the middle of the flat
    xc = (nx // 3 + 0.5) * dx
    creek = (np.abs(x - xc) < 0.5 * dx) & (y < 0.55 * Ly)
    depth = np.where(creek, depth + 1.2, depth)
    # depression on the upper flat
    r2 = ((x - 0.7 * Lx) / (4.0 * dx)) ** 2 + ((y - 0.2 * Ly) / (4.0 * dx)) ** 2
    depth = depth + 1.4 * np.exp(-r2)
    zb = _fill_dummies(g, -depth)
    th_cells, th_faces = _north_string(g)
    return Case("tidal_flat", g, zb, np.full(n, manning), th_cells, th_faces, [(amp, M2_HOURS)], dt,
                int(round(hours * 3600.0 / dt)), t0=t0_hours * 3600.0)


def gauges(case: Case, count: int = 200, seed: int = 5, min_depth: float = 1.0) -> np.ndarray:
    """count seeded gauge cells (0-based active cell numbers, ascending):
    cells at least min_depth below mean sea level, away from the drying depth,
    so that a water-level gauge there stays wet."""
    n = case.grid.ncells
    ok = np.nonzero(-case.zb[:n] >= min_depth)[0]
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(ok, size=min(count, ok.size), replace=False)).astype(np.int64)
