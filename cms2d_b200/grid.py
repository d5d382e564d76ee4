"""Cartesian and telescoping (quadtree) grids in the CMS-Flow in-memory layout.

The arrays produced here are the ones the reference builds when it reads a grid:

* ``cell2cell[i, k]`` (0-based row ``i``, face slot ``k``) holds the 1-based
  neighbour index of cell ``i+1`` across face ``k+1``; active cells are
  ``1..ncells`` and dummy (ghost) cells ``ncells+1..ncellsD`` are appended
  after them.  Faces are listed in the order n1,n2,e1,e2,s1,s2,w1,w2 of a
  ``.tel`` row with absent entries skipped (source/geospatial/geospatial.F90:
  437-453 for the row format, 556-741 for the face/dummy construction), so a
  regular cell has faces N,E,S,W exactly as the Cartesian builder assigns them
  (geospatial.F90:2840-2945).
* A dummy cell gets ``ncface = 4`` and a single back link on the opposite face
  (geospatial.F90:573-716), plus a position and size (used by the face
  metrics).
* Cell order is the natural order: row-major by the lower-left corner on the
  finest lattice (Cartesian grids: ``id = i + (j-1)*maxcol``,
  geospatial.F90:2729-2837).

The telescoping generator works on a coarse lattice of ``nbx x nby`` parent
cells of size ``dx0``; a parent at refinement level ``L`` is split into
``2**L x 2**L`` leaf cells.  Adjacent parents must differ by at most one
level, which bounds every leaf at two neighbours per side and six faces in
total (``nmaxfaces = 6`` as in read_tel, geospatial.F90:433).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

# Face direction codes (idirface): 1 north, 2 east, 3 south, 4 west.
N_, E_, S_, W_ = 1, 2, 3, 4


@dataclass
class Grid:
    ncells: int
    ncellsD: int
    nmaxfaces: int
    cell2cell: np.ndarray  # int32 [ncellsD, nmaxfaces], 1-based, 0 = none
    ncface: np.ndarray     # int32 [ncellsD]
    idirface: np.ndarray   # int32 [ncellsD, nmaxfaces]
    x: np.ndarray          # float64 [ncellsD] cell centres (local coordinates)
    y: np.ndarray
    dx: np.ndarray
    dy: np.ndarray
    level: np.ndarray      # int8 [ncellsD] refinement level (dummies copy their parent's size)
    # lower-left corner and size on the finest lattice (active cells only)
    fx: np.ndarray = field(default=None, repr=False)
    fy: np.ndarray = field(default=None, repr=False)
    fs: np.ndarray = field(default=None, repr=False)
    telescoping: bool = False

    @property
    def nfaces_total(self) -> int:
        return int(self.ncface[: self.ncells].sum())

    def interior_faces(self) -> int:
        """Faces between two active cells (counted once per direction)."""
        c = self.cell2cell[: self.ncells]
        mask = (np.arange(self.nmaxfaces)[None, :] < self.ncface[: self.ncells, None]) & (c >= 1) & (c <= self.ncells)
        return int(mask.sum())


def _owner_lookup(fx, fy, fs, ids, W, H):
    owner = np.zeros((H, W), dtype=np.int64)  # 0 = none
    # paint each leaf on the fine lattice; leaves of size s cover s*s points
    for s in np.unique(fs):
        sel = fs == s
        xs, ys, cid = fx[sel], fy[sel], ids[sel]
        for dy_ in range(s):
            for dx_ in range(s):
                owner[ys + dy_, xs + dx_] = cid
    return owner


def _lookup(owner, xx, yy):
    H, W = owner.shape
    ok = (xx >= 0) & (xx < W) & (yy >= 0) & (yy < H)
    out = np.zeros(xx.shape, dtype=np.int64)
    out[ok] = owner[yy[ok], xx[ok]]
    return out


def _leaves(level: np.ndarray):
    """All leaves of a parent-level map on the finest lattice, row-major by
    lower-left corner (y, then x): corners fx, fy, size fs (lattice units)."""
    level = np.asarray(level, dtype=np.int64)
    nby, nbx = level.shape
    # 2:1 balance between edge-adjacent parents
    if np.any(np.abs(np.diff(level, axis=0)) > 1) or np.any(np.abs(np.diff(level, axis=1)) > 1):
        raise ValueError("adjacent parent cells differ by more than one refinement level")
    lmax = int(level.max())
    R = 1 << lmax  # fine lattice points per parent side
    fxl, fyl, fsl = [], [], []
    for L in range(lmax + 1):
        jj, ii = np.nonzero(level == L)
        if ii.size == 0:
            continue
        n = 1 << L
        s = R >> L
        a, b = np.meshgrid(np.arange(n), np.arange(n), indexing="xy")
        a = a.ravel(); b = b.ravel()
        fxl.append((ii[:, None] * R + a[None, :] * s).ravel())
        fyl.append((jj[:, None] * R + b[None, :] * s).ravel())
        fsl.append(np.full(ii.size * n * n, s, dtype=np.int64))
    fx = np.concatenate(fxl); fy = np.concatenate(fyl); fs = np.concatenate(fsl)
    order = np.lexsort((fx, fy))  # row-major: y then x
    return fx[order], fy[order], fs[order], lmax, R, nbx * R, nby * R


def _neighbour_slots(owner, fx, fy, fs):
    """The .tel neighbour slots n1,n2,e1,e2,s1,s2,w1,w2 of each leaf from the
    lattice owner map (the second of a pair is 0 unless the side is split
    between two finer neighbours)."""
    x0, y0, s = fx, fy, fs
    loc = np.zeros((fx.size, 8), dtype=np.int64)
    pairs = [
        ((x0, y0 + s), (x0 + s - 1, y0 + s)),          # north: west half, east half
        ((x0 + s, y0 + s - 1), (x0 + s, y0)),          # east: north half, south half
        ((x0 + s - 1, y0 - 1), (x0, y0 - 1)),          # south: east half, west half
        ((x0 - 1, y0), (x0 - 1, y0 + s - 1)),          # west: south half, north half
    ]
    for side, ((ax, ay), (bx, by)) in enumerate(pairs):
        n1 = _lookup(owner, ax, ay)
        n2 = _lookup(owner, bx, by)
        n2 = np.where(n2 == n1, 0, n2)
        loc[:, 2 * side] = n1
        loc[:, 2 * side + 1] = n2
    return loc


def assemble(loc, xc, yc, dxc, dyc, nmaxfaces: int | None = None, level=None, telescoping: bool = False,
             fx=None, fy=None, fs=None) -> Grid:
    """read_tel's second pass (source/geospatial/geospatial.F90:540-741) for the
    active cells of a grid: loc[i, j] is the neighbour of active cell i in .tel
    slot j (n1,n2,e1,e2,s1,s2,w1,w2) as an active id (1-based), -1 for an
    inactive (land) cell, 0 for none.  xc, yc, dxc, dyc: cell centres and
    sizes.  A side with no active neighbour gets one dummy in its first slot,
    an inactive half of a split side its own dummy, active neighbours internal
    faces; dummies are numbered in cell order then slot order, with ncface 4,
    a back link on the opposite face and the position and size read_tel gives
    them (half size when the side is split)."""
    loc = np.asarray(loc, dtype=np.int64)
    ncells = loc.shape[0]
    slot_kind = np.zeros((ncells, 8), dtype=np.int8)  # 0 none, 1 internal, 2 dummy
    for q in range(4):
        a1, a2 = loc[:, 2 * q], loc[:, 2 * q + 1]
        has = (a1 > 0) | (a2 > 0)
        slot_kind[:, 2 * q] = np.where(has, np.where(a1 > 0, 1, np.where(a1 < 0, 2, 0)), 2)
        slot_kind[:, 2 * q + 1] = np.where(has, np.where(a2 > 0, 1, np.where(a2 < 0, 2, 0)), 0)
    nf = (slot_kind > 0).sum(axis=1)
    nmf_needed = int(nf.max()) if ncells else 4
    if nmaxfaces is None:
        nmaxfaces = 4 if (nmf_needed <= 4 and not telescoping) else 6
    if nmf_needed > nmaxfaces:
        raise ValueError(f"a cell has {nmf_needed} faces > nmaxfaces={nmaxfaces}")
    ndummy = int((slot_kind == 2).sum())
    ncellsD = ncells + ndummy
    cell2cell = np.zeros((ncellsD, nmaxfaces), dtype=np.int32)
    idirface = np.zeros((ncellsD, nmaxfaces), dtype=np.int32)
    ncface = np.zeros(ncellsD, dtype=np.int32)
    ncface[:ncells] = nf
    dmask = slot_kind == 2
    dnum = np.cumsum(dmask.ravel()).reshape(dmask.shape) + ncells  # 1-based id for dummy slots
    present = slot_kind > 0
    kpos = np.cumsum(present, axis=1) - 1
    rows, slots = np.nonzero(present)
    kk = kpos[rows, slots]
    vals = np.where(slot_kind[rows, slots] == 2, dnum[rows, slots], loc[rows, slots])
    cell2cell[rows, kk] = vals
    idirface[rows, kk] = slots // 2 + 1
    X = np.zeros(ncellsD); Y = np.zeros(ncellsD); DX = np.zeros(ncellsD); DY = np.zeros(ncellsD)
    LEV = np.zeros(ncellsD, dtype=np.int8)
    X[:ncells] = xc; Y[:ncells] = yc; DX[:ncells] = dxc; DY[:ncells] = dyc
    if level is not None:
        LEV[:ncells] = level
    dr, dsl = np.nonzero(dmask)
    did = dnum[dr, dsl] - 1  # 0-based row of the dummy
    side = dsl // 2 + 1
    back = {1: 3, 2: 4, 3: 1, 4: 2}
    ncface[did] = 4
    for q in (1, 2, 3, 4):
        m = side == q
        cell2cell[did[m], back[q] - 1] = dr[m] + 1
    partner = loc[dr, dsl ^ 1]  # the other slot of the pair
    split = partner > 0
    # full-size offsets per side and half-size offsets per slot, in units of
    # the cell's own dx (x) and dy (y)
    full = {1: (0.0, 1.0), 2: (1.0, 0.0), 3: (0.0, -1.0), 4: (-1.0, 0.0)}
    half = {0: (-0.25, 0.75), 1: (0.25, 0.75), 2: (0.75, 0.25), 3: (0.75, -0.25),
            4: (0.25, -0.75), 5: (-0.25, -0.75), 6: (-0.75, -0.25), 7: (-0.75, 0.25)}
    ofx = np.array([full[q][0] for q in side]) if side.size else np.zeros(0)
    ofy = np.array([full[q][1] for q in side]) if side.size else np.zeros(0)
    hfx = np.array([half[j][0] for j in dsl]) if dsl.size else np.zeros(0)
    hfy = np.array([half[j][1] for j in dsl]) if dsl.size else np.zeros(0)
    sx, sy = np.asarray(dxc)[dr], np.asarray(dyc)[dr]
    X[did] = np.asarray(xc)[dr] + np.where(split, hfx, ofx) * sx
    Y[did] = np.asarray(yc)[dr] + np.where(split, hfy, ofy) * sy
    DX[did] = np.where(split, 0.5, 1.0) * sx
    DY[did] = np.where(split, 0.5, 1.0) * sy
    LEV[did] = LEV[dr] + split.astype(np.int8)
    return Grid(ncells=ncells, ncellsD=ncellsD, nmaxfaces=nmaxfaces, cell2cell=cell2cell, ncface=ncface,
                idirface=idirface, x=X, y=Y, dx=DX, dy=DY, level=LEV, fx=fx, fy=fy, fs=fs,
                telescoping=telescoping)


def telescoping_grid(level: np.ndarray, dx0: float, active=None, nmaxfaces: int | None = None) -> Grid:
    """Builds a telescoping grid from a parent-level map.

    level:  int array [nby, nbx] of refinement levels (0 = parent size dx0).
    active: optional callable (xc, yc, size) -> bool array selecting active leaves
            (inactive leaves are land: depth -999 in a .tel file).
    """
    fx, fy, fs, lmax, R, W, H = _leaves(level)
    h = dx0 / R  # fine lattice spacing
    xc = (fx + 0.5 * fs) * h
    yc = (fy + 0.5 * fs) * h
    keep = np.ones(fx.size, dtype=bool)
    if active is not None:
        keep = np.asarray(active(xc, yc, fs * h), dtype=bool)
    # inactive (land) leaves are painted -1 so that their sides get dummies
    owner = _owner_lookup(fx[~keep], fy[~keep], fs[~keep], np.full(int((~keep).sum()), -1, dtype=np.int64), W, H)
    fx, fy, fs, xc, yc = fx[keep], fy[keep], fs[keep], xc[keep], yc[keep]
    ncells = fx.size
    ids = np.arange(1, ncells + 1, dtype=np.int64)
    act = _owner_lookup(fx, fy, fs, ids, W, H)
    owner = np.where(act > 0, act, owner)
    del act
    loc = _neighbour_slots(owner, fx, fy, fs)
    size = fs * h
    lev = (lmax - np.log2(fs).astype(np.int64)).astype(np.int8)
    return assemble(loc, xc, yc, size, size, nmaxfaces=nmaxfaces, level=lev, telescoping=lmax > 0, fx=fx, fy=fy,
                    fs=fs)


def cartesian_grid(nx: int, ny: int, dx: float = 20.0, active=None) -> Grid:
    """Uniform Cartesian grid (nmaxfaces = 4), natural order id = i + (j-1)*nx."""
    return telescoping_grid(np.zeros((ny, nx), dtype=np.int64), dx, active=active, nmaxfaces=4)


def refinement_rectangles(nbx: int, nby: int, rects) -> np.ndarray:
    """Parent-level map from nested rectangles [(level, x0, y0, x1, y1)] in parent units."""
    lev = np.zeros((nby, nbx), dtype=np.int64)
    for L, x0, y0, x1, y1 in rects:
        lev[max(y0, 0):min(y1, nby), max(x0, 0):min(x1, nbx)] = np.maximum(
            lev[max(y0, 0):min(y1, nby), max(x0, 0):min(x1, nbx)], L)
    return lev


def solver_test_grid(n_target: int, seed: int = 0) -> Grid:
    """Telescoping grid of about n_target active cells for the solver sweep.

    A square parent lattice with a band of once-refined parents across the
    middle third, so that the stencil is 5-point away from the interfaces and
    has up to two extra neighbours per face along them.
    """
    # the refined band covers 1/3 of the parents and holds 4 leaves each:
    # n = P * (2/3 + 4/3) = 2 P  ->  P = n/2 parents
    P = max(n_target // 2, 16)
    nb = int(round(np.sqrt(P)))
    lev = np.zeros((nb, nb), dtype=np.int64)
    lev[nb // 3: 2 * nb // 3, :] = 1
    return telescoping_grid(lev, 20.0, nmaxfaces=6)


def random_system(g: Grid, seed: int = 0, dominance: float = 1.02, dtype=np.float64):
    """Seeded solver-sweep system on grid g in the solve() argument layout.

    Off-diagonal coefficients acoef(k,i) ~ U[0.1, 1] (so A's off-diagonals lie in
    [-1, -0.1]); the diagonal ap = dominance * sum_k acoef(k,i) is produced by
    solve() from sp = -(dominance-1) * sum_k acoef(k,i) at relax = 1; the RHS
    ss ~ N(0,1).  Ghost neighbours carry phi = 0.
    Returns (acoef[ncellsD, nmaxfaces], ss[ncellsD], sp[ncellsD], phi[ncellsD]).
    """
    rng = np.random.default_rng(seed)
    nD, nmf = g.ncellsD, g.nmaxfaces
    acoef = np.zeros((nD, nmf), dtype=np.float64)
    mask = np.arange(nmf)[None, :] < g.ncface[:, None]
    mask[g.ncells:] = False
    acoef[mask] = rng.uniform(0.1, 1.0, size=int(mask.sum()))
    rowsum = acoef.sum(axis=1)
    sp = np.zeros(nD); sp[: g.ncells] = -(dominance - 1.0) * rowsum[: g.ncells]
    ss = np.zeros(nD); ss[: g.ncells] = rng.standard_normal(g.ncells)
    phi = np.zeros(nD)
    return acoef.astype(dtype), ss.astype(dtype), sp.astype(dtype), phi.astype(dtype)
