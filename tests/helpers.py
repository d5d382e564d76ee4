"""Shared test helpers (system assembly, permutations)."""
from __future__ import annotations

import numpy as np
import scipy.sparse as sps

from cms2d_b200 import grid as G


def interior_matrix(g, acoef, sp, relax=1.0):
    """A = diag(ap) - offdiag(acoef) over active cells (ghost terms excluded)."""
    n = g.ncells
    ap = (acoef[:n].sum(axis=1) - sp[:n]) / relax
    rows, cols, vals = [np.arange(n)], [np.arange(n)], [ap]
    for k in range(g.nmaxfaces):
        c = g.cell2cell[:n, k]
        m = (k < g.ncface[:n]) & (c >= 1) & (c <= n)
        rows.append(np.nonzero(m)[0]); cols.append(c[m] - 1); vals.append(-acoef[:n, k][m])
    return sps.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))


def permuted_grid(g, perm):
    """Renumbers active cells: new cell r is old cell perm[r] (ghosts keep their ids)."""
    n = g.ncells
    iperm = np.empty(n, np.int64); iperm[perm] = np.arange(n)
    remap = np.arange(g.ncellsD + 1, dtype=np.int64)  # 1-based old -> new
    remap[1:n + 1] = iperm + 1
    c2c = g.cell2cell.astype(np.int64)
    new = np.zeros_like(g.cell2cell)
    act = np.asarray(perm)
    new[:n] = remap[c2c[act]] * (c2c[act] > 0)
    new[n:] = remap[c2c[n:]] * (c2c[n:] > 0)
    ncf = g.ncface.copy(); ncf[:n] = g.ncface[act]
    order = np.concatenate([act, np.arange(n, g.ncellsD)])
    return G.Grid(ncells=n, ncellsD=g.ncellsD, nmaxfaces=g.nmaxfaces, cell2cell=new.astype(np.int32),
                  ncface=ncf.astype(np.int32), idirface=g.idirface[order], x=g.x[order], y=g.y[order],
                  dx=g.dx[order], dy=g.dy[order], level=g.level[order], telescoping=g.telescoping), order


def permute_system(order, *arrs):
    return [np.ascontiguousarray(a[order]) for a in arrs]
