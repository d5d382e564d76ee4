"""Model check of the pipelined-pass protocol of k_gs_pipe (cms_legacy.cuh).

Work units are chunks of one level set; a unit of pass h may run once every
row in it sees: couplings on the pass's new side done with pass h, couplings
on the old side and the row itself done with pass h-1.  Here units run in
random orders among those that are ready (a stronger adversary than the
kernel's in-order claims): every run must finish, and every row must complete
its passes in order -- with forward-only and with alternating (symmetric
Gauss-Seidel) passes.  Without the row's wait on itself, alternating passes
let a row start a pass before finishing the previous one, which the check
must catch.
"""
import random

import numpy as np
import pytest

from cms2d_b200 import grid as G


def _schedule(g, chunk=8):
    n = g.ncells
    nb = [[int(c) - 1 for c in g.cell2cell[i, : g.ncface[i]] if 1 <= c <= n] for i in range(n)]
    lev = np.zeros(n, dtype=np.int64)
    for i in range(n):
        lev[i] = 1 + max([lev[j] for j in nb[i] if j < i], default=-1)
    order = np.lexsort((np.arange(n), lev))
    pos = np.empty(n, dtype=np.int64)
    pos[order] = np.arange(n)
    gstart = np.searchsorted(lev[order], np.arange(lev.max() + 2))
    cs = [r for gi in range(len(gstart) - 1) for r in range(gstart[gi], gstart[gi + 1], chunk)] + [n]
    lower = [[pos[j] for j in nb[order[r]] if j < order[r]] for r in range(n)]
    upper = [[pos[j] for j in nb[order[r]] if j > order[r]] for r in range(n)]
    return cs, lower, upper


def _run(cs, lower, upper, npass, sym, self_wait, seed):
    n = len(lower)
    nch = len(cs) - 1
    done = np.zeros(n, dtype=np.int64)
    pending = list(range(npass * nch))
    rnd = random.Random(seed)
    in_order = True

    def unit(t):
        h, c0 = divmod(t, nch)
        bwd = bool(sym and (h & 1))
        c = nch - 1 - c0 if bwd else c0
        return h, bwd, range(cs[c], cs[c + 1])

    while pending:
        ready = []
        for t in pending[:4 * nch]:
            h, bwd, rows = unit(t)
            mine = h + 1
            ok = all((not self_wait or done[r] >= mine - 1)
                     and all(done[j] >= (mine - 1 if bwd else mine) for j in lower[r])
                     and all(done[j] >= (mine if bwd else mine - 1) for j in upper[r]) for r in rows)
            if ok:
                ready.append(t)
        if not ready:
            return False, in_order
        t = rnd.choice(ready)
        pending.remove(t)
        h, _, rows = unit(t)
        for r in rows:
            in_order &= bool(done[r] == h)
            done[r] = h + 1
    return True, in_order


@pytest.mark.parametrize("kind", ["cart", "tel"])
@pytest.mark.parametrize("sym", [0, 1])
def test_pipelined_passes_finish_in_order(kind, sym):
    g = G.cartesian_grid(9, 7) if kind == "cart" else G.solver_test_grid(150)
    cs, lower, upper = _schedule(g)
    for seed in range(8):
        finished, in_order = _run(cs, lower, upper, 6, sym, True, seed)
        assert finished and in_order, seed


def test_alternating_passes_need_the_self_wait():
    cs, lower, upper = _schedule(G.cartesian_grid(9, 7))
    results = [_run(cs, lower, upper, 6, 1, False, seed) for seed in range(8)]
    assert any(not (fin and ordered) for fin, ordered in results)
