"""CPU tests of the oracle (the checker) and of the host-side ordering logic."""
import numpy as np
import pytest
import scipy.sparse.linalg as spl

from cms2d_b200 import grid as G
from cms2d_b200 import solver as S
from oracle import oracle as O
from tests.helpers import interior_matrix, permute_system, permuted_grid


def _copy(*a):
    return [np.array(x, copy=True) for x in a]


@pytest.mark.parametrize("nsolv", [3, 4])
@pytest.mark.parametrize("pc", [O.PC_ILU0, O.PC_ILUTP])
@pytest.mark.parametrize("kind", ["cart", "tel"])
def test_oracle_matches_direct_solve(nsolv, pc, kind):
    g = G.cartesian_grid(40, 25) if kind == "cart" else G.solver_test_grid(3000)
    acoef, ss, sp, phi = G.random_system(g, seed=3)
    A = interior_matrix(g, acoef, sp)
    xs = spl.spsolve(A.tocsc(), ss[: g.ncells])
    o = O.OracleSolver(g)
    a, b, c, p = _copy(acoef, ss, sp, phi)
    res = np.zeros_like(b)
    out = o.solve(a, b, c, res, p, relax=1.0, nswp=400, nsolv=nsolv, precond=pc, tol=1e-9)
    assert out["status"] == 0
    assert np.abs(p[: g.ncells] - xs).max() <= 1e-6 * np.abs(xs).max()


def test_oracle_prologue_relaxation():
    """solve() prologue: ap, ss under-relaxation and the normalised residual (solvers.f90:233-240)."""
    g = G.cartesian_grid(12, 9)
    acoef, ss, sp, phi = G.random_system(g, seed=5)
    rng = np.random.default_rng(0)
    phi[:] = rng.standard_normal(g.ncellsD)
    relax = 0.8
    n = g.ncells
    ap = (acoef[:n].sum(1) - sp[:n]) / relax
    ss_exp = ss[:n] + (1 - relax) * phi[:n] * ap
    nb = np.where(np.arange(4)[None, :] < g.ncface[:n, None], g.cell2cell[:n] - 1, 0)
    res_exp = ((acoef[:n] * phi[nb]).sum(1) + ss_exp - ap * phi[:n]) / ap
    a, b, c, p = _copy(acoef, ss, sp, phi)
    res = np.zeros_like(b)
    out = O.OracleSolver(g).solve(a, b, c, res, p, relax=relax, nswp=0, nsolv=3, precond=O.PC_ILU0)
    np.testing.assert_allclose(b[:n], ss_exp, rtol=1e-14, atol=1e-14)
    np.testing.assert_allclose(res[:n], res_exp, rtol=1e-12, atol=1e-14)
    assert abs(out["rmom"] - np.sqrt((res_exp ** 2).sum() / n)) <= 1e-12 * out["rmom"]


def test_oracle_fp32_close_to_fp64():
    g = G.solver_test_grid(2000)
    acoef, ss, sp, phi = G.random_system(g, seed=7)
    o = O.OracleSolver(g)
    a, b, c, p = _copy(acoef, ss, sp, phi)
    r = np.zeros_like(b)
    o.solve(a, b, c, r, p, nswp=50, nsolv=3, precond=O.PC_ILU0, tol=1e-5)
    a32, b32, c32, p32 = [x.astype(np.float32) for x in (acoef, ss, sp, phi)]
    r32 = np.zeros_like(b32)
    o.solve(a32, b32, c32, r32, p32, nswp=50, nsolv=3, precond=O.PC_ILU0, tol=1e-5)
    assert np.abs(p32 - p).max() <= 1e-4 * np.abs(p).max()


def test_indexm_last_cell_quirk():
    """indexm's `nterm1 = ncells` bound (sparse.f90:46-49) drops the coupling to cell ncells."""
    nx, ny = 6, 4
    g = G.cartesian_grid(nx, ny)
    n = g.ncells
    ia_q, ja_q = O.OracleSolver(g, fix_last_cell=False).pattern()
    ia_f, ja_f = O.OracleSolver(g, fix_last_cell=True).pattern()
    assert ia_q[-1] == ia_f[-1]  # same number of stored entries
    # rows n-1 (east neighbour n) and n-nx (north neighbour n), 1-based
    for row in (n - 1, n - nx):
        q = ja_q[ia_q[row - 1] - 1: ia_q[row] - 1]
        f = ja_f[ia_f[row - 1] - 1: ia_f[row] - 1]
        assert n in f and n not in q
    # every other row is identical
    for row in range(1, n + 1):
        if row in (n - 1, n - nx):
            continue
        assert list(ja_q[ia_q[row - 1] - 1: ia_q[row] - 1]) == list(ja_f[ia_f[row - 1] - 1: ia_f[row] - 1])


def test_indexm_quirk_still_converges():
    g = G.cartesian_grid(30, 20)
    acoef, ss, sp, phi = G.random_system(g, seed=11)
    its = []
    for fix in (False, True):
        a, b, c, p = _copy(acoef, ss, sp, phi)
        r = np.zeros_like(b)
        out = O.OracleSolver(g, fix_last_cell=fix).solve(a, b, c, r, p, nswp=100, nsolv=3, precond=O.PC_ILU0, tol=1e-8)
        assert out["status"] == 0 and out["relres"] < 1e-8
        its.append(out["iters"])
    assert abs(its[0] - its[1]) <= 2


def test_manufactured_solution():
    """Known answer: x* chosen, b = A x*, solved to 1e-12 (L1 ratio)."""
    g = G.solver_test_grid(4000)
    acoef, _, sp, phi = G.random_system(g, seed=2)
    A = interior_matrix(g, acoef, sp)
    xstar = np.sin(np.arange(g.ncells) * 0.01) + 2.0
    ss = np.zeros(g.ncellsD); ss[: g.ncells] = A @ xstar
    a, b, c, p = _copy(acoef, ss, sp, phi)
    r = np.zeros_like(b)
    out = O.OracleSolver(g).solve(a, b, c, r, p, nswp=300, nsolv=4, precond=O.PC_ILU0, tol=1e-12)
    assert out["status"] == 0
    np.testing.assert_allclose(p[: g.ncells], xstar, rtol=1e-9)


# ---- host-side ordering (C-ABI cms_order_build; no device calls) ----

@pytest.mark.parametrize("kind", ["cart", "tel"])
@pytest.mark.parametrize("ordering", ["multicolor", "natural"])
def test_groups_are_independent_sets(kind, ordering):
    g = G.cartesian_grid(33, 17) if kind == "cart" else G.solver_test_grid(5000)
    perm, gstart, (KL, KU) = S.order_build(g, ordering)
    n = g.ncells
    assert sorted(perm.tolist()) == list(range(n))
    grp = np.empty(n, np.int64)
    for q in range(len(gstart) - 1):
        grp[perm[gstart[q]:gstart[q + 1]]] = q
    for k in range(g.nmaxfaces):
        c = g.cell2cell[:n, k]
        m = (k < g.ncface[:n]) & (c >= 1) & (c <= n)
        i = np.nonzero(m)[0]
        assert np.all(grp[i] != grp[c[m] - 1])
    if ordering == "multicolor" and kind == "cart":
        assert len(gstart) - 1 == 2 and KL == 4 and KU == 4
    if ordering == "natural":
        # natural order is preserved inside each level and every lower neighbour sits in an earlier level
        for k in range(g.nmaxfaces):
            c = g.cell2cell[:n, k]
            m = (k < g.ncface[:n]) & (c >= 1) & (c <= n)
            i = np.nonzero(m)[0]
            lower = (c[m] - 1) < i
            assert np.all(grp[c[m][lower] - 1] < grp[i[lower]])


def test_level_order_is_natural_ilu0():
    """ILU(0) in level order equals natural-order ILU(0) up to rounding (the GPU's natural mode)."""
    g = G.solver_test_grid(3000)
    acoef, ss, sp, phi = G.random_system(g, seed=4)
    perm, _, _ = S.order_build(g, "natural")
    o_nat = O.OracleSolver(g)
    a, b, c, p = _copy(acoef, ss, sp, phi)
    r = np.zeros_like(b)
    o_nat.solve(a, b, c, r, p, nswp=0, nsolv=3, precond=O.PC_ILU0)  # builds the factor
    gp, order = permuted_grid(g, perm)
    o_lev = O.OracleSolver(gp)
    a2, b2, c2, p2 = permute_system(order, acoef, ss, sp, phi)
    r2 = np.zeros_like(b2)
    o_lev.solve(a2, b2, c2, r2, p2, nswp=0, nsolv=3, precond=O.PC_ILU0)
    y = np.random.default_rng(0).standard_normal(g.ncells)
    x_nat = o_nat.lusol(y)
    x_lev = o_lev.lusol(y[perm])
    np.testing.assert_allclose(x_lev, x_nat[perm], rtol=1e-12, atol=1e-13)


def test_multicolor_iteration_counts_reported():
    """Multicolour ILU(0) is a different preconditioner; it still converges (counts compared in bench)."""
    g = G.cartesian_grid(64, 48)
    acoef, ss, sp, phi = G.random_system(g, seed=9)
    perm, _, _ = S.order_build(g, "multicolor")
    gp, order = permuted_grid(g, perm)
    counts = {}
    for name, gg, arrs in (("natural", g, (acoef, ss, sp, phi)), ("multicolor", gp, permute_system(order, acoef, ss, sp, phi))):
        a, b, c, p = _copy(*arrs)
        r = np.zeros_like(b)
        out = O.OracleSolver(gg).solve(a, b, c, r, p, nswp=200, nsolv=3, precond=O.PC_ILU0, tol=1e-6)
        assert out["status"] == 0 and out["relres"] < 1e-6
        counts[name] = out["iters"]
    assert counts["multicolor"] <= 3 * counts["natural"] + 5
