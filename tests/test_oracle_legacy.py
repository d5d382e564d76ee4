"""CPU tests of the oracle's remaining MATRIX_SOLVER options (solvers.f90:242-289):
Gauss-Seidel (1), symmetric Gauss-Seidel / SSOR (2), the hybrid BiCGStab /
Gauss-Seidel switch (5), SIP (6), ICCG (7) and ICCGSTAB (8).

Each solver's fixed point is the direct solution of the system; the Gauss-
Seidel passes are also checked against a literal loop on a small grid, and the
dispatch (which branch runs for which variable index and residual) against the
sweep counts the reference sets.
"""
import numpy as np
import pytest
import scipy.sparse.linalg as spl

from cms2d_b200 import grid as G
from oracle import oracle as O
from tests.helpers import interior_matrix


def _copy(*a):
    return [np.array(x, copy=True) for x in a]


def symmetric_system(g, seed=0, dominance=1.02):
    """random_system with acoef(k,i) equal to the coefficient of the back face (symmetric matrix)."""
    acoef, ss, sp, phi = G.random_system(g, seed=seed, dominance=dominance)
    n = g.ncells
    for i in range(n):
        for k in range(int(g.ncface[i])):
            j = int(g.cell2cell[i, k]) - 1
            if j < i or j >= n:
                continue
            for kk in range(int(g.ncface[j])):
                if int(g.cell2cell[j, kk]) - 1 == i:
                    acoef[j, kk] = acoef[i, k]
    rowsum = acoef[:n].sum(axis=1)
    sp[:n] = -(dominance - 1.0) * rowsum
    return acoef, ss, sp, phi


def _solve(g, sysm, **kw):
    a, b, c, p = _copy(*sysm)
    res = np.zeros_like(b)
    out = O.OracleSolver(g).solve(a, b, c, res, p, **kw)
    return out, p, b


@pytest.mark.parametrize("nsolv,n,sweeps", [(1, 2, 400), (2, 2, 400), (2, 1, 400)])
def test_gauss_seidel_family_converges(nsolv, n, sweeps):
    g = G.cartesian_grid(20, 14)
    sysm = G.random_system(g, seed=2, dominance=1.3)
    out, p, _ = _solve(g, sysm, relax=1.0, nswp=sweeps, nsolv=nsolv, n=n, relaxsor=1.2)
    assert out["status"] == 0
    assert out["iters"] == (sweeps // 2 if nsolv == 2 else sweeps)
    A = interior_matrix(g, sysm[0], sysm[2])
    xs = spl.spsolve(A.tocsc(), sysm[1][: g.ncells])
    assert np.abs(p[: g.ncells] - xs).max() <= 1e-9 * np.abs(xs).max()


def _gs_loop(g, acoef, ap, su, phi, order, w=None):
    for i in order:
        t = 0.0
        for k in range(int(g.ncface[i])):
            t = t + acoef[i, k] * phi[int(g.cell2cell[i, k]) - 1]
        phi[i] = (t + su[i]) / ap[i] if w is None else w * (t + su[i]) / ap[i] + (1.0 - w) * phi[i]


@pytest.mark.parametrize("nsolv,n", [(1, 2), (2, 2), (2, 1)])
def test_gauss_seidel_passes_match_literal_loop(nsolv, n):
    g = G.cartesian_grid(6, 5)
    acoef, ss, sp, phi = G.random_system(g, seed=4)
    rng = np.random.default_rng(1)
    phi[:] = rng.standard_normal(g.ncellsD)
    relax, nswp, w = 0.8, 5, 1.6
    out, p, b = _solve(g, (acoef, ss, sp, phi), relax=relax, nswp=nswp, nsolv=nsolv, n=n, relaxsor=w)
    nn = g.ncells
    sa = np.zeros(nn)
    for k in range(g.nmaxfaces):  # face order, as the prologue sums
        sa = sa + acoef[:nn, k]
    ap = (sa - sp[:nn]) * (1.0 / relax)  # solvers.f90 multiplies by rinv = 1/relax
    su = ss.copy(); su[:nn] = ss[:nn] + (1.0 - relax) * phi[:nn] * ap
    np.testing.assert_array_equal(b[:nn], su[:nn])
    q = phi.copy()
    sor = nsolv == 2 and n == 1 and out["rmom"] < 1e-3
    fwd, bwd = range(nn), range(nn - 1, -1, -1)
    if nsolv == 1:
        for _ in range(nswp):
            _gs_loop(g, acoef, ap, su, q, fwd)
    else:
        for _ in range(nswp // 2):
            _gs_loop(g, acoef, ap, su, q, fwd, w if sor else None)
            _gs_loop(g, acoef, ap, su, q, bwd, w if sor else None)
    np.testing.assert_allclose(p[:nn], q[:nn], rtol=1e-14, atol=1e-14)


def test_hybrid_dispatch():
    """nsolv=5: BiCGStab for the pressure correction while rmom(1) > 1e-4, else
    Gauss-Seidel with 4 nswp sweeps (n <= 3) or 3 nswp0(2) sweeps (n = 4, 5),
    SOR for the pressure correction (solvers.f90:255-272)."""
    g = G.cartesian_grid(16, 12)
    sysm = G.random_system(g, seed=6, dominance=1.2)
    out, _, _ = _solve(g, sysm, relax=1.0, nswp=20, nsolv=5, n=1, tol=1e-3)
    assert out["rmom"] > 1e-4 and 1 <= out["iters"] <= 20 and out["relres"] < 1e-3  # BiCGStab
    for n, expect in ((2, 4 * 5), (3, 4 * 5), (4, 3 * 7), (5, 3 * 7)):
        out, _, _ = _solve(g, sysm, relax=0.8, nswp=5, nsolv=5, n=n, nswp0_vel=7)
        assert out["iters"] == expect, (n, out)
    # pressure correction once the residual is small: SOR with 4 nswp sweeps
    a, b, c, p = _copy(*sysm)
    A = interior_matrix(g, a, c)
    p[: g.ncells] = spl.spsolve(A.tocsc(), b[: g.ncells]) * (1 + 1e-9)
    res = np.zeros_like(b)
    out = O.OracleSolver(g).solve(a, b, c, res, p, relax=1.0, nswp=20, nsolv=5, n=1, relaxsor=1.5)
    assert out["rmom"] < 1e-4 and out["iters"] == 80


@pytest.mark.parametrize("nsolv,n", [(6, 1), (6, 2), (7, 1), (7, 2), (8, 1), (8, 5)])
def test_five_point_solvers_converge(nsolv, n):
    g = G.cartesian_grid(30, 22)
    sysm = symmetric_system(g, seed=8, dominance=1.05) if n == 1 else G.random_system(g, seed=8, dominance=1.05)
    out, p, _ = _solve(g, sysm, relax=1.0, nswp=400, nsolv=nsolv, n=n)
    assert out["status"] == 0
    assert out["relres"] < 1e-3
    A = interior_matrix(g, sysm[0], sysm[2])
    xs = spl.spsolve(A.tocsc(), sysm[1][: g.ncells])
    assert np.abs(p[: g.ncells] - xs).max() <= 2e-2 * np.abs(xs).max()
    # more than nswp/2 iterations before the SIP/ICCG test may stop
    if nsolv in (6, 7) or n == 1:
        assert out["iters"] > 200


def test_five_point_solvers_need_compass_faces():
    g = G.solver_test_grid(2000)  # telescoping: up to 6 faces per cell
    assert int(g.ncface[: g.ncells].max()) > 4
    sysm = G.random_system(g, seed=1)
    for nsolv in (6, 7, 8):
        out, _, _ = _solve(g, sysm, relax=1.0, nswp=10, nsolv=nsolv, n=1)
        assert out["status"] == -1
