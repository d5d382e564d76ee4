"""GPU parity of the MATRIX_SOLVER options other than BiCGStab and GMRES
(solvers.f90:242-289) against the CPU oracle, same inputs, same unknown order.

The oracle runs the reference's serial loops on the system renumbered into the
GPU's device order: in the natural (level-scheduled) ordering that is the
reference's own order of every recurrence; in the multicolour ordering it is
the multicolour form of the same method, which the GPU runs one colour per
launch.  Tolerances: FP64 solution within 1e-10 of the oracle's (relative to
its largest value), the same iteration or sweep count and rmom to 1e-12
relative; FP32 within 2e-4.
"""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse.linalg as spl

from cms2d_b200 import _lib
from cms2d_b200 import grid as G
from cms2d_b200 import solver as S
from oracle import oracle as O
from tests.helpers import interior_matrix, permute_system, permuted_grid
from tests.test_oracle_legacy import symmetric_system

pytestmark = pytest.mark.gpu


def _copy(*a):
    return [np.array(x, copy=True) for x in a]


def _grid(kind):
    return G.cartesian_grid(37, 23) if kind == "cart" else G.solver_test_grid(5000)


def _near_solution(g, sysm, scale=1e-7, relax=1.0):
    """phi close to the solution, so that rmom < 1e-3 (SSOR / SOR branches)."""
    a, b, c, p = _copy(*sysm)
    x = spl.spsolve(interior_matrix(g, a, c, relax).tocsc(), b[: g.ncells])
    p[: g.ncells] = x * (1.0 + scale * np.random.default_rng(3).standard_normal(g.ncells))
    return a, b, c, p


def _compare(g, s, sysm, n, nsolv, nswp, relax, tol_rel=1e-10, **okw):
    a, b, c, p = _copy(*sysm)
    res = np.zeros_like(b)
    info = s.solve(a, b, c, res, p, n=n, relax=relax, nswp=nswp, nsolv=nsolv, raise_on_error=False)
    gp, order = permuted_grid(g, s.perm())
    ao, bo, co, po = permute_system(order, *sysm)
    ro = np.zeros_like(bo)
    out = O.OracleSolver(gp, fix_last_cell=True).solve(ao, bo, co, ro, po, relax=relax, nswp=nswp, nsolv=nsolv,
                                                      precond=O.PC_ILU0, n=n, **okw)
    inv = np.empty_like(order); inv[order] = np.arange(order.size)
    nn = g.ncells
    assert info["iters"] == out["iters"], (info, out)
    # near the solution rmom is a cancellation; 1e-15 absolute covers its rounding
    assert abs(info["rmom"] - out["rmom"]) <= 1e-12 * out["rmom"] + 1e-15
    np.testing.assert_allclose(b[:nn], bo[inv][:nn], rtol=1e-13, atol=1e-13)
    err = np.abs(p[:nn] - po[inv][:nn]).max() / np.abs(po[inv][:nn]).max()
    assert err <= tol_rel, err
    return info, out


@pytest.mark.parametrize("kind", ["cart", "tel"])
@pytest.mark.parametrize("ordering", ["natural", "multicolor"])
@pytest.mark.parametrize("nsolv,n", [(1, 2), (2, 2), (2, 1), (5, 2), (5, 4), (5, 1)])
def test_gauss_seidel_family(kind, ordering, nsolv, n):
    g = _grid(kind)
    sysm = G.random_system(g, seed=13, dominance=1.1)
    relax = 1.0 if n == 1 else 0.8
    if n == 1:  # SSOR / SOR branches need rmom < 1e-3 (and rmom <= 1e-4 for the hybrid)
        sysm = _near_solution(g, sysm, relax=relax)
    s = S.Solver(g, ordering=ordering, relaxsor=1.4, nswp0_vel=4)
    info, out = _compare(g, s, sysm, n, nsolv, 6, relax, relaxsor=1.4, nswp0_vel=4)
    expect = {1: 6, 2: 3, 5: (12 if n == 4 else 24)}[nsolv]
    assert info["iters"] == expect
    if n == 1:
        assert info["rmom"] < 1e-4


@pytest.mark.parametrize("ordering", ["natural", "multicolor"])
def test_hybrid_pressure_bicgstab_branch(ordering):
    g = _grid("tel")
    sysm = G.random_system(g, seed=14)
    s = S.Solver(g, ordering=ordering)
    info, _ = _compare(g, s, sysm, 1, 5, 20, 1.0)
    assert info["rmom"] > 1e-4 and info["inner"] == info["iters"] <= 20


@pytest.mark.parametrize("nsolv,n", [(6, 1), (6, 3), (7, 2), (7, 1), (8, 1), (8, 4)])
def test_five_point_solvers_natural(nsolv, n):
    g = _grid("cart")
    sysm = symmetric_system(g, seed=15, dominance=1.05) if n == 1 else G.random_system(g, seed=15, dominance=1.05)
    s = S.Solver(g, ordering="natural")
    info, out = _compare(g, s, sysm, n, nsolv, 60, 1.0)
    assert info["status"] in (_lib.CMS_OK, _lib.CMS_NOT_CONVERGED)
    # the ratio of the last residual to the first; at 1e-12 it is rounding-level itself
    assert abs(info["relres"] - out["relres"]) <= 1e-8 * out["relres"] + 1e-14


@pytest.mark.parametrize("nsolv,n", [(7, 1), (8, 1), (8, 5)])
def test_incomplete_cholesky_multicolor_converges(nsolv, n):
    """The multicolour form of the diagonal incomplete Cholesky solvers reaches
    the same solution as a direct solve."""
    g = _grid("cart")
    sysm = symmetric_system(g, seed=16, dominance=1.05) if n == 1 else G.random_system(g, seed=16, dominance=1.05)
    s = S.Solver(g, ordering="multicolor", max_iters=400)
    a, b, c, p = _copy(*sysm)
    res = np.zeros_like(b)
    info = s.solve(a, b, c, res, p, n=n, relax=1.0, nsolv=nsolv, raise_on_error=False)
    assert info["status"] == _lib.CMS_OK and info["relres"] < 1e-3
    xs = spl.spsolve(interior_matrix(g, *sysm[:1], sysm[2]).tocsc(), sysm[1][: g.ncells])
    assert np.abs(p[: g.ncells] - xs).max() <= 2e-2 * np.abs(xs).max()


def test_unsupported_combinations_and_adi():
    L = _lib.lib()
    gc, gt = _grid("cart"), _grid("tel")
    sysm = G.random_system(gc, seed=17)
    for g, ordering, nsolv, n in ((gc, "multicolor", 6, 1), (gc, "multicolor", 7, 2), (gt, "natural", 7, 1),
                                  (gt, "natural", 8, 2)):
        sy = G.random_system(g, seed=17)
        s = S.Solver(g, ordering=ordering)
        a, b, c, p = _copy(*sy)
        info = s.solve(a, b, c, np.zeros_like(b), p, n=n, relax=1.0, nswp=5, nsolv=nsolv, raise_on_error=False)
        assert info["status"] == _lib.CMS_UNSUPPORTED, (ordering, nsolv, n)
        assert "5-point" in L.cms_gpu_last_error().decode() or "SIP" in L.cms_gpu_last_error().decode()
    # ADI: the prologue only (ss relaxed, res and rmom), phi unchanged
    s = S.Solver(gc)
    a, b, c, p = _copy(*sysm)
    p0 = p.copy()
    info = s.solve(a, b, c, np.zeros_like(b), p, n=2, relax=0.8, nswp=5, nsolv=0)
    assert info["status"] == _lib.CMS_OK and info["iters"] == 0 and info["rmom"] > 0
    np.testing.assert_array_equal(p, p0)


@pytest.mark.parametrize("nsolv,n", [(1, 2), (2, 2), (6, 2), (8, 1)])
def test_fp32(nsolv, n):
    g = _grid("cart")
    sysm = symmetric_system(g, seed=18) if n == 1 else G.random_system(g, seed=18, dominance=1.1)
    s = S.Solver(g, ordering="natural")
    a, b, c, p = [np.ascontiguousarray(x, np.float32) for x in _copy(*sysm)]
    info = s.solve(a, b, c, np.zeros_like(b), p, n=n, relax=1.0, nswp=12, nsolv=nsolv, raise_on_error=False)
    gp, order = permuted_grid(g, s.perm())
    ao, bo, co, po = permute_system(order, *[np.ascontiguousarray(x, np.float32) for x in sysm])
    out = O.OracleSolver(gp, fix_last_cell=True).solve(ao, bo, co, np.zeros_like(bo), po, relax=1.0, nswp=12,
                                                      nsolv=nsolv, n=n)  # the oracle's single-precision build
    inv = np.empty_like(order); inv[order] = np.arange(order.size)
    nn = g.ncells
    err = np.abs(p[:nn] - po[inv][:nn]).max() / np.abs(po[inv][:nn]).max()
    assert err <= 2e-4, err
    assert abs(info["iters"] - out["iters"]) <= 1


def test_global_api_five_point_solvers():
    """cms_gpu_set_opts(natural) + cms_gpu_init, then solve(..., n) with
    MATRIX_SOLVER = ICCG: ICCG for the pressure correction, SIP for velocity."""
    L = _lib.lib()
    g = _grid("cart")
    c2c = np.ascontiguousarray(g.cell2cell, np.int32)
    ncf = np.ascontiguousarray(g.ncface, np.int32)
    opts = _lib.SolverOpts()
    L.cms_solver_default_opts(C.byref(opts))
    opts.ordering = _lib.ORDER_NATURAL
    assert L.cms_gpu_set_opts(C.byref(opts)) == 0
    assert L.cms_gpu_init(g.ncells, g.ncellsD, g.nmaxfaces, c2c.ctypes.data, ncf.ctypes.data, None) == 0
    try:
        for n, sysm in ((1, symmetric_system(g, seed=19)), (2, G.random_system(g, seed=19))):
            a, b, c, p = _copy(*sysm)
            res = np.zeros_like(b)
            rm = C.c_double()
            rc = L.cms_gpu_solve_d(n, a.ctypes.data, b.ctypes.data, c.ctypes.data, res.ctypes.data, p.ctypes.data,
                                   1.0, 30, 7, C.byref(rm))
            assert rc in (_lib.CMS_OK, _lib.CMS_NOT_CONVERGED)
            s = S.Solver(g, ordering="natural")
            gp, order = permuted_grid(g, s.perm())
            ao, bo, co, po = permute_system(order, *sysm)
            out = O.OracleSolver(gp, fix_last_cell=True).solve(ao, bo, co, np.zeros_like(bo), po, relax=1.0,
                                                              nswp=30, nsolv=7, n=n)
            inv = np.empty_like(order); inv[order] = np.arange(order.size)
            err = np.abs(p[: g.ncells] - po[inv][: g.ncells]).max() / np.abs(po).max()
            assert err <= 1e-10, (n, err)
            assert abs(rm.value - out["rmom"]) <= 1e-12 * out["rmom"]
    finally:
        L.cms_gpu_finalize()
        L.cms_solver_default_opts(C.byref(opts))
        L.cms_gpu_set_opts(C.byref(opts))
