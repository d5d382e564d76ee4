"""GPU parity of libcmsgpu's solve() against the CPU oracle (same inputs, same ordering).

Tolerances: FP64 solution within 1e-10 relative of the oracle and the same
iteration count; FP32 within 1e-4; FP32+FP64-refinement within 1e-5 of the
FP64 oracle solution (the accuracy required of the refined solver).
"""
import numpy as np
import pytest
import scipy.sparse.linalg as spla

from cms2d_b200 import grid as G
from cms2d_b200 import solver as S
from oracle import oracle as O
from tests.helpers import interior_matrix, permute_system, permuted_grid

pytestmark = pytest.mark.gpu

FP64_RTOL = 1e-10


def _copy(*a):
    return [np.array(x, copy=True) for x in a]


def _grids():
    return {
        "cart": G.cartesian_grid(48, 31),
        "tel": G.solver_test_grid(6000),
    }


def _oracle_on_device_order(g, perm, acoef, ss, sp, phi, **kw):
    """Runs the oracle on the system renumbered into the GPU's device order."""
    gp, order = permuted_grid(g, perm)
    a, b, c, p = permute_system(order, acoef, ss, sp, phi)
    r = np.zeros_like(b)
    out = O.OracleSolver(gp, fix_last_cell=True).solve(a, b, c, r, p, **kw)
    # back to natural order
    inv = np.empty_like(order); inv[order] = np.arange(order.size)
    return out, b[inv], r[inv], p[inv]


@pytest.mark.parametrize("kind", ["cart", "tel"])
@pytest.mark.parametrize("ordering", ["natural", "multicolor"])
@pytest.mark.parametrize("nsolv,multi", [(3, False), (3, True), (4, False)])
def test_fp64_parity(kind, ordering, nsolv, multi):
    """BiCGStab runs both as one persistent launch and as per-phase kernels."""
    g = _grids()[kind]
    acoef, ss, sp, phi = G.random_system(g, seed=21)
    phi[: g.ncells] = np.random.default_rng(1).standard_normal(g.ncells) * 0.1
    relax = 0.8
    nswp = 40 if nsolv == 3 else 15
    tol = 1e-8
    s = S.Solver(g, ordering=ordering, tol=tol, multi_kernel=multi)
    a, b, c, p = _copy(acoef, ss, sp, phi)
    res = np.zeros_like(b)
    info = s.solve(a, b, c, res, p, relax=relax, nswp=nswp, nsolv=nsolv)
    out, b_o, r_o, p_o = _oracle_on_device_order(g, s.perm(), acoef, ss, sp, phi, relax=relax, nswp=nswp,
                                                 nsolv=nsolv, precond=O.PC_ILU0, tol=tol)
    n = g.ncells
    assert info["iters"] == out["iters"], (info, out)
    if nsolv == 4:
        assert info["inner"] == out["inner"]
    np.testing.assert_allclose(b[:n], b_o[:n], rtol=1e-13, atol=1e-13)
    np.testing.assert_allclose(res[:n], r_o[:n], rtol=1e-11, atol=1e-12)
    assert abs(info["rmom"] - out["rmom"]) <= 1e-12 * out["rmom"]
    err = np.abs(p[:n] - p_o[:n]).max() / np.abs(p_o[:n]).max()
    assert err <= FP64_RTOL, err
    assert info["status"] == out["status"] == 0


@pytest.mark.parametrize("nsolv", [3, 4])
def test_reference_default_mode(nsolv):
    """tol 1e-3 and nswp caps of the reference (pp: 15 BiCGStab / 20 GMRES restarts)."""
    g = G.cartesian_grid(40, 40)
    acoef, ss, sp, phi = G.random_system(g, seed=8)
    nswp = 15 if nsolv == 3 else 20
    s = S.Solver(g, ordering="natural", tol=1e-3)
    a, b, c, p = _copy(acoef, ss, sp, phi)
    res = np.zeros_like(b)
    info = s.solve(a, b, c, res, p, n=1, nsolv=nsolv)
    out, _, _, p_o = _oracle_on_device_order(g, s.perm(), acoef, ss, sp, phi, relax=1.0, nswp=nswp, nsolv=nsolv,
                                             precond=O.PC_ILU0, tol=1e-3)
    assert info["iters"] == out["iters"]
    n = g.ncells
    assert np.abs(p[:n] - p_o[:n]).max() <= FP64_RTOL * np.abs(p_o[:n]).max()


def test_iteration_cap_not_converged():
    g = G.cartesian_grid(30, 30)
    acoef, ss, sp, phi = G.random_system(g, seed=2)
    s = S.Solver(g, tol=1e-12)
    a, b, c, p = _copy(acoef, ss, sp, phi)
    res = np.zeros_like(b)
    info = s.solve(a, b, c, res, p, nswp=1, nsolv=3)
    assert info["iters"] == 1 and info["status"] == 1 and info["iconv"] == 1


@pytest.mark.parametrize("nsolv", [3, 4])
def test_fp32_dropin(nsolv):
    g = G.solver_test_grid(5000)
    acoef, ss, sp, phi = G.random_system(g, seed=5)
    s = S.Solver(g, tol=1e-5)
    a, b, c, p = [x.astype(np.float32) for x in (acoef, ss, sp, phi)]
    res = np.zeros_like(b)
    info = s.solve(a, b, c, res, p, relax=1.0, nswp=60, nsolv=nsolv)
    out, _, _, p_o = _oracle_on_device_order(g, s.perm(), acoef, ss, sp, phi, relax=1.0, nswp=200, nsolv=nsolv,
                                             precond=O.PC_ILU0, tol=1e-9)
    n = g.ncells
    assert info["status"] == 0
    assert np.abs(p[:n] - p_o[:n]).max() <= 1e-4 * np.abs(p_o[:n]).max()


@pytest.mark.parametrize("nsolv", [3, 4])
def test_fp32_refinement_matches_fp64(nsolv):
    g = G.solver_test_grid(20000)
    acoef, ss, sp, phi = G.random_system(g, seed=6)
    s = S.Solver(g, precision="fp32_refine", tol=1e-8, inner_tol=1e-2, norm=2)
    a, b, c, p = _copy(acoef, ss, sp, phi)
    res = np.zeros_like(b)
    info = s.solve(a, b, c, res, p, relax=1.0, nswp=500, nsolv=nsolv)
    assert info["status"] == 0 and info["refine_steps"] >= 1
    assert info["true_relres"] <= 1e-8
    A = interior_matrix(g, acoef, sp)
    import scipy.sparse.linalg as spl
    xs = spl.spsolve(A.tocsc(), ss[: g.ncells])
    assert np.abs(p[: g.ncells] - xs).max() <= 1e-5 * np.abs(xs).max()


def test_device_pointer_path_matches_host_path():
    torch = pytest.importorskip("torch")
    g = G.solver_test_grid(8000)
    acoef, ss, sp, phi = G.random_system(g, seed=12)
    s = S.Solver(g, tol=1e-8)
    a, b, c, p = _copy(acoef, ss, sp, phi)
    res = np.zeros_like(b)
    i1 = s.solve(a, b, c, res, p, nswp=100, nsolv=3)
    ta, tb, tc, tp = [torch.from_numpy(x.copy()).cuda() for x in (acoef, ss, sp, phi)]
    tr = torch.zeros_like(tb)
    i2 = s.solve(ta, tb, tc, tr, tp, nswp=100, nsolv=3)
    assert i1["iters"] == i2["iters"]
    np.testing.assert_array_equal(tp.cpu().numpy()[: g.ncells], p[: g.ncells])
    np.testing.assert_array_equal(tb.cpu().numpy()[: g.ncells], b[: g.ncells])


def test_global_api_matches_handle():
    import ctypes as C
    from cms2d_b200 import _lib
    L = _lib.lib()
    g = G.cartesian_grid(20, 15)
    acoef, ss, sp, phi = G.random_system(g, seed=1)
    c2c = np.ascontiguousarray(g.cell2cell, np.int32)
    ncf = np.ascontiguousarray(g.ncface, np.int32)
    assert L.cms_gpu_init(g.ncells, g.ncellsD, g.nmaxfaces, c2c.ctypes.data, ncf.ctypes.data, None) == 0
    a, b, c, p = _copy(acoef, ss, sp, phi)
    res = np.zeros_like(b)
    rm = C.c_double()
    rc = L.cms_gpu_solve_d(1, a.ctypes.data, b.ctypes.data, c.ctypes.data, res.ctypes.data, p.ctypes.data, 1.0, 15,
                           3, C.byref(rm))
    info = _lib.SolveInfo()
    L.cms_gpu_last_info(C.byref(info))
    L.cms_gpu_finalize()
    s = S.Solver(g)
    a2, b2, c2, p2 = _copy(acoef, ss, sp, phi)
    r2 = np.zeros_like(b2)
    i2 = s.solve(a2, b2, c2, r2, p2, relax=1.0, nswp=15, nsolv=3)
    assert rc == i2["status"] and info.iters == i2["iters"]
    np.testing.assert_array_equal(p, p2)
    assert rm.value == i2["rmom"]


def test_dry_cells_and_zero_rhs():
    """Dry rows (sp=-1, su=0, acoef=0 as bound_uv sets them) and an all-zero RHS."""
    g = G.cartesian_grid(25, 20)
    acoef, ss, sp, phi = G.random_system(g, seed=3)
    iwet = np.ones(g.ncellsD, np.int32)
    dry = np.arange(0, g.ncells, 7)
    iwet[dry] = 0
    acoef[dry] = 0.0
    sp[dry] = -1.0
    ss[dry] = 0.0
    s = S.Solver(g, iwet=iwet, ordering="natural", tol=1e-8)
    a, b, c, p = _copy(acoef, ss, sp, phi)
    res = np.zeros_like(b)
    info = s.solve(a, b, c, res, p, relax=1.0, nswp=60, nsolv=3)
    o = O.OracleSolver(g, iwet=iwet)
    a2, b2, c2, p2 = _copy(acoef, ss, sp, phi)
    r2 = np.zeros_like(b2)
    out = o.solve(a2, b2, c2, r2, p2, relax=1.0, nswp=60, nsolv=3, precond=O.PC_ILU0, tol=1e-8)
    assert info["iters"] == out["iters"]
    n = g.ncells
    assert np.all(res[dry] == 0.0)
    assert np.abs(p[:n] - p2[:n]).max() <= FP64_RTOL * np.abs(p2[:n]).max()
    # zero RHS: stays at zero
    z = np.zeros_like(ss)
    a, c, p = _copy(acoef, sp, z)
    b = z.copy(); res = np.zeros_like(b)
    info = s.solve(a, b, c, res, p, relax=1.0, nswp=10, nsolv=3)
    assert np.abs(p).max() < 1e-12


def test_unsupported_solver_code():
    g = G.cartesian_grid(6, 5)
    acoef, ss, sp, phi = G.random_system(g, seed=1)
    s = S.Solver(g)
    info = s.solve(acoef, ss, sp, np.zeros_like(ss), phi, nsolv=6, raise_on_error=False)
    assert info["status"] == 5


@pytest.mark.parametrize("n_target", [250_000, 1_000_000])
def test_large_system_residual_property(n_target):
    """At the sweep sizes: the FP64 true residual meets the tolerance for FP64 and for refinement."""
    g = G.solver_test_grid(n_target)
    acoef, ss, sp, phi = G.random_system(g, seed=31)
    for prec in ("fp64", "fp32_refine"):
        s = S.Solver(g, precision=prec, tol=1e-6, norm=2)
        a, b, c, p = _copy(acoef, ss, sp, phi)
        res = np.zeros_like(b)
        info = s.solve(a, b, c, res, p, relax=1.0, nswp=1000, nsolv=3)
        assert info["status"] == 0, info
        assert 0 <= info["true_relres"] <= 2e-6, info


@pytest.mark.parametrize("precision", ["fp64", "fp32_refine", "fp32"])
@pytest.mark.parametrize("kind", ["tel", "big"])
def test_persistent_matches_multi_kernel(precision, kind):
    """The persistent BiCGStab launch and the per-phase kernels run the same
    arithmetic; only the block partition of the dot products differs, so the
    iteration counts agree and the solutions agree to rounding."""
    g = G.solver_test_grid(250_000) if kind == "big" else _grids()["tel"]
    acoef, ss, sp, phi = G.random_system(g, seed=5)
    if precision == "fp32":
        acoef, ss, sp, phi = (x.astype(np.float32) for x in (acoef, ss, sp, phi))
    out = []
    for multi in (False, True):
        # exact multicolour factor on both sides (the two-phase inner factor is
        # tested on its own below)
        s = S.Solver(g, precision="fp64" if precision == "fp32" else precision, tol=1e-6, norm=2,
                     multi_kernel=multi, inner_relax=False)
        a, b, c, p = _copy(acoef, ss, sp, phi)
        res = np.zeros_like(b)
        info = s.solve(a, b, c, res, p, nswp=500, nsolv=3)
        assert info["status"] == 0, info
        out.append((info, p[: g.ncells].astype(np.float64)))
    (i0, p0), (i1, p1) = out
    assert i0["iters"] == i1["iters"] and i0["refine_steps"] == i1["refine_steps"], (i0, i1)
    # FP64: rounding only; FP32 solves and refined solves: both within their
    # stopping tolerance of the same solution
    tol = {"fp64": 1e-9, "fp32_refine": 1e-5, "fp32": 1e-4}[precision]
    assert np.abs(p0 - p1).max() <= tol * np.abs(p1).max()


@pytest.mark.parametrize("kind", ["cart", "tel", "big"])
def test_inner_solve_forms(kind):
    """FP32 + refinement with each inner BiCGStab form -- the reduced
    (Schur complement) system, the two-phase factor (couplings among the rows
    of colours >= 2 dropped; the exact factor on a two-colour grid) and the
    exact multicolour factor -- converges to the FP64 tolerance and to the same
    solution, which is the direct solution of the system."""
    g = {"big": lambda: G.solver_test_grid(250_000), "tel": lambda: _grids()["tel"],
         "cart": lambda: G.cartesian_grid(300, 200)}[kind]()
    acoef, ss, sp, phi = G.random_system(g, seed=9)
    res = {}
    for relax in (2, 1, 0):
        s = S.Solver(g, precision="fp32_refine", tol=1e-8, norm=2, inner_relax=relax)
        assert s.last_info is None
        a, b, c, p = _copy(acoef, ss, sp, phi)
        r = np.zeros_like(b)
        info = s.solve(a, b, c, r, p, nswp=2000, nsolv=3)
        assert info["status"] == 0 and info["ncolors"] == (2 if kind == "cart" else info["ncolors"]), info
        assert info["true_relres"] <= 1e-8, info
        res[relax] = (info, p[: g.ncells].copy())
    print(kind, {k: (v[0]["iters"], v[0]["refine_steps"]) for k, v in res.items()})
    p0 = res[0][1]
    for relax in (2, 1):
        assert np.abs(res[relax][1] - p0).max() <= 1e-6 * np.abs(p0).max(), relax
    if kind != "big":
        A = interior_matrix(g, acoef, sp)
        n = g.ncells
        rhs = ss[:n] + np.array([sum(acoef[i, k] * phi[g.cell2cell[i, k] - 1] for k in range(g.ncface[i])
                                     if g.cell2cell[i, k] > n) for i in range(n)])
        x = spla.spsolve(A.tocsc(), rhs)
        assert np.abs(res[2][1] - x).max() <= 1e-6 * np.abs(x).max()


@pytest.mark.parametrize("kind", ["cart", "tel", "big"])
def test_reduced_layouts(kind):
    """Every block/row layout of the reduced inner solve, in the three-phase
    and the single-reduction form, converges to the same solution; the
    single-reduction form's iteration counts stay close to the three-phase
    form's (the same iterates up to rounding)."""
    g = {"big": lambda: G.solver_test_grid(250_000), "tel": lambda: _grids()["tel"],
         "cart": lambda: G.cartesian_grid(300, 200)}[kind]()
    acoef, ss, sp, phi = G.random_system(g, seed=11)
    res = {}
    for layout in range(1, 8):
        s = S.Solver(g, precision="fp32_refine", tol=1e-8, norm=2, inner_relax=2, reduced_layout=layout)
        a, b, c, p = _copy(acoef, ss, sp, phi)
        r = np.zeros_like(b)
        info = s.solve(a, b, c, r, p, nswp=2000, nsolv=3)
        assert info["status"] == 0 and info["true_relres"] <= 1e-8, (layout, info)
        res[layout] = (info, p[: g.ncells].copy())
    print(kind, {k: (v[0]["iters"], v[0]["refine_steps"]) for k, v in res.items()})
    p0 = res[4][1]
    for layout, (info, p) in res.items():
        assert np.abs(p - p0).max() <= 1e-6 * np.abs(p0).max(), layout
    assert res[5][0]["iters"] <= 1.5 * res[4][0]["iters"] + 10, (res[5][0], res[4][0])
