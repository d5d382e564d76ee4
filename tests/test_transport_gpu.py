"""Transport solves (salinity n=5, suspended sediment n=4) through solve() on
the GPU against the CPU oracle.

The reference's transport modules call the same solve() as the flow step
(sediment/sed_imp.f90:230, salinity/salinity.F90:599, temperature/heat.f90:559)
with their own relax(n) and nswp(n) and non-symmetric upwind-type matrices.
The systems here are assembled from an intertidal-flat flow state with dry
cells (tests/transport_systems.py) and solved through the reference-shaped
global API (cms_gpu_init / cms_gpu_solve_d / cms_gpu_solve_f) and through a
solver handle.  The oracle solves the same systems renumbered into the GPU's
unknown order.  Tolerances: FP64 within 1e-10 of the largest concentration at
every iteration of the sal_imp loop, with the same rmom(5) to 1e-9 relative
and the same number of loop iterations; FP32 within 2e-4 relative.
"""
import ctypes as C

import numpy as np
import pytest

from cms2d_b200 import _lib
from cms2d_b200 import solver as S
from oracle import oracle as O
from tests import transport_systems as T
from tests.helpers import permuted_grid
from tests.test_transport import flat_state

pytestmark = pytest.mark.gpu

ITERMAXSAL, TOLSAL = 30, 1e-5  # salinity/salinity.F90:42-43


def _p(a):
    return a.ctypes.data


def _sal_imp(solve, a, su0, sp, sal, iwet, itermax=ITERMAXSAL, tolsal=TOLSAL):
    """The sal_imp iteration (salinity.F90:575-615): su reset before every solve."""
    tempsal = sal.copy()
    rms = []
    for it in range(1, itermax + 1):
        su = su0.copy()
        rms.append(solve(a, su, sp, sal))
        if rms[-1] < tolsal and it > 5:
            break
    dry = iwet == 0
    sal[dry] = tempsal[dry]
    return rms


def _salinity_case(refine, scheme):
    case, st = flat_state(refine=refine)
    g = case.grid
    rng = np.random.default_rng(7)
    # fresher water landward, seawater offshore, plus noise
    sal1 = 10.0 + 25.0 * np.clip(g.y / g.y[: g.ncells].max(), 0.0, 1.0) + rng.uniform(-1.0, 1.0, g.ncellsD)
    sal = sal1.copy()
    a, su0, sp = T.salinity_system(g, st, sal, sal1, case.dt, scheme=scheme, str_cells=case.th_cells,
                                   str_faces=case.th_faces, salbnd=35.0)
    return case, st, a, su0, sp, sal


def _oracle_sal_imp(g, perm, iwet, a, su0, sp, sal, nsolv, nswp):
    gp, order = permuted_grid(g, perm)
    o = O.OracleSolver(gp, iwet=iwet[order], fix_last_cell=True)
    ap_, su_, sp_, sal_ = (np.ascontiguousarray(x[order]) for x in (a, su0, sp, sal))

    def solve(a_, su, spp, phi):
        return o.solve(a_, su, spp, np.zeros_like(su), phi, relax=0.8, nswp=nswp, nsolv=nsolv,
                       precond=O.PC_ILU0)["rmom"]

    rms = _sal_imp(solve, ap_, su_, sp_, sal_, iwet[order])
    inv = np.empty_like(order); inv[order] = np.arange(order.size)
    return rms, sal_[inv]


@pytest.mark.parametrize("refine", [False, True])
@pytest.mark.parametrize("scheme,nsolv", [("exponential", 4), ("exponential", 3), ("upwind", 3)])
def test_salinity_global_api_matches_oracle(refine, scheme, nsolv):
    case, st, a, su0, sp, sal = _salinity_case(refine, scheme)
    g = case.grid
    n = g.ncells
    nswp = S.NSWP_DEFAULT[nsolv][5]
    iwet = np.ascontiguousarray(st["iwet"], np.int32)
    L = _lib.lib()
    c2c = np.ascontiguousarray(g.cell2cell, np.int32)
    ncf = np.ascontiguousarray(g.ncface, np.int32)
    assert L.cms_gpu_init(g.ncells, g.ncellsD, g.nmaxfaces, _p(c2c), _p(ncf), _p(iwet)) == 0
    try:
        def solve(a_, su, spp, phi):
            res = np.zeros_like(su)
            rm = C.c_double()
            rc = L.cms_gpu_solve_d(5, _p(a_), _p(su), _p(spp), _p(res), _p(phi), 0.8, nswp, nsolv, C.byref(rm))
            assert rc == 0, _lib.lib().cms_gpu_last_error()
            return rm.value

        sal_g = sal.copy()
        rms_g = _sal_imp(solve, np.ascontiguousarray(a), su0, sp, sal_g, iwet)
    finally:
        L.cms_gpu_finalize()
    perm = S.Solver(g, iwet=iwet).perm()
    rms_o, sal_o = _oracle_sal_imp(g, perm, iwet, a, su0, sp, sal.copy(), nsolv, nswp)
    assert len(rms_g) == len(rms_o), (rms_g, rms_o)
    np.testing.assert_allclose(rms_g, rms_o, rtol=1e-9, atol=1e-14)
    assert rms_o[-1] < TOLSAL  # the loop converged
    err = np.abs(sal_g[:n] - sal_o[:n]).max() / np.abs(sal_o[:n]).max()
    assert err <= 1e-10, err
    # dry cells keep their salinity; wet cells stay within the data's range
    dry = iwet[:n] == 0
    assert np.array_equal(sal_g[:n][dry], sal[:n][dry])
    assert sal_g[:n].min() > 8.0 and sal_g[:n].max() < 36.5


def test_salinity_fp32_global_api():
    case, st, a, su0, sp, sal = _salinity_case(False, "exponential")
    g = case.grid
    n = g.ncells
    iwet = np.ascontiguousarray(st["iwet"], np.int32)
    L = _lib.lib()
    c2c = np.ascontiguousarray(g.cell2cell, np.int32)
    ncf = np.ascontiguousarray(g.ncface, np.int32)
    assert L.cms_gpu_init(g.ncells, g.ncellsD, g.nmaxfaces, _p(c2c), _p(ncf), _p(iwet)) == 0
    try:
        def solve(a_, su, spp, phi):
            res = np.zeros_like(su)
            rm = C.c_float()
            rc = L.cms_gpu_solve_f(5, _p(a_), _p(su), _p(spp), _p(res), _p(phi), C.c_float(0.8), 3, 4, C.byref(rm))
            assert rc == 0, _lib.lib().cms_gpu_last_error()
            return float(rm.value)

        f32 = [np.ascontiguousarray(x, np.float32) for x in (a, su0, sp, sal)]
        rms_g = _sal_imp(solve, *f32[:3], f32[3], iwet)
    finally:
        L.cms_gpu_finalize()
    perm = S.Solver(g, iwet=iwet).perm()
    rms_o, sal_o = _oracle_sal_imp(g, perm, iwet, a, su0, sp, sal.copy(), 4, 3)
    assert rms_g[-1] < TOLSAL
    err = np.abs(f32[3][:n].astype(np.float64) - sal_o[:n]).max() / np.abs(sal_o[:n]).max()
    assert err <= 2e-4, err


@pytest.mark.parametrize("nsolv", [3, 4])
def test_sediment_handle_matches_oracle(nsolv):
    """sed_imp's solve(n=4) then the bound to [0, Cteqmax] (sed_imp.f90:230-236),
    three concentration updates in a row, through a solver handle with the
    reference's relax(4) and nswp(4)."""
    case, st = flat_state(refine=True)
    g = case.grid
    n = g.ncells
    rng = np.random.default_rng(11)
    iwet = np.ascontiguousarray(st["iwet"], np.int32)
    alphat = iwet.astype(np.float64) * rng.uniform(0.5, 1.0, g.ncellsD)
    ctkstar = rng.uniform(0.0, 0.8, g.ncellsD)
    ctk1 = rng.uniform(0.0, 0.5, g.ncellsD)
    cteqmax = 0.6
    s = S.Solver(g, iwet=iwet, nsolv=nsolv)
    gp, order = permuted_grid(g, s.perm())
    o = O.OracleSolver(gp, iwet=iwet[order], fix_last_cell=True)
    inv = np.empty_like(order); inv[order] = np.arange(order.size)
    ctk_g = ctk1.copy()
    ctk_o = ctk1.copy()
    nswp = S.NSWP_DEFAULT[nsolv][4]
    for _ in range(3):
        a, su, sp = T.sediment_system(g, st, ctk_g, ctk1, case.dt, ctkstar, alphat, 2e-3)
        a2, su2, sp2 = T.sediment_system(g, st, ctk_o, ctk1, case.dt, ctkstar, alphat, 2e-3)
        res = np.zeros(g.ncellsD)
        info = s.solve(a, su, sp, res, ctk_g, n=4)
        ao, suo, spo, co = (np.ascontiguousarray(x[order]) for x in (a2, su2, sp2, ctk_o))
        out = o.solve(ao, suo, spo, np.zeros(g.ncellsD), co, relax=0.8, nswp=nswp, nsolv=nsolv, precond=O.PC_ILU0)
        ctk_o = co[inv]
        assert info["iters"] == out["iters"] and info["status"] == out["status"] == 0
        assert abs(info["rmom"] - out["rmom"]) <= 1e-9 * out["rmom"]
        ctk_g[:n] = np.clip(ctk_g[:n], 0.0, cteqmax)
        ctk_o[:n] = np.clip(ctk_o[:n], 0.0, cteqmax)
        err = np.abs(ctk_g[:n] - ctk_o[:n]).max() / max(np.abs(ctk_o[:n]).max(), 1e-300)
        assert err <= 1e-10, err
