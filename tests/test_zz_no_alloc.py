"""The allocation-free residual entry point against the solver's own prologue.

cms_solve_residual_noalloc_d serves callers that cannot allocate device memory
at the moment they need the normalised residual (a fixed device-memory budget,
or no implicit device synchronisation allowed mid-step).  Its scratch is a
fixed array inside the library, shared by every call.  This test checks it
against cms_solver_solve_dev_d run with no iterations (the same prologue of
solve(), source/solvers/solvers.f90:230-240), on two calls in a row so that
leftovers of the first call cannot leak into the second.  The file name
places it last in collection order.
"""
import ctypes as C

import numpy as np
import pytest

from cms2d_b200 import _lib
from cms2d_b200 import grid as G
from cms2d_b200 import solver as S

pytestmark = pytest.mark.gpu

RTOL = 1e-12  # FP64, same arithmetic as the handle's prologue


def _noalloc(L, g, d_c2c, d_ncf, d_iwet, ta, tss, tsp, tres, tphi, relax):
    rm = C.c_double()
    rc = L.cms_solve_residual_noalloc_d(g.ncells, g.ncellsD, g.nmaxfaces, d_c2c.data_ptr(), d_ncf.data_ptr(),
                                        d_iwet.data_ptr(), ta.data_ptr(), tss.data_ptr(), tsp.data_ptr(),
                                        tres.data_ptr(), tphi.data_ptr(), relax, C.byref(rm), None)
    return rc, rm.value


def test_noalloc_residual_matches_solver_prologue():
    torch = pytest.importorskip("torch")
    L = _lib.lib()
    L.cms_solve_residual_noalloc_d.argtypes = [C.c_int, C.c_int, C.c_int] + [C.c_void_p] * 8 + \
        [C.c_double, C.POINTER(C.c_double), C.c_void_p]
    dev = torch.device("cuda", 0)
    for seed, g in ((3, G.cartesian_grid(57, 41)), (4, G.solver_test_grid(30000))):
        acoef, ss, sp, phi = G.random_system(g, seed=seed)
        phi[:] = np.random.default_rng(seed).standard_normal(g.ncellsD)
        iwet = np.ones(g.ncellsD, np.int32)
        iwet[::13] = 0
        relax = 0.8
        # reference values: the solver handle's solve() with zero iterations
        s = S.Solver(g, iwet=iwet)
        ta, tsp, tphi = (torch.from_numpy(x.copy()).to(dev) for x in (acoef, sp, phi))
        tss = torch.from_numpy(ss.copy()).to(dev)
        tres = torch.zeros_like(tss)
        info = s.solve(ta, tss, tsp, tres, tphi.clone(), relax=relax, nswp=0, nsolv=3)
        ss_ref = tss.cpu().numpy()[: g.ncells]
        res_ref = tres.cpu().numpy()[: g.ncells]
        d_c2c = torch.from_numpy(np.ascontiguousarray(g.cell2cell, np.int32)).to(dev)
        d_ncf = torch.from_numpy(np.ascontiguousarray(g.ncface, np.int32)).to(dev)
        d_iwet = torch.from_numpy(iwet).to(dev)
        for call in range(2):
            tss2 = torch.from_numpy(ss.copy()).to(dev)
            tres2 = torch.full_like(tss2, float("nan"))
            rc, rmom = _noalloc(L, g, d_c2c, d_ncf, d_iwet, ta, tss2, tsp, tres2, tphi, relax)
            assert rc == _lib.CMS_OK, L.cms_noalloc_last_error()
            np.testing.assert_allclose(tss2.cpu().numpy()[: g.ncells], ss_ref, rtol=RTOL, atol=1e-14)
            np.testing.assert_allclose(tres2.cpu().numpy()[: g.ncells], res_ref, rtol=RTOL, atol=1e-14)
            assert abs(rmom - info["rmom"]) <= RTOL * info["rmom"], (call, rmom, info["rmom"])


def test_noalloc_rejects_sizes_beyond_limit():
    L = _lib.lib()
    L.cms_solve_residual_noalloc_d.argtypes = [C.c_int, C.c_int, C.c_int] + [C.c_void_p] * 8 + \
        [C.c_double, C.POINTER(C.c_double), C.c_void_p]
    L.cms_noalloc_last_error.restype = C.c_char_p
    rm = C.c_double()
    too_many = 16777216 + 1
    dummy = C.c_void_p(16)  # never dereferenced: the size check comes first
    rc = L.cms_solve_residual_noalloc_d(too_many, too_many, 4, *([dummy] * 8), 1.0, C.byref(rm), None)
    assert rc == _lib.CMS_BAD_ARGUMENT
    assert b"limit" in L.cms_noalloc_last_error()
