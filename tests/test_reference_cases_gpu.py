"""The reference's own flow test cases (L05_Implicit_Test01, L08_Sed_LSTF,
L10_Sed_BedAggradation_SedSorting: their telescoping grids and card
settings, from the committed fixture) stepped by the GPU flow model and by
the oracle on the same case.

The cards select GMRES (nsolv 4), skewness correction on and each case's
drying depth; the strings and Manning fields of the cases live in HDF5
files, so each case takes a north water-level string and a uniform n.
FP64: the oracle solves in the GPU's unknown order, both sides drive every
solve to a 1e-10 relative L2 residual and run 4 outer iterations per step;
water level within 1e-9 m, velocities and fluxes within 1e-6 of their
largest value.  FP32 + FP64 refinement against the oracle in the natural
(reference) order at converged solves: within 1e-5.
"""
import numpy as np
import pytest

from cms2d_b200.flow import FlowModel
from oracle import oracle as O
from tests import reference_cases as RC
from tests.test_flow_gpu import _errors

pytestmark = pytest.mark.gpu

NAMES = RC.names()


def _run(name, precision, ordering, same_order, steps=3, maxit=4):
    case, kw = RC.case(name)
    wd = dict(hdry=kw["hdry"], ponding=kw.get("ponding", False), narrowchannels=kw.get("narrowchannels", False))
    solver = dict(nsolv=kw["nsolv"], tol=1e-10, norm=2, nswp_pp=400, nswp_uv=400)
    m = FlowModel(case, precision=precision, maxit=maxit, ordering=ordering, skewcor=kw["skewcor"], **solver, **wd)
    m.init()
    o = O.FlowOracle(case)
    o.set_solver(nsolv=solver["nsolv"], precond=O.PC_ILU0, tol=solver["tol"], nswp_pp=solver["nswp_pp"],
                 nswp_uv=solver["nswp_uv"], norm=2)
    o.set_wetdry(**wd)
    if same_order:
        o.set_order(m.perm())
    o.init()
    for _ in range(steps):
        r = o.step(maxit=maxit)
        i = m.step()
        assert r["status"] == 0 and i["status"] == 0, (r, i)
        assert r["niter"] == i["niter"]
        np.testing.assert_array_equal(m.get("iwet")[: case.grid.ncells], o.get("iwet")[: case.grid.ncells])
    return _errors(o, m, case.grid)


@pytest.mark.parametrize("ordering", ["natural", "multicolor"])
@pytest.mark.parametrize("name", NAMES)
def test_reference_case_fp64_matches_oracle(name, ordering):
    e = _run(name, "fp64", ordering, same_order=True)
    print(name, ordering, e)
    assert e["eta_m"] <= 1e-9
    for k in ("u", "v", "h", "flux"):
        assert e[k] <= 1e-6, (k, e)


@pytest.mark.parametrize("name", NAMES)
def test_reference_case_fp32_refine_matches_fp64_oracle(name):
    e = _run(name, "fp32_refine", "multicolor", same_order=False)
    print(name, "fp32+refine", e)
    assert e["eta_m"] <= 1e-6
    for k in ("u", "v", "h", "flux"):
        assert e[k] <= 1e-5, (k, e)
