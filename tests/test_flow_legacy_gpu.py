"""GPU flow step with the MATRIX_SOLVER options other than BiCGStab and GMRES
against the CPU flow oracle.

The flow step hands its three systems to the same dispatch as solve(..., n)
(u: n = 2, v: n = 3, pressure correction: n = 1), at the reference's default
nswp(n) for each option; the oracle solves the same systems in the GPU's
unknown order with its restatement of gauss-seidel.f90, sip.f90, iccg.f90 and
iccgstab.f90.  On a Cartesian basin (the 5-point options need four faces per
cell; SIP the natural ordering) four outer iterations of two steps: water
level within 1e-9 m, velocities, depths and fluxes within 1e-6 of their
largest value, as for the Krylov options.  ICCG / ICCGSTAB in the multicolour
ordering are a method of their own and are checked against a converged step.
"""
import numpy as np
import pytest

from cms2d_b200 import cases
from cms2d_b200 import solver as S
from cms2d_b200.flow import FlowModel
from oracle import oracle as O
from tests.test_flow_gpu import _errors, _pair

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nsolv,ordering", [(1, "natural"), (1, "multicolor"), (2, "natural"), (2, "multicolor"),
                                            (5, "natural"), (5, "multicolor"), (6, "natural"), (7, "natural"),
                                            (8, "natural")])
def test_flow_step_legacy_solvers(nsolv, ordering):
    c = cases.tidal_basin(40, 30, seed=1)
    d = S.NSWP_DEFAULT[nsolv]
    o, m = _pair(c, steps=2, ordering=ordering, nsolv=nsolv, tol=1e-3, nswp_pp=d[1], nswp_uv=d[2])
    e = _errors(o, m, c.grid)
    print(nsolv, ordering, e, m.last_solves())
    assert e["eta_m"] <= 1e-9
    for k in ("u", "v", "h", "flux"):
        assert e[k] <= 1e-6, (k, e)


def test_flow_step_incomplete_cholesky_multicolor():
    """ICCG / ICCGSTAB in the multicolour ordering: the GPU's multicolour
    diagonal incomplete factor is its own method there (the oracle restates
    the compass-slot loops of iccg5, which only make sense in the natural
    order), so the step is compared with the oracle's converged GMRES step:
    the water level agrees to the solvers' truncation."""
    c = cases.tidal_basin(40, 30, seed=1)
    d = S.NSWP_DEFAULT[8]
    m = FlowModel(c, ordering="multicolor", nsolv=8, tol=1e-3, nswp_pp=d[1], nswp_uv=d[2])
    m.init()
    o = O.FlowOracle(c)
    o.set_solver(nsolv=4, precond=O.PC_ILU0, tol=1e-3, nswp_pp=20, nswp_uv=5)
    o.init()
    n = c.grid.ncells
    for _ in range(2):
        assert m.step()["status"] == 0 and o.step()["status"] == 0
    assert np.abs(m.get("eta")[:n] - o.get("eta")[:n]).max() <= 1e-5

