"""Transport fixtures (salinity n=5, sediment n=4) on the CPU oracle.

Checks the fixture assembly before the GPU parity tests use it: the
convection-scheme coefficients against hand-computed values
(schemes/comp_lib.f90:54-109), and the assembled systems for consistency --
a uniform concentration with matching boundary, old and equilibrium values is
an exact solution of every row (time term, wet faces, inflow boundary, dry
averaging rows), so the solver must hand it back unchanged.
"""
import math

import numpy as np
import pytest

from cms2d_b200 import cases
from oracle import oracle as O
from tests import transport_systems as T


def test_scheme_coefficients():
    assert T.upwindcoef(2.0, -3.0) == 5.0 and T.upwindcoef(2.0, 3.0) == 2.0
    assert T.hybridcoef(2.0, 1.0) == pytest.approx(2.0 * 0.75)
    assert T.hybridcoef(2.0, 5.0) == 0.0 and T.hybridcoef(2.0, -5.0) == 5.0
    assert T.powerlawcoef(2.0, 1.0) == pytest.approx(2.0 * (1.0 - 0.5 ** 5))
    assert T.exponentialcoef(2.0, 1.0) == pytest.approx(2.0 * 0.5 / (math.exp(0.5) - 1.0))
    assert T.exponentialcoef(2.0, -1.0) == pytest.approx(2.0 * 0.5 / (math.exp(0.5) - 1.0) + 1.0)
    # zero flux: the exponential scheme gives 0 rather than the diffusion dk
    assert T.exponentialcoef(2.0, 0.0) == 0.0


def flat_state(refine=False, steps=3, t0=1.0):
    """Flow state of the intertidal flat during the falling tide (dry cells present)."""
    case = cases.tidal_flat(t0_hours=t0, refine=refine)
    fl = O.FlowOracle(case)
    fl.init()
    h1 = None
    for _ in range(steps):
        h1 = fl.get("h")
        r = fl.step()
        assert r["status"] == 0
    st = T.flow_state(fl, h1)
    assert 0 < int(st["iwet"][: case.grid.ncells].sum()) < case.grid.ncells
    return case, st


@pytest.mark.parametrize("scheme", ["exponential", "upwind", "hybrid", "powerlaw"])
def test_uniform_salinity_is_preserved(scheme):
    case, st = flat_state()
    g = case.grid
    c = 17.5
    sal = np.full(g.ncellsD, c)
    a, su0, sp = T.salinity_system(g, st, sal, sal.copy(), case.dt, scheme=scheme, str_cells=case.th_cells,
                                   str_faces=case.th_faces, salbnd=c)
    n = g.ncells
    assert np.all(a[:n].sum(axis=1) - sp[:n] > 0.0)  # every row has a positive diagonal
    s = O.OracleSolver(g, iwet=st["iwet"])
    su = su0.copy()
    res = np.zeros(g.ncellsD)
    out = s.solve(a, su, sp, res, sal, relax=0.8, nswp=5, nsolv=3, precond=O.PC_ILU0)
    assert out["rmom"] < 1e-12
    assert np.abs(sal[:n] - c).max() < 1e-10


def test_uniform_sediment_is_preserved():
    case, st = flat_state()
    g = case.grid
    n = g.ncells
    c = 0.3
    rng = np.random.default_rng(4)
    ctk = np.full(g.ncellsD, c)
    alphat = st["iwet"].astype(np.float64) * rng.uniform(0.5, 1.0, g.ncellsD)
    a, su, sp = T.sediment_system(g, st, ctk, ctk.copy(), case.dt, np.full(g.ncellsD, c), alphat, 1e-3)
    s = O.OracleSolver(g, iwet=st["iwet"])
    res = np.zeros(g.ncellsD)
    out = s.solve(a, su, sp, res, ctk, relax=0.8, nswp=3, nsolv=4, precond=O.PC_ILU0)
    assert out["rmom"] < 1e-12
    assert np.abs(ctk[:n] - c).max() < 1e-10
