"""GPU hot start (cms_flow_init_hot) against the CPU oracle.

The pressure and velocities of a running oracle model (with velocities also
perturbed in dry cells, so that hot_init's rules act), and in one case its
face fluxes, start both a GPU model
and a second oracle; both then step with the same fixed Krylov and outer
iteration counts in the same unknown order (the wet/dry test's settings).
The wet set must agree cell for cell right after the start and at every step;
the fields after the start (face fluxes included) to 1e-12 of their largest
value, and after each step as in the wet/dry test (water level within 1e-9 m,
other fields within 1e-6).
"""
import numpy as np
import pytest

from cms2d_b200 import cases
from cms2d_b200.flow import FlowModel
from oracle import oracle as O
from tests.test_wetdry_gpu import FIXED, _errors

pytestmark = pytest.mark.gpu


def _hot_inputs(case, steps, seed=5):
    o = O.FlowOracle(case)
    o.init()
    for _ in range(steps):
        assert o.step()["status"] == 0
    rng = np.random.default_rng(seed)
    u = o.get("u") + rng.normal(0, 0.02, case.grid.ncellsD)
    v = o.get("v") + rng.normal(0, 0.02, case.grid.ncellsD)
    return o.get("p"), u, v, o.t, o.get("flux")


@pytest.mark.parametrize("refine,with_flux", [(False, False), (True, False), (True, True)])
def test_hot_start_matches_oracle(refine, with_flux):
    case = cases.tidal_flat(t0_hours=1.0, refine=refine)
    n = case.grid.ncells
    p, u, v, t, flux = _hot_inputs(case, 4)
    flux = flux if with_flux else None
    m = FlowModel(case, maxit=4, **FIXED)
    m.init_hot(p, u, v, t=t, flux=flux)
    o = O.FlowOracle(case)
    o.set_solver(nsolv=FIXED["nsolv"], precond=O.PC_ILU0, tol=FIXED["tol"], nswp_pp=FIXED["nswp_pp"],
                 nswp_uv=FIXED["nswp_uv"], norm=1)
    o.set_order(m.perm())
    o.init_hot(p, u, v, t=t, flux=flux)
    assert np.array_equal(m.get("iwet"), o.get("iwet"))
    for k in ("p", "h", "u", "v", "eta", "vis", "flux"):
        a, b = m.get(k)[:n], o.get(k)[:n]
        assert np.abs(a - b).max() <= 1e-12 * max(np.abs(b).max(), 1.0), k
    worst = {}
    for step in range(6):
        r = o.step(maxit=4)
        i = m.step()
        assert r["status"] == 0 and i["status"] == 0, (step, r, i)
        assert r["niter"] == i["niter"]
        assert np.array_equal(m.get("iwet"), o.get("iwet")), step
        for k, val in _errors(o, m, n).items():
            worst[k] = max(worst.get(k, 0.0), val)
    print("refine" if refine else "cartesian", worst)
    assert worst["eta_m"] <= 1e-9
    for k in ("u", "v", "h", "vis", "flux"):
        assert worst[k] <= 1e-6, (k, worst)
