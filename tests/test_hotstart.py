"""Hot start (hot_init + prestart, hot_start.F90:1125-1215, prestart.f90:298-325)
on the CPU oracle.

* Restarting from the pressure and velocities of a running model (with or
  without its face fluxes) reproduces the uninterrupted run: the fields agree
  to rounding at the restart and the water level within 1e-7 m three steps
  later (the restart rebuilds what the file does not hold: the face fluxes
  from the velocities when they are absent, the eddy viscosity's history).
* hot_init's rules: cells with h < hmin + 1e-5 dry and at rest, each water-
  level string dummy with its cell's values, face fluxes antisymmetric and zero
  across dry faces.
"""
import numpy as np
import pytest

from cms2d_b200 import cases
from oracle import oracle as O


def _running(case, steps):
    o = O.FlowOracle(case)
    o.init()
    for _ in range(steps):
        assert o.step()["status"] == 0
    return o


@pytest.mark.parametrize("with_flux", [False, True])
@pytest.mark.parametrize("refine", [False, True])
def test_hot_start_continues_the_run(refine, with_flux):
    case = cases.tidal_flat(t0_hours=1.0, refine=refine)
    n = case.grid.ncells
    o = _running(case, 4)
    h = O.FlowOracle(case)
    h.init_hot(o.get("p"), o.get("u"), o.get("v"), t=o.t, flux=o.get("flux") if with_flux else None)
    for k in ("p", "u", "v", "h"):
        assert np.abs(o.get(k)[:n] - h.get(k)[:n]).max() <= 1e-12, k
    for _ in range(3):
        assert o.step()["status"] == 0 and h.step()["status"] == 0
    assert np.abs(o.get("eta")[:n] - h.get("eta")[:n]).max() <= 1e-7
    vel = np.hypot(o.get("u")[:n], o.get("v")[:n]).max()
    assert np.abs(o.get("u")[:n] - h.get("u")[:n]).max() <= 1e-5 * vel


def test_hot_init_rules():
    case = cases.tidal_flat(t0_hours=1.0)
    g = case.grid
    n = g.ncells
    o = _running(case, 3)
    p, u, v = o.get("p"), o.get("u").copy(), o.get("v").copy()
    rng = np.random.default_rng(2)
    u += rng.normal(0, 0.05, u.size)  # velocities everywhere, also in dry cells
    v += rng.normal(0, 0.05, v.size)
    h = O.FlowOracle(case)
    h.init_hot(p, u, v)
    zb = case.zb
    depth = p / 9.81 - zb
    dry = depth < 0.05 + 1e-5
    wet = h.get("iwet")
    hu, hv = h.get("u"), h.get("v")
    # dry by hot_init's rule and still dry: at rest
    still = dry[:n] & (wet[:n] == 0)
    assert still.any() and np.all(hu[:n][still] == 0.0) and np.all(hv[:n][still] == 0.0)
    # wet and wet before: the file's velocities
    keep = (~dry[:n]) & (wet[:n] == 1)
    np.testing.assert_array_equal(hu[:n][keep], u[:n][keep])
    # water-level string dummies carry their cell's velocity
    for c, k in zip(case.th_cells, case.th_faces):
        d = int(g.cell2cell[c - 1, k - 1]) - 1
        assert hu[d] == hu[c - 1] and hv[d] == hv[c - 1]
    # fluxes: antisymmetric, zero across faces with a dry side
    fl = h.get("flux")
    for i in range(n):
        for k in range(int(g.ncface[i])):
            j = int(g.cell2cell[i, k]) - 1
            if wet[i] * wet[j] == 0:
                assert fl[i, k] == 0.0
            if j < n:
                kk = [q for q in range(int(g.ncface[j])) if int(g.cell2cell[j, q]) - 1 == i][0]
                assert fl[j, kk] == -fl[i, k]
