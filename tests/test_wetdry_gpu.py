"""GPU flow step with wetting and drying against the CPU flow oracle.

The intertidal flat (Cartesian, and telescoping so that fronts cross
refinement interfaces) is stepped through a falling and a rising tide: cells
dry and wet every few steps, the narrow-channel rules and flow_pond fire, and
der_update recomputes the gradient weights around each change.  Both sides
run the same fixed numbers of Krylov and outer iterations in the same unknown
order (as in the fixed-wet-set flow tests), so the wet sets must agree cell
for cell at every step and the fields to rounding: water level within 1e-9 m,
velocities, depths, viscosity and fluxes within 1e-6 of their largest value.
"""
import numpy as np
import pytest

from cms2d_b200 import cases
from cms2d_b200.flow import FlowModel
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FIXED = dict(nsolv=3, tol=1e-30, nswp_pp=8, nswp_uv=4)


def _errors(o, m, n):
    vel = max(np.hypot(o.get("u")[:n], o.get("v")[:n]).max(), 1e-12)
    e = {"eta_m": float(np.abs(m.get("eta")[:n] - o.get("eta")[:n]).max())}
    for k in ("u", "v"):
        e[k] = float(np.abs(m.get(k)[:n] - o.get(k)[:n]).max() / vel)
    for k in ("h", "vis", "flux"):
        a, b = m.get(k)[:n], o.get(k)[:n]
        e[k] = float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
    return e


def _run(case, steps, maxit=4, precision="fp64", same_order=True, **solver):
    n = case.grid.ncells
    m = FlowModel(case, precision=precision, maxit=maxit, **solver)
    m.init()
    o = O.FlowOracle(case)
    o.set_solver(nsolv=solver["nsolv"], precond=O.PC_ILU0, tol=solver["tol"], nswp_pp=solver["nswp_pp"],
                 nswp_uv=solver["nswp_uv"], norm=solver.get("norm", 1))
    if same_order:
        o.set_order(m.perm())
    o.init()
    assert np.array_equal(m.get("iwet"), o.get("iwet"))
    changed = 0
    worst = {}
    for step in range(steps):
        r = o.step(maxit=maxit)
        i = m.step()
        assert r["status"] == 0 and i["status"] == 0, (step, r, i)
        assert r["niter"] == i["niter"]
        wm, wo = m.get("iwet"), o.get("iwet")
        assert np.array_equal(wm, wo), (step, np.nonzero(wm != wo)[0][:10])
        assert i["nwet"] == int(wo[:n].sum())
        changed += i["nchanged"]
        e = _errors(o, m, n)
        for k, v in e.items():
            worst[k] = max(worst.get(k, 0.0), v)
    return changed, worst


@pytest.mark.parametrize("refine", [False, True])
@pytest.mark.parametrize("phase", [("falling", 1.0), ("rising", 7.0)])
def test_wetdry_steps_match_oracle(phase, refine):
    c = cases.tidal_flat(refine=refine, t0_hours=phase[1])
    changed, worst = _run(c, steps=10, **FIXED)
    print(phase[0], "refine" if refine else "cartesian", "cells changed", changed, worst)
    assert changed > 0
    assert worst["eta_m"] <= 1e-9
    for k in ("u", "v", "h", "vis", "flux"):
        assert worst[k] <= 1e-6, (k, worst)


def test_wetdry_fp32_refine_matches_fp64_oracle():
    """FP32 + FP64 refinement with converged solves against the FP64 oracle."""
    c = cases.tidal_flat(t0_hours=1.5)
    changed, worst = _run(c, steps=6, precision="fp32_refine", same_order=False, nsolv=3, tol=1e-9, norm=2,
                          nswp_pp=2000, nswp_uv=2000)
    print("fp32+refine", changed, worst)
    assert changed > 0
    assert worst["eta_m"] <= 1e-6
    for k in ("u", "v", "h", "flux"):
        assert worst[k] <= 1e-4, (k, worst)


@pytest.mark.parametrize("settings", ["reference", "production"])
def test_wetdry_long_run_tracks_tide(settings):
    """A whole tidal cycle: every step finishes and the wet area falls and
    rises with the tide.  "reference": the reference's solver defaults
    (GMRES(3), tol 1e-3, 20/5 iterations) on its natural-order ILU(0);
    "production": FP32 + refinement BiCGStab on the multicolour order."""
    c = cases.tidal_flat(t0_hours=0.0, dt=600.0)
    if settings == "reference":
        m = FlowModel(c, ordering="natural")
    else:
        m = FlowModel(c, precision="fp32_refine", nsolv=3, tol=1e-6, norm=2, nswp_pp=200, nswp_uv=200)
    m.init()
    nwet = []
    for _ in range(int(12.42 * 3600 / 600)):
        info = m.step()
        assert info["status"] == 0, info
        nwet.append(info["nwet"])
    k = int(np.argmin(nwet))
    assert nwet[k] < nwet[0] - 200 and nwet[-1] > nwet[k] + 200
