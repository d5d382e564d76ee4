"""GPU flow step (cms_flow_*) against the CPU flow oracle on the same case.

Same algorithm on both sides: every solve runs a fixed number of Krylov
iterations (the tolerance is never met) and the oracle solves in the GPU's
unknown order (natural/level order or multicolour).  The only differences are
FP64 rounding: the GPU sums dot products and face terms in another order.
The iteration counts are chosen so that no solve runs on after its residual
has reached rounding level (there BiCGStab's scalars are formed from noise and
the two sides drift apart): on the small basin the velocity systems reach
1e-15 within a few iterations.  Observed: water level within 1e-10 m,
velocities and fluxes within 1e-8 relative to their largest value; the bounds
below are 1e-9 m and 1e-6.  The outer iteration count is
fixed at 4 (check_conv only tests divergence before the sixth iteration).
FP32 + FP64 refinement is compared with the FP64 oracle on converged solves
(1e-5).
"""
import numpy as np
import pytest

from cms2d_b200 import cases
from cms2d_b200.flow import FlowModel
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FIXED = {"inlet": dict(nsolv=3, tol=1e-30, nswp_pp=12, nswp_uv=8),
         "basin": dict(nsolv=3, tol=1e-30, nswp_pp=8, nswp_uv=4)}


def _pair(case, steps, maxit=4, precision="fp64", ordering="multicolor", same_order=True, ndsch=4, **solver):
    m = FlowModel(case, precision=precision, maxit=maxit, ordering=ordering, ndsch=ndsch, **solver)
    m.init()
    o = O.FlowOracle(case)
    o.set_scheme(ndsch)
    o.set_solver(nsolv=solver["nsolv"], precond=O.PC_ILU0, tol=solver["tol"], nswp_pp=solver["nswp_pp"],
                 nswp_uv=solver["nswp_uv"], norm=solver.get("norm", 1))
    if same_order:
        o.set_order(m.perm())
    o.init()
    for _ in range(steps):
        r = o.step(maxit=maxit)
        i = m.step()
        assert r["status"] == 0 and i["status"] == 0, (r, i, m.last_solves())
        assert r["niter"] == i["niter"]
    return o, m


def _errors(o, m, g):
    n = g.ncells
    vel = np.hypot(o.get("u")[:n], o.get("v")[:n]).max()
    e = {"eta_m": float(np.abs(m.get("eta")[:n] - o.get("eta")[:n]).max())}
    for k in ("u", "v"):
        e[k] = float(np.abs(m.get(k)[:n] - o.get(k)[:n]).max() / vel)
    for k in ("h", "vis", "flux"):
        a, b = m.get(k)[:n], o.get(k)[:n]
        e[k] = float(np.abs(a - b).max() / np.abs(b).max())
    return e


def test_geometry_matches_oracle():
    c = cases.tidal_inlet(12000, seed=2)
    o = O.FlowOracle(c)
    m = FlowModel(c)
    assert m.njoint == o.njoint > 0
    n = c.grid.ncells
    np.testing.assert_allclose(m.get("fintp")[:n], o.get("fintp")[:n], rtol=0, atol=1e-15)
    o.init(); m.init()
    for name in ("zbk", "hk"):
        np.testing.assert_allclose(m.get(name)[:n], o.get(name)[:n], rtol=1e-13, atol=1e-13)
    for name in ("vis", "cfrict", "dpx", "dpy"):
        np.testing.assert_allclose(m.get(name)[:n], o.get(name)[:n], rtol=1e-12, atol=1e-15)


@pytest.mark.parametrize("ordering", ["natural", "multicolor"])
@pytest.mark.parametrize("kind", ["basin", "inlet"])
def test_flow_step_matches_oracle(kind, ordering):
    c = cases.tidal_basin(40, 30, seed=1) if kind == "basin" else cases.tidal_inlet(12000, seed=3)
    o, m = _pair(c, steps=2, ordering=ordering, **FIXED[kind])
    e = _errors(o, m, c.grid)
    print(kind, ordering, e)
    assert e["eta_m"] <= 1e-9
    for k in ("u", "v", "h", "vis", "flux"):
        assert e[k] <= 1e-6, (k, e)


@pytest.mark.parametrize("ndsch", [0, 1, 2, 3])
def test_flow_step_advection_schemes(ndsch):
    """ADVECTION_SCHEME NONE, UPWIND, HYBRID and POWERLAW (EXPONENTIAL is the
    default of the other tests) on the telescoping inlet, joint cells
    included."""
    c = cases.tidal_inlet(12000, seed=3)
    o, m = _pair(c, steps=2, ndsch=ndsch, **FIXED["inlet"])
    e = _errors(o, m, c.grid)
    print("ndsch", ndsch, e)
    assert e["eta_m"] <= 1e-9
    for k in ("u", "v", "h", "vis", "flux"):
        assert e[k] <= 1e-6, (k, e)


def test_unsupported_advection_scheme_rejected():
    from cms2d_b200 import _lib
    with pytest.raises(_lib.CmsError, match="ADVECTION_SCHEME"):
        FlowModel(cases.tidal_basin(20, 10, seed=1), ndsch=5)


@pytest.mark.parametrize("nsolv", [3, 4])
def test_flow_step_gmres_and_bicgstab(nsolv):
    c = cases.tidal_inlet(12000, seed=5)
    o, m = _pair(c, steps=2, nsolv=nsolv, tol=1e-30, nswp_pp=6, nswp_uv=3)
    e = _errors(o, m, c.grid)
    print("nsolv", nsolv, e)
    assert e["eta_m"] <= 1e-9
    for k in ("u", "v", "h", "flux"):
        assert e[k] <= 1e-6, (k, e)


def test_fp32_refine_matches_fp64_oracle():
    """FP32 + FP64 refinement against the FP64 oracle, solves driven to 1e-8 (L2)."""
    c = cases.tidal_inlet(12000, seed=4)
    o, m = _pair(c, steps=2, precision="fp32_refine", same_order=False, nsolv=3, tol=1e-8, norm=2,
                 nswp_pp=2000, nswp_uv=2000)
    e = _errors(o, m, c.grid)
    print("fp32+refine", e)
    assert e["eta_m"] <= 1e-7
    for k in ("u", "v", "h", "flux"):
        assert e[k] <= 1e-5, (k, e)


def test_reference_default_solver_settings_run():
    """GMRES(3), tol 1e-3, nswp 20/5 and the default outer loop: the step converges and tracks the tide."""
    c = cases.tidal_basin(60, 30, seed=5)
    m = FlowModel(c)  # reference defaults
    m.init()
    for _ in range(4):
        info = m.step()
        assert info["status"] == 0 and info["iconv"] in (1, 2)
    eta = m.get("eta")[: c.grid.ncells]
    assert abs(eta.mean() - c.wse(m.t)) < 0.02


@pytest.mark.parametrize("kind", ["inlet", "through_flow"])
def test_device_tide_matches_host_levels(kind):
    """bnd_eval's harmonic string evaluated on the device (cms_flow_set_tide)
    against the same levels computed on the host and passed in: the M2 + K1
    inlet from a tide phase, and a flume driven by per-entry level offsets."""
    if kind == "inlet":
        c = cases.tidal_inlet(12000, seed=3)
        c.t0 = 3600.0
    else:
        from tests import reference_cases as RC
        gf, _, dt = RC.load("L10_Sed_BedAggradation_SedSorting")
        c = cases.through_flow(gf, 0.004, dt=dt)
    out = []
    for device in (False, True):
        m = FlowModel(c, precision="fp64", nsolv=3, tol=1e-10, norm=2, nswp_pp=400, nswp_uv=400)
        m.init()
        if device:
            m.set_tide()
        for _ in range(3):
            assert m.step()["status"] == 0
        out.append(m.get("eta")[: c.grid.ncells].copy())
        m.close()
    assert np.abs(out[0] - out[1]).max() <= 1e-10


@pytest.mark.parametrize("precision", ["fp32_refine", "fp64"])
def test_flow_step_is_deterministic(precision):
    """Two models of one case step to the same bits: the persistent kernels'
    dot products are summed in a fixed order and nothing depends on timing."""
    c = cases.tidal_inlet(12000, seed=6)
    out = []
    for _ in range(2):
        m = FlowModel(c, precision=precision, nsolv=3, tol=1e-6, norm=2, nswp_pp=200, nswp_uv=200)
        m.init()
        hist = [m.step()["krylov_iters"] for _ in range(4)]
        out.append((hist, m.get("eta").copy(), m.get("u").copy()))
        m.close()
    assert out[0][0] == out[1][0]
    np.testing.assert_array_equal(out[0][1], out[1][1])
    np.testing.assert_array_equal(out[0][2], out[1][2])
