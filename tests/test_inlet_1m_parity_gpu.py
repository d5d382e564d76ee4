"""The benchmarked workload against the FP64 oracle: the three-level tidal
inlet of about 1.0M cells (tidal_inlet(1_000_000, seed=11), dt = 300 s),
first 6 steps from the cold start.

The oracle's side is the committed fixture tests/golden/inlet_1m_oracle.npz
(made by tests/golden/make_inlet_1m_oracle.py): natural cell order, every
solve to a 1e-9 relative L2 residual (or 600 iterations, where the
reference's small guards stall it), the outer loop ended by check_conv;
water level and velocities at 8192 seeded cells after every step, and
statistics over all cells.

The GPU runs the bench's settings: BiCGStab + ILU(0) solves to a 1e-6
relative L2 residual (cap 200), multicolour order, the outer loop ended by
check_conv; once as the FP32 + FP64 refinement headline (adaptive inner
tolerance, reduced inner form) and once as the plain FP64 drop-in.  Errors are
the largest difference over the sample cells and steps relative to the
largest oracle value, |eta| for the water level and |(u, v)| for the
velocity.  Bounds: 1e-6 for the FP64 drop-in, 1e-5 after refinement.
"""
import os

import numpy as np
import pytest

from cms2d_b200 import cases
from cms2d_b200.flow import FlowModel

FIXTURE = os.path.join(os.path.dirname(__file__), "golden", "inlet_1m_oracle.npz")
pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not os.path.exists(FIXTURE), reason="oracle fixture not generated")]
SETTINGS = dict(nsolv=3, tol=1e-6, norm=2, nswp_pp=200, nswp_uv=200)
BOUND = {"fp64": 1e-6, "fp32_refine": 1e-5}


@pytest.fixture(scope="module")
def inlet():
    z = np.load(FIXTURE)
    case = cases.tidal_inlet(int(z["cells"]), seed=int(z["seed"]))
    assert case.grid.ncells == int(z["cells"])
    return case, z


@pytest.mark.parametrize("precision", ["fp32_refine", "fp64"])
def test_inlet_1m_matches_fp64_oracle(inlet, precision):
    case, z = inlet
    n = case.grid.ncells
    idx = z["sample"]
    m = FlowModel(case, precision=precision, **SETTINGS)
    m.init()
    e_eta = e_vel = 0.0
    for s in range(z["eta"].shape[0]):
        info = m.step()
        assert info["status"] == 0 and info["iconv"] == 2, info
        eta, u, v = (m.get(k)[:n] for k in ("eta", "u", "v"))
        eo, uo, vo = z["eta"][s], z["u"][s], z["v"][s]
        e_eta = max(e_eta, float(np.abs(eta[idx] - eo).max() / np.abs(eo).max()))
        e_vel = max(e_vel, float(np.hypot(u[idx] - uo, v[idx] - vo).max() / np.hypot(uo, vo).max()))
        # whole-grid statistics (a wrong cell outside the sample shows here)
        h = m.get("h")[:n]
        st = np.array([eta.mean(), eta.min(), eta.max(), np.sqrt(np.mean(eta * eta)), np.abs(u).max(),
                       np.abs(v).max(), h.sum()])
        np.testing.assert_allclose(st, z["stats"][s], rtol=10 * BOUND[precision], atol=1e-12)
    m.close()
    print(precision, {"eta_max_rel": e_eta, "vel_max_rel": e_vel})
    assert e_eta <= BOUND[precision]
    assert e_vel <= BOUND[precision]
