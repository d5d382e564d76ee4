"""Failure detection on the GPU without a fault: a device wait that cannot be
satisfied (a progress flag that nothing sets: the wait of the pipelined
sweeps, the persistent BiCGStab kernel's wait on a neighbour tile and its
grid barrier) gives up after its poll limit, the host reads CMS_DEVICE_ERROR
with where it happened, and the same handle and device go on working."""
import numpy as np
import pytest

from cms2d_b200 import _lib
from cms2d_b200 import grid as G
from cms2d_b200 import solver as S

pytestmark = pytest.mark.gpu


def test_bounded_wait_gives_up_and_device_stays_usable():
    g = G.cartesian_grid(20, 15)
    s = S.Solver(g, ordering="natural")
    L = _lib.lib()
    rc = L.cms_solver_wait_selftest(s._h, 20000)
    assert rc == _lib.CMS_DEVICE_ERROR
    msg = L.cms_gpu_last_error().decode()
    assert "timed out waiting for row 0 to complete 1 passes (saw 0" in msg, msg
    # the handle and the device still work: natural-order Gauss-Seidel uses the same waits
    a, b, c, p = G.random_system(g, seed=2, dominance=1.2)
    info = s.solve(a, b, c, np.zeros_like(b), p, n=2, relax=0.8, nswp=5, nsolv=1)
    assert info["status"] == _lib.CMS_OK and info["iters"] == 5
    assert np.all(np.isfinite(p))


@pytest.mark.parametrize("which", [0, 1], ids=["neighbour_wait", "grid_barrier"])
def test_persistent_kernel_waits_give_up(which):
    g = G.cartesian_grid(40, 30)
    s = S.Solver(g, tol=1e-8)
    L = _lib.lib()
    rc = L.cms_solver_persist_wait_selftest(s._h, 20000, which)
    assert rc == _lib.CMS_DEVICE_ERROR
    msg = L.cms_gpu_last_error().decode()
    want = ("the neighbour wait gave up after 20000 polls (tile 1 never completed phase 1)" if which == 0 else
            "the grid barrier gave up after 20000 polls (1 of 2 blocks arrived)")
    assert want in msg, msg
    # the same handle then solves normally through the persistent kernel
    a, b, c, p = G.random_system(g, seed=3)
    info = s.solve(a, b, c, np.zeros_like(b), p, relax=1.0, nswp=200, nsolv=3)
    assert info["status"] == _lib.CMS_OK and info["iters"] > 0
    assert np.all(np.isfinite(p))
