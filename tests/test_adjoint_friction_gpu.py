"""Gradient of a gauge water-level-style misfit of the momentum solve with
respect to per-cell Manning's n: the bottom-friction sink of the momentum
assembly (cms_fric_sink_dev_d, Manning closure of friction.F90:647-662 /
fric_lib.f90:965-966, sink of coeffsourcesink_uv) and its hand-written
adjoint (cms_fric_sink_adjoint_dev_d), chained with the adjoint of solve()
(cms_solver_adjoint_dev_d) through cms2d_b200.adjoint.

Forward model: sp = sp0 - Cd(n) |u| A, x = solve(acoef, ss, sp, phi) (FP64,
to 1e-10), L = sum over 200 seeded gauge cells of (x_g - target_g)^2; depth,
speed and cell areas held fixed.  A few cells are nearly dry (h = 1e-4 m),
where the closure's 0.1 n floor is the active branch, and some are deeper
than 10 m, where min(10, h) caps the depth.

Checks: the friction kernel against the closure in numpy (1e-14); the
solution against a direct FP64 solve (1e-8); dL/dn against an FP64 CPU
tangent-linear of the same model (scipy; 1e-7 relative in random directions)
and against central finite differences of the GPU forward model (5e-5, as
for solve()'s own adjoint).
"""
import numpy as np
import pytest
import scipy.sparse.linalg as spl

from cms2d_b200 import grid as G
from cms2d_b200 import solver as S
from tests.helpers import interior_matrix

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

GRAV = 9.81


def _manning(n, h):
    """Cd and dCd/dn of the closure (depth branch unless 0.1 n is larger)."""
    p = 0.3333
    hd = np.minimum(10.0, h)
    hh = np.maximum(hd, 0.1 * n)
    cd = GRAV * n * n / hh ** p
    dcd = np.where(0.1 * n > hd, (2.0 - p) * cd / n, 2.0 * GRAV * n / hh ** p)
    return cd, dcd


def _case(seed):
    g = G.solver_test_grid(6000)
    acoef, ss, sp0, phi = G.random_system(g, seed=seed)
    rng = np.random.default_rng(seed + 1)
    n = g.ncells
    coefman = rng.uniform(0.015, 0.035, n)
    h = rng.uniform(0.3, 14.0, n)
    h[rng.choice(n, 40, replace=False)] = 1e-4
    uv = rng.uniform(0.05, 1.2, n)
    area = rng.uniform(50.0, 300.0, n)
    gauges = np.sort(rng.choice(n, 200, replace=False))
    target = rng.standard_normal(200)
    return g, acoef, ss, sp0, phi, coefman, h, uv, area, gauges, target


def _system(g, acoef, ss, sp, phi):
    """solve()'s A (active cells) and b in numpy (relax 1)."""
    n = g.ncells
    A = interior_matrix(g, acoef, sp, 1.0)
    b = ss[:n].copy()
    for k in range(g.nmaxfaces):
        c = g.cell2cell[:n, k]
        m = (k < g.ncface[:n]) & (c > n)
        b[m] += acoef[:n, k][m] * phi[c[m] - 1]
    return A.tocsc(), b


def _solver(g):
    return S.Solver(g, tol=1e-10, norm=2, max_iters=4000, verify=False, nsolv=3)


def _tensor(a, rg=False):
    return torch.tensor(a, dtype=torch.float64, device="cuda", requires_grad=rg)


def _loss_and_grad(s, case, coefman, grad=True):
    from cms2d_b200.adjoint import friction_sink_fn, solve_fn
    g, acoef, ss, sp0, phi, _, h, uv, area, gauges, target = case
    cm = _tensor(coefman, grad)
    sp = friction_sink_fn(cm, _tensor(h), _tensor(uv), _tensor(area), _tensor(sp0))
    x = solve_fn(s, _tensor(acoef), _tensor(ss), sp, _tensor(phi), relax=1.0, nswp=4000, tol=1e-9)
    gi = torch.tensor(gauges, device="cuda")
    loss = ((x[gi] - _tensor(target)) ** 2).sum()
    if grad:
        loss.backward()
        torch.cuda.synchronize()
        return float(loss.detach()), cm.grad.cpu().numpy(), x.detach().cpu().numpy(), sp.detach().cpu().numpy()
    return float(loss.detach()), None, x.detach().cpu().numpy(), sp.detach().cpu().numpy()


def test_friction_sink_matches_closure():
    case = _case(31)
    g, acoef, ss, sp0, phi, coefman, h, uv, area, gauges, target = case
    s = _solver(g)
    _, _, _, sp = _loss_and_grad(s, case, coefman, grad=False)
    n = g.ncells
    cd, _ = _manning(coefman, h)
    ref = sp0.copy()
    ref[:n] = sp0[:n] - cd * uv * area
    assert np.abs(sp - ref).max() <= 1e-14 * np.abs(ref).max()
    assert np.any(0.1 * coefman > np.minimum(10.0, h)) and np.any(h > 10.0)  # both branches present


def test_manning_gradient_matches_tangent_linear():
    case = _case(37)
    g, acoef, ss, sp0, phi, coefman, h, uv, area, gauges, target = case
    n = g.ncells
    s = _solver(g)
    loss, gn, x, sp = _loss_and_grad(s, case, coefman)
    A, b = _system(g, acoef, ss, sp, phi)
    xs = spl.spsolve(A, b)
    assert np.abs(x[:n] - xs).max() <= 1e-8 * np.abs(xs).max()
    _, dcd = _manning(coefman, h)
    rng = np.random.default_rng(41)
    for _ in range(4):
        dn = coefman * rng.standard_normal(n)
        dsp = -uv * area * dcd * dn
        dx = spl.spsolve(A, dsp * xs)  # dA = -diag(dsp): dx = -A^-1 dA x
        tl = float(2.0 * np.sum((xs[gauges] - target) * dx[gauges]))
        ad = float(gn @ dn)
        assert abs(ad - tl) <= 1e-7 * max(abs(tl), 1e-30), (ad, tl)


def test_manning_gradient_matches_finite_differences():
    case = _case(43)
    g, acoef, ss, sp0, phi, coefman, h, uv, area, gauges, target = case
    n = g.ncells
    s = _solver(g)
    _, gn, _, _ = _loss_and_grad(s, case, coefman)
    rng = np.random.default_rng(47)
    for _ in range(3):
        dn = 0.2 * coefman * rng.standard_normal(n)
        eps = 1e-3
        lp = _loss_and_grad(s, case, coefman + eps * dn, grad=False)[0]
        lm = _loss_and_grad(s, case, coefman - eps * dn, grad=False)[0]
        fd = (lp - lm) / (2 * eps)
        ad = float(gn @ dn)
        assert abs(ad - fd) <= 5e-5 * abs(fd), (ad, fd)
