"""Gradient of a gauge misfit of the momentum solve with respect to the face
viscosity, face depth and face flux: the momentum face coefficients
acoef = scheme(visk hk ds, flux) of coeffsourcesink_uv (cms_momentum_coef_dev_d,
every ADVECTION_SCHEME function of comp_lib.f90:40-109) and their
hand-written adjoint (cms_momentum_coef_adjoint_dev_d), chained with the
adjoint of solve() through cms2d_b200.adjoint.

Forward model: acoef from (visk, hk, ds, flux) on the faces of the active
cells, sp fixed and negative (the system stays diagonally dominant),
x = solve(acoef, ss, sp, phi) (FP64, to 1e-10), L = sum over 200 seeded gauge
cells of (x_g - target_g)^2.  The face Peclet ratios |F|/D are kept away from
the schemes' branch points (|F| = D, |F| = 2 D, F = 0) so that the model is
smooth where it is differentiated.

Checks per scheme: the coefficients against the scheme functions in numpy
(1e-14); dL/d(visk, hk, flux) against an FP64 CPU tangent-linear (the
coefficients' derivatives by central differences of the numpy functions,
scipy solves; 1e-6 relative in random directions) and against central finite
differences of the GPU forward model (5e-5).
"""
import numpy as np
import pytest
import scipy.sparse.linalg as spl

from cms2d_b200 import grid as G
from cms2d_b200 import solver as S
from tests.helpers import interior_matrix

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _scheme(ndsch, dk, fk):
    """comp_lib.f90:40-109 in numpy (the functions the flow step uses)."""
    absf = np.abs(fk)
    up = np.maximum(0.0, -fk)
    if ndsch == 1:
        return dk + up
    if ndsch == 2:
        pk = absf / np.maximum(dk, 1e-6)
        return dk * np.maximum(0.0, 1.0 - 0.5 * pk) + up
    if ndsch == 3:
        pk = absf / np.maximum(np.maximum(dk, absf), 1e-6)
        return dk * (1.0 - pk ** 5) + up
    pk = absf / np.maximum(np.maximum(dk, 1e-6), absf)
    return dk * pk / np.maximum(np.exp(pk) - 1.0, 1e-6) + up


def _case(seed):
    g = G.solver_test_grid(6000)
    acoef0, ss, _, phi = G.random_system(g, seed=seed)
    rng = np.random.default_rng(seed + 1)
    n, nD, nmf = g.ncells, g.ncellsD, g.nmaxfaces
    shape = (nD, nmf)
    visk = rng.uniform(0.5, 2.0, shape)
    hk = rng.uniform(0.5, 3.0, shape)
    ds = rng.uniform(0.5, 2.0, shape)
    dk = visk * hk * ds
    # |F| / D away from the branch points 1 and 2 (and from F = 0)
    bands = np.array([[0.1, 0.9], [1.1, 1.9], [2.1, 3.0]])
    b = bands[rng.integers(0, 3, shape)]
    ratio = b[..., 0] + (b[..., 1] - b[..., 0]) * rng.random(shape)
    flux = np.where(rng.random(shape) < 0.5, -1.0, 1.0) * ratio * dk
    sp = np.zeros(nD)
    sp[:n] = -rng.uniform(1.0, 2.0, n)
    gauges = np.sort(rng.choice(n, 200, replace=False))
    target = rng.standard_normal(200)
    mask = np.arange(nmf)[None, :] < g.ncface[:, None]
    mask[n:] = False
    return g, ss, sp, phi, visk, hk, ds, flux, mask, gauges, target


def _acoef(ndsch, visk, hk, ds, flux, mask):
    return np.where(mask, _scheme(ndsch, visk * hk * ds, flux), 0.0)


def _system(g, acoef, ss, sp, phi):
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


def _t(a, rg=False):
    return torch.tensor(a, dtype=torch.float64, device="cuda", requires_grad=rg)


def _run(s, case, ndsch, visk, hk, flux, grad=True):
    from cms2d_b200.adjoint import momentum_coef_fn, solve_fn
    g, ss, sp, phi, _, _, ds, _, _, gauges, target = case
    V, H, F = _t(visk, grad), _t(hk, grad), _t(flux, grad)
    ncf = torch.tensor(np.asarray(g.ncface, np.int32), device="cuda")
    acoef = momentum_coef_fn(ncf, g.ncells, V, H, _t(ds), F, ndsch)
    x = solve_fn(s, acoef, _t(ss), _t(sp), _t(phi), relax=1.0, nswp=4000, tol=1e-9)
    gi = torch.tensor(gauges, device="cuda")
    loss = ((x[gi] - _t(target)) ** 2).sum()
    out = {"loss": float(loss.detach()), "acoef": acoef.detach().cpu().numpy(), "x": x.detach().cpu().numpy()}
    if grad:
        loss.backward()
        torch.cuda.synchronize()
        out.update(gv=V.grad.cpu().numpy(), gh=H.grad.cpu().numpy(), gf=F.grad.cpu().numpy())
    return out


@pytest.mark.parametrize("ndsch", [1, 2, 3, 4])
def test_momentum_coef_gradient_matches_tangent_linear(ndsch):
    case = _case(50 + ndsch)
    g, ss, sp, phi, visk, hk, ds, flux, mask, gauges, target = case
    n = g.ncells
    s = _solver(g)
    r = _run(s, case, ndsch, visk, hk, flux)
    ref = _acoef(ndsch, visk, hk, ds, flux, mask)
    assert np.abs(np.where(mask, r["acoef"], 0.0) - ref).max() <= 1e-14 * np.abs(ref).max()
    A, b = _system(g, ref, ss, sp, phi)
    xs = spl.spsolve(A, b)
    assert np.abs(r["x"][:n] - xs).max() <= 1e-8 * np.abs(xs).max()
    rng = np.random.default_rng(60 + ndsch)
    for _ in range(3):
        dv, dh, df = (rng.standard_normal(visk.shape) * mask * scale for scale in (visk, hk, flux))
        # the coefficients' directional derivative by central differences of the numpy functions
        e = 1e-6
        dac = (_acoef(ndsch, visk + e * dv, hk + e * dh, ds, flux + e * df, mask)
               - _acoef(ndsch, visk - e * dv, hk - e * dh, ds, flux - e * df, mask)) / (2 * e)
        A1, b1 = _system(g, ref + dac, ss, sp, phi)  # A and b are linear in acoef
        dx = spl.spsolve(A, (b1 - b) - (A1 - A) @ xs)
        tl = float(2.0 * np.sum((xs[gauges] - target) * dx[gauges]))
        ad = float((r["gv"] * dv).sum() + (r["gh"] * dh).sum() + (r["gf"] * df).sum())
        assert abs(ad - tl) <= 1e-6 * max(abs(tl), 1e-30), (ndsch, ad, tl)


@pytest.mark.parametrize("ndsch", [2, 4])
def test_momentum_coef_gradient_matches_finite_differences(ndsch):
    case = _case(70 + ndsch)
    g, ss, sp, phi, visk, hk, ds, flux, mask, gauges, target = case
    s = _solver(g)
    r = _run(s, case, ndsch, visk, hk, flux)
    rng = np.random.default_rng(80 + ndsch)
    for _ in range(2):
        dv, dh, df = (rng.standard_normal(visk.shape) * mask * scale for scale in (visk, hk, flux))
        eps = 1e-4
        lp = _run(s, case, ndsch, visk + eps * dv, hk + eps * dh, flux + eps * df, grad=False)["loss"]
        lm = _run(s, case, ndsch, visk - eps * dv, hk - eps * dh, flux - eps * df, grad=False)["loss"]
        fd = (lp - lm) / (2 * eps)
        ad = float((r["gv"] * dv).sum() + (r["gh"] * dh).sum() + (r["gf"] * df).sum())
        assert abs(ad - fd) <= 5e-5 * abs(fd), (ndsch, ad, fd)
