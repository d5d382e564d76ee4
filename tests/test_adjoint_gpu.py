"""Adjoint of solve() (cms_solver_adjoint_dev_d, cms2d_b200.adjoint.solve_fn).

Checks: (1) dL/dss = lam = A^-T w against a direct FP64 solve of the
transposed system (scipy); (2) the gradients of acoef, ss and sp against an
FP64 CPU tangent-linear of the same solve (dx = A^-1 (db - dA x), scipy) in
random directions, with and without under-relaxation and with non-zero
dummy-cell values; (3) against central finite differences of the GPU forward
solve.  FP64 solves to 1e-10 (relative L2; BiCGStab stagnates near 4e-11
on these systems, the reference's algorithm on the CPU alike), so solutions
carry ~1e-9 relative error; bounds 1e-8 (lam, x), 1e-7 (tangent-linear) and,
for finite differences with h = 3e-4 (truncation ~1e-6, solve noise ~3e-6),
5e-5 relative.
"""
import numpy as np
import pytest
import scipy.sparse.linalg as spl

from cms2d_b200 import grid as G
from cms2d_b200 import solver as S
from tests.helpers import interior_matrix

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _case(seed, relax):
    g = G.solver_test_grid(6000)
    acoef, ss, sp, phi = G.random_system(g, seed=seed)
    rng = np.random.default_rng(seed + 100)
    phi[:] = rng.standard_normal(g.ncellsD)  # initial guess and dummy values
    return g, acoef, ss, sp, phi


def _system(g, acoef, ss, sp, phi, relax):
    """solve()'s A (active cells) and b in numpy."""
    n = g.ncells
    A = interior_matrix(g, acoef, sp, relax)
    ap = (acoef[:n].sum(axis=1) - sp[:n]) / relax
    b = ss[:n] + (1 - relax) * phi[:n] * ap
    for k in range(g.nmaxfaces):
        c = g.cell2cell[:n, k]
        m = (k < g.ncface[:n]) & (c > n)
        b[m] += acoef[:n, k][m] * phi[c[m] - 1]
    return A.tocsc(), b


def _solver(g):
    return S.Solver(g, tol=1e-10, norm=2, max_iters=4000, verify=False, nsolv=3)


def _grads(s, g, acoef, ss, sp, phi, relax, w):
    from cms2d_b200.adjoint import solve_fn
    t = lambda a, rg=False: torch.tensor(a, dtype=torch.float64, device="cuda", requires_grad=rg)
    A, SS, SP = t(acoef, True), t(ss, True), t(sp, True)
    x = solve_fn(s, A, SS, SP, t(phi), relax=relax, nswp=4000, tol=1e-9)
    (x * t(w)).sum().backward()
    torch.cuda.synchronize()
    return x.detach().cpu().numpy(), A.grad.cpu().numpy(), SS.grad.cpu().numpy(), SP.grad.cpu().numpy()


def _weights(g, seed):
    w = np.random.default_rng(seed).standard_normal(g.ncellsD)
    w[g.ncells:] = 0.0  # the loss sees active cells (dummies pass through)
    return w


def test_lambda_matches_direct_transposed_solve():
    g, acoef, ss, sp, phi = _case(3, 1.0)
    s = _solver(g)
    w = _weights(g, 7)
    x, gac, gss, gsp = _grads(s, g, acoef, ss, sp, phi, 1.0, w)
    A, b = _system(g, acoef, ss, sp, phi, 1.0)
    n = g.ncells
    lam = spl.spsolve(A.T.tocsc(), w[:n])
    assert np.abs(gss[:n] - lam).max() <= 1e-8 * np.abs(lam).max()
    assert np.abs(x[:n] - spl.spsolve(A, b)).max() <= 1e-8 * np.abs(x[:n]).max()
    assert s.last_adjoint["relres"] <= 1e-8, s.last_adjoint  # at or below its stagnation level


@pytest.mark.parametrize("relax", [1.0, 0.8])
def test_gradients_match_tangent_linear(relax):
    g, acoef, ss, sp, phi = _case(5, relax)
    n = g.ncells
    s = _solver(g)
    w = _weights(g, 11)
    x, gac, gss, gsp = _grads(s, g, acoef, ss, sp, phi, relax, w)
    A, b = _system(g, acoef, ss, sp, phi, relax)
    xs = spl.spsolve(A, b)
    rng = np.random.default_rng(17)
    mask = np.arange(g.nmaxfaces)[None, :] < g.ncface[:, None]
    mask[n:] = False
    for _ in range(4):
        da = rng.standard_normal(acoef.shape) * mask
        dss = np.zeros_like(ss); dss[:n] = rng.standard_normal(n)
        dsp = np.zeros_like(sp); dsp[:n] = rng.standard_normal(n)
        # tangent-linear: A(a + e da) x = b(...), dx = A^-1 (db - dA x)
        eps = 1.0
        A1, b1 = _system(g, acoef + eps * da, ss + eps * dss, sp + eps * dsp, phi, relax)
        dA = A1 - A
        db = b1 - b
        dx = spl.spsolve(A, db - dA @ xs)
        tl = float(w[:n] @ dx)
        ad = float((gac * da).sum() + (gss * dss).sum() + (gsp * dsp).sum())
        assert abs(ad - tl) <= 1e-7 * max(abs(tl), 1e-30), (ad, tl)


def test_gradients_match_finite_differences():
    g, acoef, ss, sp, phi = _case(9, 1.0)
    n = g.ncells
    s = _solver(g)
    w = _weights(g, 13)
    x, gac, gss, gsp = _grads(s, g, acoef, ss, sp, phi, 1.0, w)
    rng = np.random.default_rng(23)
    mask = np.arange(g.nmaxfaces)[None, :] < g.ncface[:, None]
    mask[n:] = False

    def loss(a, q, p):
        aa, qq, pp, ph = (np.ascontiguousarray(v).copy() for v in (a, q, p, phi))
        s.solve(aa, qq, pp, np.zeros_like(qq), ph, relax=1.0, nswp=4000, nsolv=3)
        return float(w @ ph)

    for _ in range(3):
        da = rng.standard_normal(acoef.shape) * mask
        dsp = np.zeros_like(sp); dsp[:n] = rng.standard_normal(n)
        h = 3e-4
        fd = (loss(acoef + h * da, ss, sp + h * dsp) - loss(acoef - h * da, ss, sp - h * dsp)) / (2 * h)
        ad = float((gac * da).sum() + (gsp * dsp).sum())
        assert abs(ad - fd) <= 5e-5 * abs(fd), (ad, fd)
