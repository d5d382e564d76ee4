"""Gradient of a gauge misfit of the pressure-correction solve with respect to
Manning's n, the momentum coefficients and the face depth: the Manning
friction sink (cms_fric_sink_dev_d) feeds the momentum diagonal, the
pressure-correction coefficients are built from the momentum system
(cms_pp_coef_dev_d, coefsourcesink_pp without the skewness correction), the
pressure-correction system is solved (solve()); the gradient comes from the
three hand-written adjoints (cms_pp_coef_adjoint_dev_d, the friction sink's,
solve()'s) through cms2d_b200.adjoint.

Forward model on a telescoping solver-test grid (all cells wet, relax 0.8):
sp_u = spuv0 - Cd(n) |u| A, acoef_pp = pp(acoef_u, sp_u, hk, ...),
x = solve(acoef_pp, ss, sp_pp, phi) (FP64, to 1e-10), L = sum over 200 seeded
gauge cells of (x_g - target_g)^2.  Face geometry is symmetric across each
face and the interpolation weights of its two sides add to 1.

Checks: the coefficients against the formula in numpy (1e-13); dL/d(n,
acoef_u, hk) against an FP64 CPU tangent-linear (the coefficients'
directional derivative by central differences of the numpy model, scipy
solves; 1e-6 relative) and against central finite differences of the GPU
forward model (5e-5).  The same again with the right-hand side built too
(cms_pp_rhs_dev_d: continuity source with the Rhie-Chow fluxes of
flow_imp_flux_noskew, Hu = u + ap dpx h; adjoint cms_pp_rhs_adjoint_dev_d),
so that n reaches both sides of the pressure-correction system; face
directions are opposite on the two sides of a face.
"""
import numpy as np
import pytest
import scipy.sparse.linalg as spl

from cms2d_b200 import grid as G
from cms2d_b200 import solver as S
from tests.helpers import interior_matrix

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

GRAV, RELAX = 9.81, 0.8


def _cd(nm, h):
    hh = np.maximum(np.minimum(10.0, h), 0.1 * nm)
    return GRAV * nm * nm / hh ** 0.3333


def _case(seed):
    g = G.solver_test_grid(6000)
    _, ss, _, phi = G.random_system(g, seed=seed)
    rng = np.random.default_rng(seed + 1)
    n, nD, nmf = g.ncells, g.ncellsD, g.nmaxfaces
    c2c = np.asarray(g.cell2cell, np.int32).reshape(nD, nmf)
    mask = np.arange(nmf)[None, :] < np.asarray(g.ncface)[:, None]
    mask[n:] = False
    shape = (nD, nmf)
    hk, ds, dn, fintp = (np.zeros(shape) for _ in range(4))
    for i in range(n):
        for k in range(g.ncface[i]):
            c = c2c[i, k] - 1
            if c >= n:
                hk[i, k], ds[i, k], dn[i, k], fintp[i, k] = rng.uniform(1, 3), rng.uniform(0.5, 2), \
                    rng.uniform(0.5, 2), 0.5
            elif c > i:
                kb = [q for q in range(g.ncface[c]) if c2c[c, q] - 1 == i][0]
                vals = rng.uniform(1, 3), rng.uniform(0.5, 2), rng.uniform(0.5, 2)
                u = rng.uniform(0.3, 0.7)
                hk[i, k], ds[i, k], dn[i, k], fintp[i, k] = *vals, u
                hk[c, kb], ds[c, kb], dn[c, kb], fintp[c, kb] = *vals, 1.0 - u
    acoef_u = np.where(mask, rng.uniform(0.2, 1.5, shape), 0.0)
    spuv0 = np.zeros(nD)
    spuv0[:n] = -rng.uniform(0.5, 1.5, n)
    nman = rng.uniform(0.015, 0.035, n)
    h = rng.uniform(0.3, 14.0, n)
    uv = rng.uniform(0.05, 1.2, n)
    area = np.zeros(nD)
    area[:n] = rng.uniform(50.0, 150.0, n)
    sp_pp = np.zeros(nD)
    sp_pp[:n] = -rng.uniform(20.0, 60.0, n)
    gauges = np.sort(rng.choice(n, 200, replace=False))
    target = rng.standard_normal(200)
    # right-hand side inputs: face directions opposite on the two sides of a face
    idir = np.zeros(shape, np.int32)
    opp = {1: 3, 3: 1, 2: 4, 4: 2}
    for i in range(n):
        for k in range(g.ncface[i]):
            c = c2c[i, k] - 1
            if c >= n:
                idir[i, k] = rng.integers(1, 5)
            elif c > i:
                kb = [q for q in range(g.ncface[c]) if c2c[c, q] - 1 == i][0]
                idir[i, k] = rng.integers(1, 5)
                idir[c, kb] = opp[int(idir[i, k])]
    cell = lambda lo, hi: np.concatenate([rng.uniform(lo, hi, n), np.zeros(nD - n)])
    u, v, dpx, dpy = cell(-1, 1), cell(-1, 1), cell(-0.01, 0.01), cell(-0.01, 0.01)
    p = rng.uniform(-1.0, 1.0, nD)
    sspp0 = cell(-5, 5)
    sppp0 = sp_pp.copy()
    hcell = np.concatenate([h, np.zeros(nD - n)])
    return dict(g=g, ss=ss, phi=phi, c2c=c2c, mask=mask, hk=hk, ds=ds, dn=dn, fintp=fintp, acoef_u=acoef_u,
                spuv0=spuv0, nman=nman, h=h, uv=uv, area=area, sp_pp=sp_pp, gauges=gauges, target=target,
                idir=idir, u=u, v=v, dpx=dpx, dpy=dpy, p=p, sspp0=sspp0, sppp0=sppp0, hcell=hcell)


def _pp_numpy(cs, nman, acoef_u, hk):
    """The forward model up to acoef_pp in numpy."""
    g, c2c, n = cs["g"], cs["c2c"], cs["g"].ncells
    sp_u = cs["spuv0"].copy()
    sp_u[:n] = cs["spuv0"][:n] - _cd(nman, cs["h"]) * cs["uv"] * cs["area"][:n]
    asum = acoef_u[:n].sum(axis=1)
    apu = RELAX / np.maximum(asum - sp_u[:n], 1e-6)
    ap, sumu = apu * cs["area"][:n], asum * apu
    out = np.zeros_like(acoef_u)
    for i in range(n):
        for k in range(g.ncface[i]):
            c = c2c[i, k] - 1
            K = hk[i, k] ** 2 * cs["ds"][i, k] / cs["dn"][i, k]
            if c >= n:
                out[i, k] = K * ap[i] / (1.0 - sumu[i])
            else:
                fk = cs["fintp"][i, k]
                out[i, k] = K * (fk * ap[c] + (1 - fk) * ap[i]) / (1.0 - (fk * sumu[c] + (1 - fk) * sumu[i]))
    return out


def _rhs_numpy(cs, nman, acoef_u, hk):
    """The pressure-correction right-hand side in numpy."""
    g, c2c, n = cs["g"], cs["c2c"], cs["g"].ncells
    sp_u = cs["spuv0"].copy()
    sp_u[:n] = cs["spuv0"][:n] - _cd(nman, cs["h"]) * cs["uv"] * cs["area"][:n]
    asum = acoef_u[:n].sum(axis=1)
    ap = RELAX / np.maximum(asum - sp_u[:n], 1e-6) * cs["area"][:n]
    hc, u, v, dpx, dpy, p = cs["hcell"], cs["u"], cs["v"], cs["dpx"], cs["dpy"], cs["p"]
    hu = u[:n] + ap * dpx[:n] * hc[:n]
    hv = v[:n] + ap * dpy[:n] * hc[:n]
    nxd = {1: 0.0, 2: 1.0, 3: 0.0, 4: -1.0}
    nyd = {1: 1.0, 2: 0.0, 3: -1.0, 4: 0.0}
    out = np.zeros(g.ncellsD)
    for i in range(n):
        sf = 0.0
        for k in range(g.ncface[i]):
            c = c2c[i, k] - 1
            d = int(cs["idir"][i, k])
            if c >= n:
                huf, hvf, apf = hu[i], hv[i], ap[i]
            else:
                fk = cs["fintp"][i, k]
                huf, hvf = fk * hu[c] + (1 - fk) * hu[i], fk * hv[c] + (1 - fk) * hv[i]
                apf = fk * ap[c] + (1 - fk) * ap[i]
            sf += hk[i, k] * cs["ds"][i, k] * (nxd[d] * huf + nyd[d] * hvf
                                               - apf * hk[i, k] * (p[c] - p[i]) / cs["dn"][i, k])
        out[i] = cs["sspp0"][i] - sf + p[i] * cs["sppp0"][i]
    return out


def _system(g, acoef, ss, sp, phi):
    n = g.ncells
    A = interior_matrix(g, acoef, sp, 1.0)
    b = ss[:n].copy()
    for k in range(g.nmaxfaces):
        c = g.cell2cell[:n, k]
        m = (k < g.ncface[:n]) & (c > n)
        b[m] += acoef[:n, k][m] * phi[c[m] - 1]
    return A.tocsc(), b


def _t(a, rg=False):
    return torch.tensor(a, dtype=torch.float64, device="cuda", requires_grad=rg)


def _run(s, cs, nman, acoef_u, hk, grad=True):
    from cms2d_b200.adjoint import friction_sink_fn, pp_coef_fn, solve_fn
    g = cs["g"]
    NM, AU, HK = _t(nman, grad), _t(acoef_u, grad), _t(hk, grad)
    area = _t(cs["area"])
    sp_u = friction_sink_fn(NM, _t(cs["h"]), _t(cs["uv"]), area, _t(cs["spuv0"]))
    i32 = lambda a: torch.tensor(np.ascontiguousarray(a, np.int32), device="cuda")
    app = pp_coef_fn(i32(cs["c2c"]), i32(g.ncface), i32(np.ones(g.ncellsD)), g.ncells, RELAX, AU, sp_u, area, HK,
                     _t(cs["ds"]), _t(cs["dn"]), _t(cs["fintp"]))
    x = solve_fn(s, app, _t(cs["ss"]), _t(cs["sp_pp"]), _t(cs["phi"]), relax=1.0, nswp=4000, tol=1e-9)
    gi = torch.tensor(cs["gauges"], device="cuda")
    loss = ((x[gi] - _t(cs["target"])) ** 2).sum()
    out = {"loss": float(loss.detach()), "app": app.detach().cpu().numpy(), "x": x.detach().cpu().numpy()}
    if grad:
        loss.backward()
        torch.cuda.synchronize()
        out.update(gn=NM.grad.cpu().numpy(), ga=AU.grad.cpu().numpy(), gh=HK.grad.cpu().numpy())
    return out


def _solver(g):
    return S.Solver(g, tol=1e-10, norm=2, max_iters=4000, verify=False, nsolv=3)


def _directions(cs, rng):
    mask = cs["mask"]
    return (cs["nman"] * rng.standard_normal(cs["nman"].shape),
            cs["acoef_u"] * rng.standard_normal(mask.shape) * mask,
            cs["hk"] * rng.standard_normal(mask.shape) * mask)


def test_pp_gradient_matches_tangent_linear():
    cs = _case(91)
    g, n = cs["g"], cs["g"].ncells
    s = _solver(g)
    r = _run(s, cs, cs["nman"], cs["acoef_u"], cs["hk"])
    ref = _pp_numpy(cs, cs["nman"], cs["acoef_u"], cs["hk"])
    assert np.abs(r["app"] - ref).max() <= 1e-13 * np.abs(ref).max()
    A, b = _system(g, ref, cs["ss"], cs["sp_pp"], cs["phi"])
    xs = spl.spsolve(A, b)
    assert np.abs(r["x"][:n] - xs).max() <= 1e-8 * np.abs(xs).max()
    rng = np.random.default_rng(93)
    for _ in range(3):
        dn_, da, dh = _directions(cs, rng)
        e = 1e-6
        dapp = (_pp_numpy(cs, cs["nman"] + e * dn_, cs["acoef_u"] + e * da, cs["hk"] + e * dh)
                - _pp_numpy(cs, cs["nman"] - e * dn_, cs["acoef_u"] - e * da, cs["hk"] - e * dh)) / (2 * e)
        A1, b1 = _system(g, ref + dapp, cs["ss"], cs["sp_pp"], cs["phi"])  # linear in acoef_pp
        dx = spl.spsolve(A, (b1 - b) - (A1 - A) @ xs)
        tl = float(2.0 * np.sum((xs[cs["gauges"]] - cs["target"]) * dx[cs["gauges"]]))
        ad = float(r["gn"] @ dn_ + (r["ga"] * da).sum() + (r["gh"] * dh).sum())
        assert abs(ad - tl) <= 1e-6 * max(abs(tl), 1e-30), (ad, tl)


def test_pp_gradient_matches_finite_differences():
    cs = _case(97)
    s = _solver(cs["g"])
    r = _run(s, cs, cs["nman"], cs["acoef_u"], cs["hk"])
    rng = np.random.default_rng(99)
    for _ in range(2):
        dn_, da, dh = _directions(cs, rng)
        eps = 1e-4
        lp = _run(s, cs, cs["nman"] + eps * dn_, cs["acoef_u"] + eps * da, cs["hk"] + eps * dh, grad=False)["loss"]
        lm = _run(s, cs, cs["nman"] - eps * dn_, cs["acoef_u"] - eps * da, cs["hk"] - eps * dh, grad=False)["loss"]
        fd = (lp - lm) / (2 * eps)
        ad = float(r["gn"] @ dn_ + (r["ga"] * da).sum() + (r["gh"] * dh).sum())
        assert abs(ad - fd) <= 5e-5 * abs(fd), (ad, fd)


def _run_full(s, cs, nman, acoef_u, hk, grad=True):
    """The whole pressure-correction system (coefficients and right-hand side)
    from n, the momentum coefficients and the face depth."""
    from cms2d_b200.adjoint import friction_sink_fn, pp_coef_fn, pp_rhs_fn, solve_fn
    g = cs["g"]
    NM, AU, HK = _t(nman, grad), _t(acoef_u, grad), _t(hk, grad)
    area = _t(cs["area"])
    sp_u = friction_sink_fn(NM, _t(cs["h"]), _t(cs["uv"]), area, _t(cs["spuv0"]))
    i32 = lambda a: torch.tensor(np.ascontiguousarray(a, np.int32), device="cuda")
    c2c, ncf, iwet = i32(cs["c2c"]), i32(g.ncface), i32(np.ones(g.ncellsD))
    app = pp_coef_fn(c2c, ncf, iwet, g.ncells, RELAX, AU, sp_u, area, HK, _t(cs["ds"]), _t(cs["dn"]),
                     _t(cs["fintp"]))
    ssp = pp_rhs_fn(c2c, ncf, i32(cs["idir"]), iwet, g.ncells, RELAX, AU, sp_u, area, HK, _t(cs["ds"]),
                    _t(cs["dn"]), _t(cs["fintp"]), _t(cs["u"]), _t(cs["v"]), _t(cs["hcell"]), _t(cs["dpx"]),
                    _t(cs["dpy"]), _t(cs["p"]), _t(cs["sspp0"]), _t(cs["sppp0"]))
    x = solve_fn(s, app, ssp, _t(cs["sp_pp"]), _t(cs["phi"]), relax=1.0, nswp=4000, tol=1e-9)
    gi = torch.tensor(cs["gauges"], device="cuda")
    loss = ((x[gi] - _t(cs["target"])) ** 2).sum()
    out = {"loss": float(loss.detach()), "ssp": ssp.detach().cpu().numpy(), "x": x.detach().cpu().numpy()}
    if grad:
        loss.backward()
        torch.cuda.synchronize()
        out.update(gn=NM.grad.cpu().numpy(), ga=AU.grad.cpu().numpy(), gh=HK.grad.cpu().numpy())
    return out


def test_pp_system_gradient_matches_tangent_linear():
    """Coefficients and right-hand side both from (n, acoef_u, hk)."""
    cs = _case(101)
    g, n = cs["g"], cs["g"].ncells
    s = _solver(g)
    r = _run_full(s, cs, cs["nman"], cs["acoef_u"], cs["hk"])
    rhs = _rhs_numpy(cs, cs["nman"], cs["acoef_u"], cs["hk"])
    assert np.abs(r["ssp"][:n] - rhs[:n]).max() <= 1e-12 * np.abs(rhs[:n]).max()
    ref = _pp_numpy(cs, cs["nman"], cs["acoef_u"], cs["hk"])
    A, b = _system(g, ref, rhs, cs["sp_pp"], cs["phi"])
    xs = spl.spsolve(A, b)
    assert np.abs(r["x"][:n] - xs).max() <= 1e-8 * np.abs(xs).max()
    rng = np.random.default_rng(103)
    for _ in range(3):
        dn_, da, dh = _directions(cs, rng)
        e = 1e-6
        args_p = (cs["nman"] + e * dn_, cs["acoef_u"] + e * da, cs["hk"] + e * dh)
        args_m = (cs["nman"] - e * dn_, cs["acoef_u"] - e * da, cs["hk"] - e * dh)
        dapp = (_pp_numpy(cs, *args_p) - _pp_numpy(cs, *args_m)) / (2 * e)
        drhs = (_rhs_numpy(cs, *args_p) - _rhs_numpy(cs, *args_m)) / (2 * e)
        A1, b1 = _system(g, ref + dapp, rhs + drhs, cs["sp_pp"], cs["phi"])  # linear in acoef_pp and ss
        dx = spl.spsolve(A, (b1 - b) - (A1 - A) @ xs)
        tl = float(2.0 * np.sum((xs[cs["gauges"]] - cs["target"]) * dx[cs["gauges"]]))
        ad = float(r["gn"] @ dn_ + (r["ga"] * da).sum() + (r["gh"] * dh).sum())
        assert abs(ad - tl) <= 1e-6 * max(abs(tl), 1e-30), (ad, tl)


def test_pp_system_gradient_matches_finite_differences():
    cs = _case(107)
    s = _solver(cs["g"])
    r = _run_full(s, cs, cs["nman"], cs["acoef_u"], cs["hk"])
    rng = np.random.default_rng(109)
    for _ in range(2):
        dn_, da, dh = _directions(cs, rng)
        eps = 1e-4
        lp = _run_full(s, cs, cs["nman"] + eps * dn_, cs["acoef_u"] + eps * da, cs["hk"] + eps * dh,
                       grad=False)["loss"]
        lm = _run_full(s, cs, cs["nman"] - eps * dn_, cs["acoef_u"] - eps * da, cs["hk"] - eps * dh,
                       grad=False)["loss"]
        fd = (lp - lm) / (2 * eps)
        ad = float(r["gn"] @ dn_ + (r["ga"] * da).sum() + (r["gh"] * dh).sum())
        assert abs(ad - fd) <= 5e-5 * abs(fd), (ad, fd)


# --- the momentum predictor in the chain: u, v = solve(acoef_u, su / sv, sp_u, .),
# then the pressure-correction system from (n, acoef_u, hk, u, v)

def _momentum_case(cs, seed):
    rng = np.random.default_rng(seed)
    g = cs["g"]
    n, nD = g.ncells, g.ncellsD
    cs = dict(cs)
    cs["su"] = np.concatenate([rng.uniform(-2, 2, n), np.zeros(nD - n)])
    cs["sv"] = np.concatenate([rng.uniform(-2, 2, n), np.zeros(nD - n)])
    cs["u0"] = rng.uniform(-0.5, 0.5, nD)
    cs["v0"] = rng.uniform(-0.5, 0.5, nD)
    return cs


def _uv_numpy(cs, nman, acoef_u):
    g, n = cs["g"], cs["g"].ncells
    sp_u = cs["spuv0"].copy()
    sp_u[:n] = cs["spuv0"][:n] - _cd(nman, cs["h"]) * cs["uv"] * cs["area"][:n]
    out = []
    for rhs, x0 in ((cs["su"], cs["u0"]), (cs["sv"], cs["v0"])):
        A, b = _system(g, acoef_u, rhs, sp_u, x0)
        x = x0.copy()
        x[:n] = spl.spsolve(A, b)
        out.append(x)
    return out


def _system_numpy(cs, nman, acoef_u, hk):
    u, v = _uv_numpy(cs, nman, acoef_u)
    cs2 = dict(cs, u=u, v=v)
    return _pp_numpy(cs, nman, acoef_u, hk), _rhs_numpy(cs2, nman, acoef_u, hk)


def _run_outer(s, cs, nman, acoef_u, hk, grad=True):
    from cms2d_b200.adjoint import friction_sink_fn, pp_coef_fn, pp_rhs_fn, solve_fn
    g = cs["g"]
    NM, AU, HK = _t(nman, grad), _t(acoef_u, grad), _t(hk, grad)
    area = _t(cs["area"])
    sp_u = friction_sink_fn(NM, _t(cs["h"]), _t(cs["uv"]), area, _t(cs["spuv0"]))
    u = solve_fn(s, AU, _t(cs["su"]), sp_u, _t(cs["u0"]), relax=1.0, nswp=4000, tol=1e-9)
    v = solve_fn(s, AU, _t(cs["sv"]), sp_u, _t(cs["v0"]), relax=1.0, nswp=4000, tol=1e-9)
    i32 = lambda a: torch.tensor(np.ascontiguousarray(a, np.int32), device="cuda")
    c2c, ncf, iwet = i32(cs["c2c"]), i32(g.ncface), i32(np.ones(g.ncellsD))
    app = pp_coef_fn(c2c, ncf, iwet, g.ncells, RELAX, AU, sp_u, area, HK, _t(cs["ds"]), _t(cs["dn"]),
                     _t(cs["fintp"]))
    ssp = pp_rhs_fn(c2c, ncf, i32(cs["idir"]), iwet, g.ncells, RELAX, AU, sp_u, area, HK, _t(cs["ds"]),
                    _t(cs["dn"]), _t(cs["fintp"]), u, v, _t(cs["hcell"]), _t(cs["dpx"]), _t(cs["dpy"]),
                    _t(cs["p"]), _t(cs["sspp0"]), _t(cs["sppp0"]))
    x = solve_fn(s, app, ssp, _t(cs["sp_pp"]), _t(cs["phi"]), relax=1.0, nswp=4000, tol=1e-9)
    gi = torch.tensor(cs["gauges"], device="cuda")
    loss = ((x[gi] - _t(cs["target"])) ** 2).sum()
    out = {"loss": float(loss.detach()), "x": x.detach().cpu().numpy(), "u": u.detach().cpu().numpy()}
    if grad:
        loss.backward()
        torch.cuda.synchronize()
        out.update(gn=NM.grad.cpu().numpy(), ga=AU.grad.cpu().numpy(), gh=HK.grad.cpu().numpy())
    return out


def test_outer_iteration_gradient_matches_tangent_linear():
    """n, the momentum coefficients and hk through the momentum predictor
    (u and v solves) and the whole pressure-correction system."""
    cs = _momentum_case(_case(111), 113)
    g, n = cs["g"], cs["g"].ncells
    s = _solver(g)
    r = _run_outer(s, cs, cs["nman"], cs["acoef_u"], cs["hk"])
    u_np, _ = _uv_numpy(cs, cs["nman"], cs["acoef_u"])
    assert np.abs(r["u"][:n] - u_np[:n]).max() <= 1e-8 * np.abs(u_np[:n]).max()
    app, rhs = _system_numpy(cs, cs["nman"], cs["acoef_u"], cs["hk"])
    A, b = _system(g, app, rhs, cs["sp_pp"], cs["phi"])
    xs = spl.spsolve(A, b)
    assert np.abs(r["x"][:n] - xs).max() <= 1e-8 * np.abs(xs).max()
    rng = np.random.default_rng(117)
    for _ in range(3):
        dn_, da, dh = _directions(cs, rng)
        e = 1e-6
        ap_p, rhs_p = _system_numpy(cs, cs["nman"] + e * dn_, cs["acoef_u"] + e * da, cs["hk"] + e * dh)
        ap_m, rhs_m = _system_numpy(cs, cs["nman"] - e * dn_, cs["acoef_u"] - e * da, cs["hk"] - e * dh)
        A1, b1 = _system(g, app + (ap_p - ap_m) / (2 * e), rhs + (rhs_p - rhs_m) / (2 * e), cs["sp_pp"], cs["phi"])
        dx = spl.spsolve(A, (b1 - b) - (A1 - A) @ xs)
        tl = float(2.0 * np.sum((xs[cs["gauges"]] - cs["target"]) * dx[cs["gauges"]]))
        ad = float(r["gn"] @ dn_ + (r["ga"] * da).sum() + (r["gh"] * dh).sum())
        assert abs(ad - tl) <= 1e-6 * max(abs(tl), 1e-30), (ad, tl)


def test_outer_iteration_gradient_matches_finite_differences():
    cs = _momentum_case(_case(119), 121)
    s = _solver(cs["g"])
    r = _run_outer(s, cs, cs["nman"], cs["acoef_u"], cs["hk"])
    rng = np.random.default_rng(123)
    for _ in range(2):
        dn_, da, dh = _directions(cs, rng)
        eps = 1e-4
        lp = _run_outer(s, cs, cs["nman"] + eps * dn_, cs["acoef_u"] + eps * da, cs["hk"] + eps * dh,
                        grad=False)["loss"]
        lm = _run_outer(s, cs, cs["nman"] - eps * dn_, cs["acoef_u"] - eps * da, cs["hk"] - eps * dh,
                        grad=False)["loss"]
        fd = (lp - lm) / (2 * eps)
        ad = float(r["gn"] @ dn_ + (r["ga"] * da).sum() + (r["gh"] * dh).sum())
        assert abs(ad - fd) <= 5e-5 * abs(fd), (ad, fd)


def test_water_level_misfit_gradient_matches_finite_differences():
    """The loss config 5 names: gauge water-level misfit after the outer
    iteration's pressure correction, eta = (p + pp) / g (pvfc with
    relax_p = 1, flow_imp.F90:797-1072), as a function of per-cell Manning's n
    through the chain above."""
    from cms2d_b200.adjoint import friction_sink_fn, pp_coef_fn, pp_rhs_fn, solve_fn
    cs = _momentum_case(_case(127), 129)
    g = cs["g"]
    s = _solver(g)
    rng = np.random.default_rng(131)
    eta_obs = rng.standard_normal(200) * 0.1

    def loss(nman, grad):
        NM = _t(nman, grad)
        AU, HK, area = _t(cs["acoef_u"]), _t(cs["hk"]), _t(cs["area"])
        sp_u = friction_sink_fn(NM, _t(cs["h"]), _t(cs["uv"]), area, _t(cs["spuv0"]))
        u = solve_fn(s, AU, _t(cs["su"]), sp_u, _t(cs["u0"]), relax=1.0, nswp=4000, tol=1e-9)
        v = solve_fn(s, AU, _t(cs["sv"]), sp_u, _t(cs["v0"]), relax=1.0, nswp=4000, tol=1e-9)
        i32 = lambda a: torch.tensor(np.ascontiguousarray(a, np.int32), device="cuda")
        c2c, ncf, iwet = i32(cs["c2c"]), i32(g.ncface), i32(np.ones(g.ncellsD))
        app = pp_coef_fn(c2c, ncf, iwet, g.ncells, RELAX, AU, sp_u, area, HK, _t(cs["ds"]), _t(cs["dn"]),
                         _t(cs["fintp"]))
        ssp = pp_rhs_fn(c2c, ncf, i32(cs["idir"]), iwet, g.ncells, RELAX, AU, sp_u, area, HK, _t(cs["ds"]),
                        _t(cs["dn"]), _t(cs["fintp"]), u, v, _t(cs["hcell"]), _t(cs["dpx"]), _t(cs["dpy"]),
                        _t(cs["p"]), _t(cs["sspp0"]), _t(cs["sppp0"]))
        pp = solve_fn(s, app, ssp, _t(cs["sp_pp"]), torch.zeros(g.ncellsD, dtype=torch.float64, device="cuda"),
                      relax=1.0, nswp=4000, tol=1e-9)
        gi = torch.tensor(cs["gauges"], device="cuda")
        eta = (_t(cs["p"])[gi] + pp[gi]) / GRAV
        L = ((eta - _t(eta_obs)) ** 2).sum()
        if grad:
            L.backward()
            torch.cuda.synchronize()
            return float(L.detach()), NM.grad.cpu().numpy()
        return float(L.detach()), None

    _, gn = loss(cs["nman"], True)
    assert np.isfinite(gn).all() and np.abs(gn).max() > 0
    for _ in range(2):
        dn_ = cs["nman"] * rng.standard_normal(cs["nman"].shape)
        eps = 1e-4
        fd = (loss(cs["nman"] + eps * dn_, False)[0] - loss(cs["nman"] - eps * dn_, False)[0]) / (2 * eps)
        ad = float(gn @ dn_)
        assert abs(ad - fd) <= 5e-5 * abs(fd), (ad, fd)
