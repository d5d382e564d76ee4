"""Differentiable solve(): the adjoint of the reference's solve() boundary.

``solve_fn(solver, acoef, ss, sp, phi, relax=1.0, nswp=..., tol=...)`` runs the
forward solve on the GPU (``cms_solver_solve_dev_d``) and returns x (phi after
the solve).  Its backward pass solves A^T lam = dL/dx on the GPU
(``cms_solver_adjoint_dev_d``: ILU(0)-BiCGStab on the transposed system) and
returns dL/dacoef, dL/dss and dL/dsp in the solve() layout.  FP64 CUDA
tensors, natural order, acoef [ncellsD, nmaxfaces].

``friction_sink_fn(coefman, h, uv, area, spuv0)`` is the momentum equations'
bottom-friction sink sp = spuv0 - Cd(n) |u| A with the Manning closure
(``cms_fric_sink_dev_d``); its backward pass (``cms_fric_sink_adjoint_dev_d``)
turns dL/dsp into dL/dn.  Chained with ``solve_fn`` it gives the gradient of
a loss on a momentum solve's solution with respect to per-cell Manning's n,
with the depth, the speed |u| and the cell areas held fixed.

``momentum_coef_fn(ncface, ncells, visk, hk, ds, flux, ndsch)`` is the
momentum equations' face coefficients acoef = scheme(visk hk ds, flux)
(``cms_momentum_coef_dev_d``, the ADVECTION_SCHEME functions); its backward
pass (``cms_momentum_coef_adjoint_dev_d``) gives dL/dvisk, dL/dhk and
dL/dflux from dL/dacoef.

``pp_coef_fn(...)`` is the pressure-correction coefficients built from the
momentum system (``cms_pp_coef_dev_d``, coefsourcesink_pp without the
skewness correction); its backward pass (``cms_pp_coef_adjoint_dev_d``)
gives dL/dacoef_u, dL/dsp_u and dL/dhk.  Chained with friction_sink_fn and
solve_fn, Manning's n reaches the pressure-correction solve through the
momentum diagonal.  ``pp_rhs_fn(...)`` is that system's right-hand side
(continuity source with the Rhie-Chow fluxes, ``cms_pp_rhs_dev_d``), with the
same gradients (``cms_pp_rhs_adjoint_dev_d``).
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib


def _bind(L):
    if getattr(L, "_adj_bound", False):
        return
    vp, d, i = C.c_void_p, C.c_double, C.c_int
    L.cms_solver_adjoint_dev_d.argtypes = [vp] * 6 + [d, vp, d, i] + [vp] * 4 + [C.POINTER(_lib.SolveInfo)]
    L.cms_fric_sink_dev_d.argtypes = [i, d] + [vp] * 7
    L.cms_fric_sink_adjoint_dev_d.argtypes = [i, d] + [vp] * 7
    L.cms_momentum_coef_dev_d.argtypes = [i, i, i] + [vp] * 7
    L.cms_momentum_coef_adjoint_dev_d.argtypes = [i, i, i] + [vp] * 10
    L.cms_pp_coef_dev_d.argtypes = [i, i, vp, vp, vp, d] + [vp] * 9
    L.cms_pp_coef_adjoint_dev_d.argtypes = [i, i, vp, vp, vp, d] + [vp] * 12
    L.cms_pp_rhs_dev_d.argtypes = [i, i, vp, vp, vp, vp, d] + [vp] * 17
    L.cms_pp_rhs_adjoint_dev_d.argtypes = [i, i, vp, vp, vp, vp, d] + [vp] * 20
    L._adj_bound = True


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


class _SolveFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, acoef, ss, sp, phi, solver, relax, nswp, tol):
        x = phi.detach().clone()
        ss_w = ss.detach().clone()
        res = torch.zeros_like(ss_w)
        solver.solve(acoef.detach(), ss_w, sp.detach(), res, x, relax=relax, nswp=nswp, nsolv=3)
        ctx.save_for_backward(acoef.detach(), ss.detach(), sp.detach(), phi.detach(), x)
        ctx.solver, ctx.relax, ctx.tol, ctx.maxit = solver, float(relax), float(tol), int(max(nswp, 1))
        ctx.mark_non_differentiable(res)
        return x

    @staticmethod
    def backward(ctx, gx):
        acoef, ss, sp, phi, x = ctx.saved_tensors
        L = _lib.lib()
        _bind(L)
        g = gx.detach().to(torch.float64).contiguous()
        lam = torch.zeros_like(ss)
        gac = torch.zeros_like(acoef) if ctx.needs_input_grad[0] else None
        gss = torch.zeros_like(ss) if ctx.needs_input_grad[1] else None
        gsp = torch.zeros_like(sp) if ctx.needs_input_grad[2] else None
        torch.cuda.current_stream(g.device).synchronize()
        info = _lib.SolveInfo()
        rc = L.cms_solver_adjoint_dev_d(ctx.solver._h, _ptr(acoef), _ptr(ss), _ptr(sp), _ptr(phi), _ptr(x),
                                        ctx.relax, _ptr(g), ctx.tol, ctx.maxit, _ptr(lam), _ptr(gac), _ptr(gss),
                                        _ptr(gsp), C.byref(info))
        _lib.check(rc, "cms_solver_adjoint_dev_d", allow=(_lib.CMS_OK, _lib.CMS_NOT_CONVERGED))
        ctx.solver.last_adjoint = info.as_dict()
        return gac, gss, gsp, None, None, None, None, None


def solve_fn(solver, acoef, ss, sp, phi, relax: float = 1.0, nswp: int = 2000, tol: float = 1e-9):
    """x = solve(acoef, ss, sp, phi) with gradients for acoef, ss and sp.

    The solver's own options set the forward stopping test (use a tight
    tolerance, norm 2, FP64 for gradients); tol and nswp bound the adjoint
    solve."""
    return _SolveFn.apply(acoef, ss, sp, phi, solver, relax, nswp, tol)


class _FricSinkFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, coefman, h, uv, area, spuv0, grav):
        n = coefman.numel()
        sp = spuv0.detach().clone()
        L = _lib.lib()
        _bind(L)
        stream = C.c_void_p(torch.cuda.current_stream(coefman.device).cuda_stream)
        rc = L.cms_fric_sink_dev_d(n, float(grav), _ptr(coefman.detach()), _ptr(h), _ptr(uv), _ptr(area),
                                   _ptr(spuv0.detach()), _ptr(sp), stream)
        _lib.check(rc, "cms_fric_sink_dev_d")
        ctx.save_for_backward(coefman.detach(), h, uv, area)
        ctx.grav = float(grav)
        return sp

    @staticmethod
    def backward(ctx, gsp):
        coefman, h, uv, area = ctx.saved_tensors
        n = coefman.numel()
        g = gsp.detach().to(torch.float64).contiguous()
        gn = torch.empty_like(coefman)
        L = _lib.lib()
        _bind(L)
        stream = C.c_void_p(torch.cuda.current_stream(coefman.device).cuda_stream)
        rc = L.cms_fric_sink_adjoint_dev_d(n, ctx.grav, _ptr(coefman), _ptr(h), _ptr(uv), _ptr(area), _ptr(g),
                                           _ptr(gn), stream)
        _lib.check(rc, "cms_fric_sink_adjoint_dev_d")
        gsp0 = g if ctx.needs_input_grad[4] else None
        return gn, None, None, None, gsp0, None


def friction_sink_fn(coefman, h, uv, area, spuv0, grav: float = 9.81):
    """sp = spuv0 - Cd(n) |u| A over the first coefman.numel() cells (the
    rest of spuv0, e.g. dummy cells, is copied), with gradients for coefman
    (Manning's n) and spuv0.  FP64 CUDA tensors; h, uv and area are held
    fixed."""
    for t in (coefman, h, uv, area, spuv0):
        if t.dtype != torch.float64 or not t.is_cuda or not t.is_contiguous():
            raise ValueError("friction_sink_fn takes contiguous float64 CUDA tensors")
    if not (h.numel() >= coefman.numel() and uv.numel() >= coefman.numel() and area.numel() >= coefman.numel()
            and spuv0.numel() >= coefman.numel()):
        raise ValueError("h, uv, area and spuv0 need at least coefman.numel() entries")
    return _FricSinkFn.apply(coefman, h, uv, area, spuv0, grav)


class _MomCoefFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, visk, hk, flux, ds, ncface, ncells, ndsch):
        nD, nmf = visk.shape
        acoef = torch.zeros_like(visk)
        L = _lib.lib()
        _bind(L)
        stream = C.c_void_p(torch.cuda.current_stream(visk.device).cuda_stream)
        rc = L.cms_momentum_coef_dev_d(int(ncells), int(nmf), int(ndsch), _ptr(ncface), _ptr(visk.detach()),
                                       _ptr(hk.detach()), _ptr(ds), _ptr(flux.detach()), _ptr(acoef), stream)
        _lib.check(rc, "cms_momentum_coef_dev_d")
        ctx.save_for_backward(visk.detach(), hk.detach(), flux.detach(), ds, ncface)
        ctx.ncells, ctx.ndsch = int(ncells), int(ndsch)
        return acoef

    @staticmethod
    def backward(ctx, ga):
        visk, hk, flux, ds, ncface = ctx.saved_tensors
        g = ga.detach().to(torch.float64).contiguous()
        gv = torch.zeros_like(visk) if ctx.needs_input_grad[0] else None
        gh = torch.zeros_like(hk) if ctx.needs_input_grad[1] else None
        gf = torch.zeros_like(flux) if ctx.needs_input_grad[2] else None
        L = _lib.lib()
        _bind(L)
        stream = C.c_void_p(torch.cuda.current_stream(visk.device).cuda_stream)
        rc = L.cms_momentum_coef_adjoint_dev_d(ctx.ncells, int(visk.shape[1]), ctx.ndsch, _ptr(ncface), _ptr(visk),
                                               _ptr(hk), _ptr(ds), _ptr(flux), _ptr(g), _ptr(gv), _ptr(gh),
                                               _ptr(gf), stream)
        _lib.check(rc, "cms_momentum_coef_adjoint_dev_d")
        return gv, gh, gf, None, None, None, None


def momentum_coef_fn(ncface, ncells: int, visk, hk, ds, flux, ndsch: int = 4):
    """acoef [ncellsD, nmaxfaces] = scheme(visk hk ds, flux) on the faces of
    the active cells (zero elsewhere), with gradients for visk, hk and flux.
    FP64 CUDA tensors of acoef's shape for the face fields, int32 ncface."""
    for t in (visk, hk, ds, flux):
        if t.dtype != torch.float64 or not t.is_cuda or not t.is_contiguous() or t.shape != visk.shape:
            raise ValueError("momentum_coef_fn takes contiguous float64 CUDA face arrays of one shape")
    if ncface.dtype != torch.int32 or not ncface.is_cuda or ncface.numel() < ncells:
        raise ValueError("ncface: int32 CUDA tensor with an entry per active cell")
    return _MomCoefFn.apply(visk, hk, flux, ds, ncface, ncells, ndsch)


class _PPCoefFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, acoef_u, sp_u, hk, geo):
        c2c, ncface, iwet, relax, area, ds, dn, fintp, ncells = geo
        nD, nmf = acoef_u.shape
        out = torch.zeros_like(acoef_u)
        L = _lib.lib()
        _bind(L)
        stream = C.c_void_p(torch.cuda.current_stream(acoef_u.device).cuda_stream)
        rc = L.cms_pp_coef_dev_d(int(ncells), int(nmf), _ptr(c2c), _ptr(ncface), _ptr(iwet), float(relax),
                                 _ptr(acoef_u.detach()), _ptr(sp_u.detach()), _ptr(area), _ptr(hk.detach()),
                                 _ptr(ds), _ptr(dn), _ptr(fintp), _ptr(out), stream)
        _lib.check(rc, "cms_pp_coef_dev_d")
        ctx.save_for_backward(acoef_u.detach(), sp_u.detach(), hk.detach())
        ctx.geo = geo
        return out

    @staticmethod
    def backward(ctx, ga):
        acoef_u, sp_u, hk = ctx.saved_tensors
        c2c, ncface, iwet, relax, area, ds, dn, fintp, ncells = ctx.geo
        g = ga.detach().to(torch.float64).contiguous()
        gac = torch.zeros_like(acoef_u) if ctx.needs_input_grad[0] else None
        gsp = torch.zeros_like(sp_u) if ctx.needs_input_grad[1] else None
        ghk = torch.zeros_like(hk) if ctx.needs_input_grad[2] else None
        L = _lib.lib()
        _bind(L)
        stream = C.c_void_p(torch.cuda.current_stream(acoef_u.device).cuda_stream)
        rc = L.cms_pp_coef_adjoint_dev_d(int(ncells), int(acoef_u.shape[1]), _ptr(c2c), _ptr(ncface), _ptr(iwet),
                                         float(relax), _ptr(acoef_u), _ptr(sp_u), _ptr(area), _ptr(hk), _ptr(ds),
                                         _ptr(dn), _ptr(fintp), _ptr(g), _ptr(gac), _ptr(gsp), _ptr(ghk), stream)
        _lib.check(rc, "cms_pp_coef_adjoint_dev_d")
        return gac, gsp, ghk, None


def pp_coef_fn(cell2cell, ncface, iwet, ncells: int, relax: float, acoef_u, sp_u, area, hk, ds, dn, fintp):
    """Pressure-correction coefficients [ncellsD, nmaxfaces] from the momentum
    system (acoef_u, sp_u), with gradients for acoef_u, sp_u and hk.  int32
    CUDA tensors cell2cell (1-based, [ncellsD, nmaxfaces]), ncface, iwet
    (ncellsD entries); float64 CUDA tensors otherwise (face fields of
    acoef_u's shape, area per cell)."""
    for t in (cell2cell, ncface, iwet):
        if t.dtype != torch.int32 or not t.is_cuda or not t.is_contiguous():
            raise ValueError("cell2cell, ncface, iwet: contiguous int32 CUDA tensors")
    for t in (acoef_u, hk, ds, dn, fintp):
        if t.dtype != torch.float64 or not t.is_cuda or not t.is_contiguous() or t.shape != acoef_u.shape:
            raise ValueError("face fields: contiguous float64 CUDA tensors of acoef_u's shape")
    for t in (sp_u, area):
        if t.dtype != torch.float64 or not t.is_cuda or not t.is_contiguous():
            raise ValueError("sp_u, area: contiguous float64 CUDA tensors")
    geo = (cell2cell, ncface, iwet, relax, area, ds, dn, fintp, ncells)
    return _PPCoefFn.apply(acoef_u, sp_u, hk, geo)


class _PPRhsFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, acoef_u, sp_u, hk, u, v, geo):
        c2c, ncface, idir, iwet, relax, area, h, dpx, dpy, p, ds, dn, fintp, sspp0, sppp0, ncells = geo
        u, v = u.detach().contiguous(), v.detach().contiguous()
        out = torch.zeros_like(sspp0)
        L = _lib.lib()
        _bind(L)
        stream = C.c_void_p(torch.cuda.current_stream(acoef_u.device).cuda_stream)
        rc = L.cms_pp_rhs_dev_d(int(ncells), int(acoef_u.shape[1]), _ptr(c2c), _ptr(ncface), _ptr(idir),
                                _ptr(iwet), float(relax), _ptr(acoef_u.detach()), _ptr(sp_u.detach()), _ptr(area),
                                _ptr(u), _ptr(v), _ptr(h), _ptr(dpx), _ptr(dpy), _ptr(p), _ptr(hk.detach()),
                                _ptr(ds), _ptr(dn), _ptr(fintp), _ptr(sspp0), _ptr(sppp0), _ptr(out), stream)
        _lib.check(rc, "cms_pp_rhs_dev_d")
        ctx.save_for_backward(acoef_u.detach(), sp_u.detach(), hk.detach(), u, v)
        ctx.geo = geo
        return out

    @staticmethod
    def backward(ctx, gs):
        acoef_u, sp_u, hk, u, v = ctx.saved_tensors
        c2c, ncface, idir, iwet, relax, area, h, dpx, dpy, p, ds, dn, fintp, sspp0, sppp0, ncells = ctx.geo
        g = gs.detach().to(torch.float64).contiguous()
        gac = torch.zeros_like(acoef_u) if ctx.needs_input_grad[0] else None
        gsp = torch.zeros_like(sp_u) if ctx.needs_input_grad[1] else None
        ghk = torch.zeros_like(hk) if ctx.needs_input_grad[2] else None
        gu = torch.zeros_like(u) if ctx.needs_input_grad[3] else None
        gv = torch.zeros_like(v) if ctx.needs_input_grad[4] else None
        L = _lib.lib()
        _bind(L)
        stream = C.c_void_p(torch.cuda.current_stream(acoef_u.device).cuda_stream)
        rc = L.cms_pp_rhs_adjoint_dev_d(int(ncells), int(acoef_u.shape[1]), _ptr(c2c), _ptr(ncface), _ptr(idir),
                                        _ptr(iwet), float(relax), _ptr(acoef_u), _ptr(sp_u), _ptr(area), _ptr(u),
                                        _ptr(v), _ptr(h), _ptr(dpx), _ptr(dpy), _ptr(p), _ptr(hk), _ptr(ds), _ptr(dn),
                                        _ptr(fintp), _ptr(g), _ptr(gac), _ptr(gsp), _ptr(ghk), _ptr(gu), _ptr(gv),
                                        stream)
        _lib.check(rc, "cms_pp_rhs_adjoint_dev_d")
        return gac, gsp, ghk, gu, gv, None


def pp_rhs_fn(cell2cell, ncface, idirface, iwet, ncells: int, relax: float, acoef_u, sp_u, area, hk, ds, dn, fintp,
              u, v, h, dpx, dpy, p, sspp0, sppp0):
    """Right-hand side [ncellsD] of the pressure-correction system (entries
    of the active cells; zero beyond), with gradients for acoef_u, sp_u, hk,
    u and v; the cell fields h, dpx, dpy, p, sspp0, sppp0 are held fixed.
    Tensor conventions as pp_coef_fn, idirface int32 of cell2cell's shape."""
    for t in (cell2cell, ncface, idirface, iwet):
        if t.dtype != torch.int32 or not t.is_cuda or not t.is_contiguous():
            raise ValueError("cell2cell, ncface, idirface, iwet: contiguous int32 CUDA tensors")
    for t in (acoef_u, sp_u, area, hk, ds, dn, fintp, u, v, h, dpx, dpy, p, sspp0, sppp0):
        if t.dtype != torch.float64 or not t.is_cuda or not t.is_contiguous():
            raise ValueError("fields: contiguous float64 CUDA tensors")
    geo = (cell2cell, ncface, idirface, iwet, relax, area, h, dpx, dpy, p, ds, dn, fintp, sspp0, sppp0, ncells)
    return _PPRhsFn.apply(acoef_u, sp_u, hk, u, v, geo)
