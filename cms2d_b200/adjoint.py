"""Differentiable solve(): the adjoint of the reference's solve() boundary.

``solve_fn(solver, acoef, ss, sp, phi, relax=1.0, nswp=..., tol=...)`` runs the
forward solve on the GPU (``cms_solver_solve_dev_d``) and returns x (phi after
the solve).  Its backward pass solves A^T lam = dL/dx on the GPU
(``cms_solver_adjoint_dev_d``: ILU(0)-BiCGStab on the transposed system) and
returns dL/dacoef, dL/dss and dL/dsp in the solve() layout.  FP64 CUDA
tensors, natural order, acoef [ncellsD, nmaxfaces].
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
