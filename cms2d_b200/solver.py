"""Host-side mirror of the reference's solver interface (solv_init / solve).

``Solver.solve(acoef, ss, sp, res, phi, n)`` keeps the argument meaning of
``subroutine solve(acoef,ss,sp,res,phi,n)`` (source/solvers/solvers.f90:205):
``acoef(nmaxfaces,ncellsD)`` in, ``ss`` and ``phi`` in/out, ``sp`` in, ``res``
out, ``n`` the variable index (1 pp, 2 u, 3 v, 4 sediment, 5 salinity/heat)
that selects ``relax(n)`` and ``nswp(n)`` as ``comvarbl`` does.  numpy arrays
go through the host-pointer C-ABI entry points (copies included); torch CUDA
tensors go through the device-pointer ones.  Every call runs on the GPU via
libcmsgpu.so: there is no CPU path.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib

# relax(n) defaults: source/flow/flow.F90:124-130 (pp 1.0, u 0.8, v 0.8, c 0.8, s 0.8)
RELAX_DEFAULT = {1: 1.0, 2: 0.8, 3: 0.8, 4: 0.8, 5: 0.8}
# nswp(n) defaults per solver: source/flow/flow.F90:752-821
NSWP_DEFAULT = {0: {1: 40, 2: 10, 3: 10, 4: 10, 5: 10}, 1: {1: 100, 2: 30, 3: 30, 4: 15, 5: 15},
                2: {1: 80, 2: 20, 3: 20, 4: 15, 5: 15}, 3: {1: 15, 2: 5, 3: 5, 4: 5, 5: 5},
                4: {1: 20, 2: 5, 3: 5, 4: 3, 5: 3}, 5: {1: 20, 2: 5, 3: 5, 4: 3, 5: 3},
                6: {1: 30, 2: 7, 3: 7, 4: 5, 5: 5}, 7: {1: 30, 2: 7, 3: 7, 4: 5, 5: 5},
                8: {1: 30, 2: 7, 3: 7, 4: 5, 5: 5}}
NSOLV_DEFAULT = 4  # GMRES, source/solvers/solvers.f90:8
# MATRIX_SOLVER card values (asolv, solvers.f90:9-17); ADI has no branch in solve()
SOLVER_NAMES = {"ADI": 0, "GAUSS-SEIDEL": 1, "GAUSS-SEIDEL-SOR": 2, "BICGSTAB": 3, "GMRES": 4, "HYBRID": 5,
                "SIP": 6, "ICCG": 7, "ICCGSTAB": 8}

_ORDER = {"multicolor": _lib.ORDER_MULTICOLOR, "natural": _lib.ORDER_NATURAL}
_PREC = {"fp64": _lib.PREC_FP64, "fp32_refine": _lib.PREC_FP32_REFINE, "fp32": _lib.PREC_FP32}


def _ptr(a):
    if isinstance(a, np.ndarray):
        return a.ctypes.data_as(C.c_void_p)
    return C.c_void_p(a.data_ptr())


def _is_device(a) -> bool:
    return not isinstance(a, np.ndarray) and getattr(a, "is_cuda", False)


def order_build(grid, ordering: str = "multicolor"):
    """Host-only ordering (no GPU needed): (perm, gstart, (KL, KU))."""
    L = _lib.lib()
    n = grid.ncells
    perm = np.zeros(n, np.int32)
    gstart = np.zeros(n + 1, np.int32)
    klku = np.zeros(2, np.int32)
    c2c = np.ascontiguousarray(grid.cell2cell, np.int32)
    ncf = np.ascontiguousarray(grid.ncface, np.int32)
    G = L.cms_order_build(n, grid.ncellsD, grid.nmaxfaces, _ptr(c2c), _ptr(ncf), _ORDER[ordering], _ptr(perm),
                          _ptr(gstart), _ptr(klku))
    if G <= 0:
        raise _lib.CmsError(f"cms_order_build: {_lib.last_error()}")
    return perm, gstart[: G + 1].copy(), (int(klku[0]), int(klku[1]))


class Solver:
    """solv_init (source/solvers/solvers.f90:93-202) bound to one grid.

    ordering:  "multicolor" (default; red/black on Cartesian grids) or
               "natural" (the reference order, level-scheduled sweeps).
    precision: "fp64" (drop-in), "fp32_refine" (FP32 solve inside FP64
               refinement; applies to float64 arrays) or "fp32".
    tol/norm:  stopping test; the reference uses 1e-3 on the L1 ratio
               (BiCGStab) or on the GMRES residual estimate.
    inner_relax: FP32 inner BiCGStab of refinement on a multicolour ordering:
               2 the reduced (Schur complement) system, 1 the two-phase
               factor, 0 the exact multicolour ILU(0) (True/False mean 1/0).
    inner_tol/inner_max: refinement's inner solves; 0 (default): each may use
               the solve's remaining iteration budget and is asked for
               0.5 tol / (outer residual so far) within [1e-6, 1e-3].
    reduced_layout: block/row layout and iteration form of the reduced inner
               solve (0 auto: 1024 threads x 2 rows, single reduction;
               cms_solver_opts.reduced_layout).
    """

    def __init__(self, grid, iwet=None, ordering: str = "multicolor", precision: str = "fp64", tol: float = 1e-3,
                 norm: int = 1, max_iters: int = 0, inner_tol: float = 0.0, inner_max: int = 0,
                 max_refine: int = 30, verify: bool = True, nsolv: int = NSOLV_DEFAULT,
                 multi_kernel: bool = False, inner_relax: int = 2, relaxsor: float = 1.8, nswp0_vel: int = 5,
                 reduced_layout: int = 0):
        L = _lib.lib()
        self.grid = grid
        self.nsolv = nsolv
        self.opts = _lib.SolverOpts()
        L.cms_solver_default_opts(C.byref(self.opts))
        self.opts.ordering = _ORDER[ordering]
        self.opts.precision = _PREC[precision]
        self.opts.tol = tol
        self.opts.norm = norm
        self.opts.max_iters = max_iters
        self.opts.inner_tol = inner_tol
        self.opts.inner_max = inner_max
        self.opts.max_refine = max_refine
        self.opts.verify = int(verify)
        self.opts.multi_kernel = int(multi_kernel)
        self.opts.inner_relax = int(inner_relax)
        self.opts.relaxsor = relaxsor
        self.opts.nswp0_vel = nswp0_vel
        self.opts.reduced_layout = reduced_layout
        self._c2c = np.ascontiguousarray(grid.cell2cell, np.int32)
        self._ncf = np.ascontiguousarray(grid.ncface, np.int32)
        self._iwet = np.ones(grid.ncellsD, np.int32) if iwet is None else np.ascontiguousarray(iwet, np.int32)
        h = C.c_void_p()
        rc = L.cms_solver_create(grid.ncells, grid.ncellsD, grid.nmaxfaces, _ptr(self._c2c), _ptr(self._ncf),
                                 _ptr(self._iwet), C.byref(self.opts), C.byref(h))
        _lib.check(rc, "cms_solver_create")
        self._h = h
        self.last_info = None

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().cms_solver_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- configuration --
    def set_options(self, **kw):
        for k, v in kw.items():
            if k == "precision":
                v = _PREC[v]
            if k == "ordering":
                raise ValueError("the ordering is fixed when the solver is created")
            setattr(self.opts, k, int(v) if isinstance(v, bool) else v)
        _lib.check(_lib.lib().cms_solver_set_opts(self._h, C.byref(self.opts)), "cms_solver_set_opts")

    def update_wet(self, iwet):
        self._iwet = np.ascontiguousarray(iwet, np.int32)
        _lib.check(_lib.lib().cms_solver_update_wet(self._h, _ptr(self._iwet)), "cms_solver_update_wet")

    @property
    def ncolors(self) -> int:
        return _lib.lib().cms_solver_ncolors(self._h)

    @property
    def device_bytes(self) -> int:
        return _lib.lib().cms_solver_device_bytes(self._h)

    @property
    def launches(self) -> int:
        return _lib.lib().cms_solver_launches(self._h)

    @property
    def stream_handle(self) -> int:
        return _lib.lib().cms_solver_stream(self._h) or 0

    PROFILE_CLASSES = ("prologue", "ilu0", "fwd_sweep", "bwd_sweep", "spmv", "vector", "resid64", "scalar", "flow",
                       "bicgstab_persistent", "reduced_build", "bicgstab_reduced")

    def profile(self, enable: bool = True):
        _lib.check(_lib.lib().cms_solver_profile(self._h, int(enable)), "cms_solver_profile")

    def profile_read(self, reset: bool = True) -> dict:
        k = len(self.PROFILE_CLASSES)
        ms = np.zeros(k); by = np.zeros(k); cnt = np.zeros(k, np.int64)
        _lib.check(_lib.lib().cms_solver_profile_read(self._h, int(reset), _ptr(ms), _ptr(by), _ptr(cnt)),
                   "cms_solver_profile_read")
        return {name: {"ms": float(ms[q]), "bytes": float(by[q]), "launches": int(cnt[q])}
                for q, name in enumerate(self.PROFILE_CLASSES)}

    def perm(self) -> np.ndarray:
        p = np.zeros(self.grid.ncells, np.int32)
        _lib.check(_lib.lib().cms_solver_get_perm(self._h, _ptr(p)), "cms_solver_get_perm")
        return p

    # -- solve(acoef,ss,sp,res,phi,n) --
    def solve(self, acoef, ss, sp, res, phi, n: int = 1, relax=None, nswp=None, nsolv=None, raise_on_error=True):
        """Updates ss, res, phi in place; returns the solve record (dict).

        The reference's `iconv` is 0 for a non-finite solution and 1 otherwise
        (solvers.f90:291-301); it is returned as info["iconv"].
        """
        nsolv = self.nsolv if nsolv is None else nsolv
        relax = RELAX_DEFAULT.get(n, 0.8) if relax is None else relax
        if nswp is None:
            nswp = NSWP_DEFAULT.get(nsolv, NSWP_DEFAULT[4]).get(n, 5)
        g = self.grid
        arrs = (acoef, ss, sp, res, phi)
        dev = _is_device(acoef)
        dt = acoef.dtype
        for a in arrs:
            if _is_device(a) != dev or a.dtype != dt:
                raise TypeError("acoef, ss, sp, res, phi must share dtype and device")
            if not (a.flags.c_contiguous if isinstance(a, np.ndarray) else a.is_contiguous()):
                raise ValueError("arrays must be contiguous")
        if tuple(acoef.shape) != (g.ncellsD, g.nmaxfaces):
            raise ValueError(f"acoef must be [ncellsD, nmaxfaces] = {(g.ncellsD, g.nmaxfaces)}")
        for a in arrs[1:]:
            if tuple(a.shape) != (g.ncellsD,):
                raise ValueError("ss, sp, res, phi must have ncellsD entries")
        is64 = str(dt) in ("float64", "torch.float64")
        if not is64 and str(dt) not in ("float32", "torch.float32"):
            raise TypeError("float32 or float64 arrays expected")
        L = _lib.lib()
        info = _lib.SolveInfo()
        if dev and hasattr(acoef, "device"):
            # the handle's own stream reads the tensors: finish the work that produced them
            import torch
            torch.cuda.current_stream(acoef.device).synchronize()
        fn = {(True, False): L.cms_solver_solve_n_d, (False, False): L.cms_solver_solve_n_f,
              (True, True): L.cms_solver_solve_dev_n_d, (False, True): L.cms_solver_solve_dev_n_f}[(is64, dev)]
        rc = fn(self._h, int(n), *[_ptr(a) for a in arrs], float(relax), int(nswp), int(nsolv), C.byref(info))
        if raise_on_error:
            _lib.check(rc, "solve", allow=(_lib.CMS_OK, _lib.CMS_NOT_CONVERGED, _lib.CMS_NONFINITE))
        out = info.as_dict()
        out["status"] = rc
        out["iconv"] = 0 if rc == _lib.CMS_NONFINITE else 1
        self.last_info = out
        return out
