"""Ensembles of independent flow models stepped together on one GPU.

``EnsembleModel(cases)`` builds one FlowModel per case (FP32 + FP64
refinement, BiCGStab + ILU(0) by default) and a ``cms_ensemble`` over them:
every time step advances all members, each of the three Krylov solves of an
outer iteration running for all members in one batched persistent launch.

``tune()`` is the layout autotuner: it times the candidate block counts of
the batched launch over warm-up steps (seconds per Krylov iteration of the
ensemble) and keeps the fastest.
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import _lib
from .flow import FlowInfo, FlowModel, _bind as _bind_flow


def _bind(L):
    if getattr(L, "_ens_bound", False):
        return
    _bind_flow(L)
    vp, i, d = C.c_void_p, C.c_int, C.c_double
    L.cms_ensemble_create.argtypes = [i, C.POINTER(vp), C.POINTER(vp)]
    L.cms_ensemble_set_tiles.argtypes = [vp, i]
    L.cms_ensemble_tiles.argtypes = [vp, vp]
    L.cms_ensemble_capacity.argtypes = [vp]
    L.cms_ensemble_batched.argtypes = [vp]
    L.cms_ensemble_step.argtypes = [vp, d, C.POINTER(vp), vp]
    L.cms_ensemble_launches.argtypes = [vp]
    L.cms_ensemble_launches.restype = C.c_longlong
    L.cms_ensemble_destroy.argtypes = [vp]
    L._ens_bound = True


class EnsembleModel:
    """Independent flow models (one per case) stepped together."""

    def __init__(self, cases, precision: str = "fp32_refine", nsolv: int = 3, tol: float = 1e-6, norm: int = 2,
                 nswp_pp: int = 200, nswp_uv: int = 200, inner_tol: float = 0.0, inner_max: int = 0, **kw):
        L = _lib.lib()
        _bind(L)
        self.cases = list(cases)
        self.members = [FlowModel(c, nsolv=nsolv, precision=precision, tol=tol, norm=norm, nswp_pp=nswp_pp,
                                  nswp_uv=nswp_uv, inner_tol=inner_tol, inner_max=inner_max, **kw)
                        for c in self.cases]
        arr = (C.c_void_p * len(self.members))(*[m._h.value for m in self.members])
        h = C.c_void_p()
        _lib.check(L.cms_ensemble_create(len(self.members), arr, C.byref(h)), "cms_ensemble_create")
        self._h = h
        self.t = 0.0
        self.last = None

    @property
    def ncells(self) -> int:
        return sum(c.grid.ncells for c in self.cases)

    @property
    def batched(self) -> bool:
        return bool(_lib.lib().cms_ensemble_batched(self._h))

    @property
    def capacity(self) -> int:
        return _lib.lib().cms_ensemble_capacity(self._h)

    @property
    def launches(self) -> int:
        """Batched solver launches issued so far."""
        return _lib.lib().cms_ensemble_launches(self._h)

    def tiles(self):
        per = np.zeros(len(self.members), np.int32)
        tot = _lib.lib().cms_ensemble_tiles(self._h, per.ctypes.data_as(C.c_void_p))
        return tot, per

    def set_tiles(self, total: int):
        _lib.check(_lib.lib().cms_ensemble_set_tiles(self._h, int(total)), "cms_ensemble_set_tiles")

    def init(self):
        for m in self.members:
            m.init()
        self.t = 0.0

    def step(self, dt=None):
        dts = [c.dt for c in self.cases] if dt is None else [dt] * len(self.cases)
        if len(set(dts)) != 1:
            raise ValueError("ensemble members step with one dt")
        dt = dts[0]
        wse = [np.ascontiguousarray(c.wsebnd(self.t + dt), np.float64) for c in self.cases]
        ptrs = (C.c_void_p * len(wse))(*[w.ctypes.data for w in wse])
        infos = (FlowInfo * len(self.members))()
        rc = _lib.lib().cms_ensemble_step(self._h, float(dt), ptrs, infos)
        _lib.check(rc, "cms_ensemble_step", allow=(_lib.CMS_OK, _lib.CMS_NONFINITE, _lib.CMS_UNSUPPORTED))
        self.t += dt
        for m in self.members:
            m.t = self.t
        self.last = [x.as_dict() for x in infos]
        return self.last

    def tune(self, candidates=None, steps: int = 1, sync=None):
        """Layout autotuner: runs `steps` ensemble steps with each candidate
        block count and keeps the one with the least time per Krylov
        iteration.  The steps advance the simulation (use it as warm-up)."""
        if not self.batched:
            return None
        cap = self.capacity
        if candidates is None:
            candidates = sorted({max(len(self.members), int(cap * f)) for f in (0.25, 0.5, 0.75, 1.0)})
        results = {}
        for cand in candidates:
            self.set_tiles(cand)
            t = 0.0
            iters = 0
            for _ in range(steps):
                if sync:
                    sync()
                t0 = time.perf_counter()
                info = self.step()
                if sync:
                    sync()
                t += time.perf_counter() - t0
                iters += sum(i["krylov_iters"] for i in info)
            results[cand] = t / max(iters, 1)
        best = min(results, key=results.get)
        self.set_tiles(best)
        self.tuning = {"candidates": {int(k): round(v * 1e6, 3) for k, v in results.items()},
                       "unit": "us per Krylov iteration of the ensemble", "best": int(best)}
        return best

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().cms_ensemble_destroy(self._h)
            self._h = None
        for m in getattr(self, "members", []):
            m.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
