"""Host-side mirror of the implicit flow step (flow_imp) on libcmsgpu.

``FlowModel(case)`` builds the device state for a grid (the reference's
geo_init_cart + solv_init + der_init), ``init()`` does the cold start of
prestart, and ``step()`` runs one ``flow_imp`` time step followed by
``flow_update`` on the GPU.  The caller keeps the time loop and the boundary
water levels (``bnd_eval``), as the reference's host does.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from . import solver as _solver

_ORDER = {"multicolor": _lib.ORDER_MULTICOLOR, "natural": _lib.ORDER_NATURAL}
_PREC = {"fp64": _lib.PREC_FP64, "fp32_refine": _lib.PREC_FP32_REFINE}

CELL = {"p": 0, "h": 1, "u": 2, "v": 3, "eta": 4, "vis": 5, "cfrict": 6, "dpx": 7, "dpy": 8, "iwet": 9}
FACE = {"flux": 100, "visk": 101, "hk": 102, "acoef": 103, "fintp": 104, "zbk": 105}


class FlowOpts(C.Structure):
    _fields_ = [("nsolv", C.c_int), ("ordering", C.c_int), ("precision", C.c_int), ("norm", C.c_int),
                ("tol", C.c_double), ("nswp_pp", C.c_int), ("nswp_uv", C.c_int), ("maxit", C.c_int),
                ("skewcor", C.c_int), ("inner_tol", C.c_double), ("inner_max", C.c_int),
                ("multi_kernel", C.c_int), ("hdry", C.c_double), ("ponding", C.c_int), ("narrowchannels", C.c_int),
                ("relaxsor", C.c_double), ("ndsch", C.c_int), ("reduced_layout", C.c_int)]


class FlowInfo(C.Structure):
    _fields_ = [("status", C.c_int), ("niter", C.c_int), ("iconv", C.c_int), ("rmom_p", C.c_double),
                ("rmom_u", C.c_double), ("rmom_v", C.c_double), ("krylov_iters", C.c_longlong),
                ("nwet", C.c_int), ("nchanged", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def _bind(L):
    if getattr(L, "_flow_bound", False):
        return
    vp, i, d = C.c_void_p, C.c_int, C.c_double
    L.cms_flow_default_opts.argtypes = [C.POINTER(FlowOpts)]
    L.cms_flow_create.argtypes = [i, i, i] + [vp] * 9 + [i, vp, vp, C.POINTER(FlowOpts), C.POINTER(vp)]
    L.cms_flow_init.argtypes = [vp, vp]
    L.cms_flow_init_hot.argtypes = [vp, vp, vp, vp, vp]
    L.cms_flow_step.argtypes = [vp, d, vp, C.POINTER(FlowInfo)]
    L.cms_flow_get.argtypes = [vp, i, vp]
    L.cms_flow_launches.argtypes = [vp]
    L.cms_flow_launches.restype = C.c_longlong
    L.cms_flow_device_bytes.argtypes = [vp]
    L.cms_flow_device_bytes.restype = C.c_size_t
    L.cms_flow_njoint.argtypes = [vp]
    L.cms_flow_set_graphs.argtypes = [vp, i]
    L.cms_flow_set_tide.argtypes = [vp, i] + [vp] * 7 + [d, d]
    L.cms_flow_set_time.argtypes = [vp, d]
    L.cms_flow_graph_stats.argtypes = [vp, vp, vp]
    L.cms_flow_solver.argtypes = [vp]
    L.cms_flow_solver.restype = vp
    L.cms_flow_last_solves.argtypes = [vp, C.POINTER(_lib.SolveInfo * 3)]
    L.cms_flow_destroy.argtypes = [vp]
    L._flow_bound = True


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class FlowModel:
    """One implicit flow model on the GPU for a case (cms2d_b200.cases.Case)."""

    def __init__(self, case, nsolv: int = 4, ordering: str = "multicolor", precision: str = "fp64",
                 tol: float = 1e-3, norm: int = 1, nswp_pp: int | None = None, nswp_uv: int | None = None,
                 maxit: int = 0, skewcor: bool = True, inner_tol: float = 0.0, inner_max: int = 0,
                 multi_kernel: bool = False, hdry: float = 0.05, ponding: bool = False,
                 narrowchannels: bool = False, relaxsor: float = 1.8, ndsch: int = 4, reduced_layout: int = 0):
        L = _lib.lib()
        _bind(L)
        self.case = case
        g = case.grid
        self.g = g
        o = FlowOpts()
        L.cms_flow_default_opts(C.byref(o))
        o.nsolv = nsolv
        o.ordering = _ORDER[ordering]
        o.precision = _PREC[precision]
        o.tol = tol
        o.norm = norm
        # nswp defaults per solver (flow.F90:752-821)
        o.nswp_pp = nswp_pp if nswp_pp is not None else _solver.NSWP_DEFAULT[nsolv][1]
        o.nswp_uv = nswp_uv if nswp_uv is not None else _solver.NSWP_DEFAULT[nsolv][2]
        o.maxit = maxit
        o.skewcor = int(skewcor)
        o.inner_tol = inner_tol
        o.inner_max = inner_max
        o.multi_kernel = int(multi_kernel)
        o.hdry = hdry
        o.ponding = int(ponding)
        o.narrowchannels = int(narrowchannels)
        o.relaxsor = relaxsor
        o.ndsch = ndsch
        o.reduced_layout = reduced_layout
        self.opts = o
        self._keep = [np.ascontiguousarray(a) for a in (
            g.cell2cell.astype(np.int32), g.ncface.astype(np.int32), g.idirface.astype(np.int32),
            g.x.astype(np.float64), g.y.astype(np.float64), g.dx.astype(np.float64), g.dy.astype(np.float64),
            case.zb.astype(np.float64), case.coefman.astype(np.float64), case.th_cells.astype(np.int32),
            case.th_faces.astype(np.int32))]
        k = self._keep
        h = C.c_void_p()
        rc = L.cms_flow_create(g.ncells, g.ncellsD, g.nmaxfaces, _p(k[0]), _p(k[1]), _p(k[2]), _p(k[3]), _p(k[4]),
                               _p(k[5]), _p(k[6]), _p(k[7]), _p(k[8]), int(case.th_cells.size), _p(k[9]),
                               _p(k[10]), C.byref(o), C.byref(h))
        _lib.check(rc, "cms_flow_create")
        self._h = h
        self.t = 0.0
        self.last = None

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().cms_flow_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def init(self, eta0=None):
        if eta0 is None:
            eta0 = np.full(self.g.ncellsD, self.case.wse(0.0))
        eta0 = np.ascontiguousarray(eta0, np.float64)
        _lib.check(_lib.lib().cms_flow_init(self._h, _p(eta0)), "cms_flow_init")
        self.t = 0.0

    def init_hot(self, p, u, v, t=0.0, flux=None):
        """Hot start from the water pressure and velocities of all ncellsD cells
        (natural order) and, when the hot-start file holds them, the face fluxes
        [ncellsD, nmaxfaces]; t is the simulation time the state belongs to."""
        arrs = [np.ascontiguousarray(a, np.float64) for a in (p, u, v)]
        for a in arrs:
            if a.shape != (self.g.ncellsD,):
                raise ValueError("p, u, v must have ncellsD entries")
        fl = None
        if flux is not None:
            fl = np.ascontiguousarray(flux, np.float64)
            if fl.shape != (self.g.ncellsD, self.g.nmaxfaces):
                raise ValueError("flux must be [ncellsD, nmaxfaces]")
        _lib.check(_lib.lib().cms_flow_init_hot(self._h, *[_p(a) for a in arrs], None if fl is None else _p(fl)),
                   "cms_flow_init_hot")
        self.t = float(t)
        _lib.lib().cms_flow_set_time(self._h, self.t)

    def set_tide(self):
        """Moves the case's water-level string onto the device (bnd_eval's
        harmonic form, cms_flow_set_tide): each constituent (amp, period h)
        becomes speed 2 pi / period and phase -speed * t0, the case's
        per-entry offsets the level variations; steps then pass no levels."""
        amp = np.array([a for a, _ in self.case.tide], np.float64)
        speed = np.array([2.0 * np.pi / T for _, T in self.case.tide], np.float64)
        phase = -speed * (self.case.t0 / 3600.0)
        var = None if self.case.th_offset is None else np.ascontiguousarray(self.case.th_offset, np.float64)
        self._tide = (amp, speed, phase, var)
        _lib.check(_lib.lib().cms_flow_set_tide(self._h, amp.size, _p(amp), _p(speed), _p(phase), None, None, None,
                                                None if var is None else _p(var), 0.0, 0.0), "cms_flow_set_tide")
        self.device_tide = True

    def step(self, dt=None, wsebnd=None):
        dt = self.case.dt if dt is None else dt
        if wsebnd is None and not getattr(self, "device_tide", False):
            wsebnd = self.case.wsebnd(self.t + dt)
        wp = None
        if wsebnd is not None:
            wsebnd = np.ascontiguousarray(wsebnd, np.float64)
            wp = _p(wsebnd)
        info = FlowInfo()
        rc = _lib.lib().cms_flow_step(self._h, float(dt), wp, C.byref(info))
        _lib.check(rc, "cms_flow_step", allow=(_lib.CMS_OK, _lib.CMS_NONFINITE, _lib.CMS_UNSUPPORTED))
        self.t += dt
        self.last = info.as_dict()
        return self.last

    def set_graphs(self, on: bool = True):
        """Replay the stage kernel sequences as CUDA graphs (cms_flow_set_graphs)."""
        _lib.check(_lib.lib().cms_flow_set_graphs(self._h, int(on)), "cms_flow_set_graphs")

    def graph_stats(self):
        """(graph replays, graph captures) so far."""
        r, c = C.c_longlong(), C.c_longlong()
        _lib.lib().cms_flow_graph_stats(self._h, C.byref(r), C.byref(c))
        return r.value, c.value

    def get(self, name):
        g = self.g
        if name in CELL:
            out = np.zeros(g.ncellsD)
            which = CELL[name]
        else:
            out = np.zeros((g.ncellsD, g.nmaxfaces))
            which = FACE[name]
        _lib.check(_lib.lib().cms_flow_get(self._h, which, _p(out)), "cms_flow_get")
        return out

    def last_solves(self):
        """Solve records (u, v, pp) of the last outer iteration of the last step."""
        arr = (_lib.SolveInfo * 3)()
        _lib.check(_lib.lib().cms_flow_last_solves(self._h, C.byref(arr)), "cms_flow_last_solves")
        return [a.as_dict() for a in arr]

    @property
    def launches(self) -> int:
        return _lib.lib().cms_flow_launches(self._h)

    @property
    def device_bytes(self) -> int:
        return _lib.lib().cms_flow_device_bytes(self._h)

    @property
    def njoint(self) -> int:
        return _lib.lib().cms_flow_njoint(self._h)

    def wetdry_stats(self) -> dict:
        """Wet/dry updates so far and their host time (ms): read-back, rules, application."""
        L = _lib.lib()
        L.cms_flow_wetdry_stats.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        up = C.c_longlong()
        ms = np.zeros(3)
        _lib.check(L.cms_flow_wetdry_stats(self._h, C.byref(up), _p(ms)), "cms_flow_wetdry_stats")
        return {"updates": int(up.value), "readback_ms": float(ms[0]), "rules_ms": float(ms[1]),
                "apply_ms": float(ms[2])}

    @property
    def solver_handle(self):
        return _lib.lib().cms_flow_solver(self._h)

    def perm(self) -> np.ndarray:
        """Unknown ordering of the solves: perm[r] = natural 0-based cell of row r."""
        p = np.zeros(self.g.ncells, np.int32)
        _lib.check(_lib.lib().cms_solver_get_perm(self.solver_handle, _p(p)), "cms_solver_get_perm")
        return p


def wetdry_rules(case, eta, hdry: float = 0.05, ponding: bool = False, narrowchannels: bool = False) -> np.ndarray:
    """Wet flags (ncellsD) that flow_wetdry(0) gives the case's grid for the
    water level eta (ncellsD values); host computation, no device needed."""
    L = _lib.lib()
    if not getattr(L, "_wdr_bound", False):
        L.cms_wetdry_rules.argtypes = [C.c_int] * 3 + [C.c_void_p] * 5 + [C.c_int, C.c_void_p, C.c_void_p, C.c_double,
                                                                          C.c_int, C.c_int, C.c_void_p]
        L._wdr_bound = True
    g = case.grid
    arrs = [np.ascontiguousarray(a) for a in (g.cell2cell.astype(np.int32), g.ncface.astype(np.int32),
                                               g.idirface.astype(np.int32), case.zb.astype(np.float64),
                                               np.asarray(eta, np.float64), case.th_cells.astype(np.int32),
                                               case.th_faces.astype(np.int32))]
    out = np.zeros(g.ncellsD, np.int32)
    rc = L.cms_wetdry_rules(g.ncells, g.ncellsD, g.nmaxfaces, _p(arrs[0]), _p(arrs[1]), _p(arrs[2]), _p(arrs[3]),
                            _p(arrs[4]), int(case.th_cells.size), _p(arrs[5]), _p(arrs[6]), float(hdry),
                            int(ponding), int(narrowchannels), _p(out))
    _lib.check(rc, "cms_wetdry_rules")
    return out
