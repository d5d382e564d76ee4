"""ctypes binding of the CPU oracle (oracle/liboracle.so) -- test infrastructure.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module; the product (cms2d_b200) never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

PC_ILUTP = 0
PC_ILU0 = 1


def build(force: bool = False) -> str:
    so = os.path.join(_HERE, "liboracle.so")
    srcs = [os.path.join(_HERE, f) for f in ("cms_oracle.cpp", "cms_flow_oracle.cpp", "Makefile")]
    if force or not os.path.exists(so) or any(os.path.getmtime(s) > os.path.getmtime(so) for s in srcs):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return so


def lib():
    global _LIB
    if _LIB is None:
        so = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(so):
            build()
        L = C.CDLL(so)
        P = C.c_void_p
        i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
        f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
        f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
        L.orc_create.restype = P
        L.orc_create.argtypes = [C.c_int, C.c_int, C.c_int, i32p, i32p, i32p, C.c_int]
        L.orc_destroy.argtypes = [P]
        L.orc_nnz.argtypes = [P]
        L.orc_nnz.restype = C.c_int
        L.orc_pattern.argtypes = [P, i32p, i32p]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_set_threads.restype = C.c_int
        ip = C.POINTER(C.c_int)
        dp = C.POINTER(C.c_double)
        L.orc_solve_d.argtypes = [P, f64p, f64p, f64p, f64p, f64p, C.c_double, C.c_int, C.c_int, C.c_int, C.c_double,
                                  C.c_int, C.c_double, C.c_double, dp, ip, ip, dp, C.c_int]
        L.orc_solve_d.restype = C.c_int
        fp = C.POINTER(C.c_float)
        L.orc_solve_f.argtypes = [P, f32p, f32p, f32p, f32p, f32p, C.c_float, C.c_int, C.c_int, C.c_int, C.c_float,
                                  C.c_int, C.c_float, C.c_float, fp, ip, ip, dp, C.c_int]
        L.orc_solve_f.restype = C.c_int
        L.orc_solve_n_d.argtypes = [P, C.c_int, f64p, f64p, f64p, f64p, f64p, C.c_double, C.c_int, C.c_int,
                                    C.c_double, C.c_int, C.c_int, C.c_double, dp, ip, ip, dp, C.c_int]
        L.orc_solve_n_d.restype = C.c_int
        L.orc_solve_n_f.argtypes = [P, C.c_int, f32p, f32p, f32p, f32p, f32p, C.c_float, C.c_int, C.c_int,
                                    C.c_float, C.c_int, C.c_int, C.c_float, fp, ip, ip, dp, C.c_int]
        L.orc_solve_n_f.restype = C.c_int
        L.orc_lusol_d.argtypes = [P, f64p, f64p]
        _LIB = L
    return _LIB


def set_threads(n: int) -> int:
    return lib().orc_set_threads(int(n))


class OracleSolver:
    """CPU restatement of solv_init + solve (source/solvers/solvers.f90:93-304)."""

    def __init__(self, grid, iwet=None, fix_last_cell: bool = True):
        self.g = grid
        L = lib()
        iw = np.ones(grid.ncellsD, np.int32) if iwet is None else np.ascontiguousarray(iwet, np.int32)
        self._h = L.orc_create(grid.ncells, grid.ncellsD, grid.nmaxfaces,
                               np.ascontiguousarray(grid.cell2cell, np.int32),
                               np.ascontiguousarray(grid.ncface, np.int32), iw, int(fix_last_cell))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().orc_destroy(h)
            self._h = None

    def pattern(self):
        L = lib()
        nnz = L.orc_nnz(self._h)
        ia = np.zeros(self.g.ncells + 1, np.int32)
        ja = np.zeros(nnz, np.int32)
        L.orc_pattern(self._h, ia, ja)
        return ia, ja

    def solve(self, acoef, ss, sp, res, phi, relax=1.0, nswp=15, nsolv=3, precond=PC_ILU0, tol=1e-3, lfil=None,
              droptol=1e-3, permtol=0.5, norm=1, n=None, relaxsor=1.8, nswp0_vel=5):
        """Arguments mirror solve(acoef,ss,sp,res,phi,n): ss, res and phi are updated in place.

        n (the variable index), relaxsor and nswp0_vel select the branches of
        nsolv = 1, 2, 5, 6, 7, 8 (solvers.f90:242-289); nsolv 3 and 4 ignore them.
        Returns dict(status, rmom, iters, inner, relres).
        """
        L = lib()
        if n is not None or nsolv not in (3, 4):
            dt = acoef.dtype
            rm = (C.c_double if dt == np.float64 else C.c_float)()
            it = C.c_int(); inner = C.c_int(); rr = C.c_double()
            fn = L.orc_solve_n_d if dt == np.float64 else L.orc_solve_n_f
            for a in (acoef, ss, sp, res, phi):
                assert a.dtype == dt and a.flags.c_contiguous
            st = fn(self._h, int(n or 0), acoef, ss, sp, res, phi, relax, int(nswp), int(nsolv), relaxsor,
                    int(nswp0_vel), int(precond), tol, C.byref(rm), C.byref(it), C.byref(inner), C.byref(rr),
                    int(norm))
            return dict(status=st, rmom=rm.value, iters=it.value, inner=inner.value, relres=rr.value)
        if lfil is None:
            lfil = 8 if nsolv == 4 else 35  # solvers.f90:195-199
        dt = acoef.dtype
        rm = (C.c_double if dt == np.float64 else C.c_float)()
        it = C.c_int(); inner = C.c_int(); rr = C.c_double()
        fn = L.orc_solve_d if dt == np.float64 else L.orc_solve_f
        for a in (acoef, ss, sp, res, phi):
            assert a.dtype == dt and a.flags.c_contiguous
        st = fn(self._h, acoef, ss, sp, res, phi, relax, int(nswp), int(nsolv), int(precond), tol, int(lfil), droptol,
                permtol, C.byref(rm), C.byref(it), C.byref(inner), C.byref(rr), int(norm))
        return dict(status=st, rmom=rm.value, iters=it.value, inner=inner.value, relres=rr.value)

    def lusol(self, y):
        x = np.zeros_like(y)
        lib().orc_lusol_d(self._h, np.ascontiguousarray(y, np.float64), x)
        return x


class FlowOracle:
    """CPU restatement of one implicit flow step (flow_imp, flow_imp.F90:29-312)."""

    CELL = {"p": 0, "h": 1, "u": 2, "v": 3, "eta": 4, "vis": 5, "cfrict": 6, "dpx": 7, "dpy": 8, "iwet": 200,
            "icorner": 201, "areap": 202}
    FACE = {"flux": 100, "visk": 101, "hk": 102, "acoef": 103, "fintp": 104, "zbk": 105, "dsxy": 106}

    def __init__(self, case, skewcor: bool = True):
        L = lib()
        if not hasattr(L, "_flow_bound"):
            P = C.c_void_p
            L.orcf_create.restype = P
            i32 = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
            f64 = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
            L.orcf_create.argtypes = [C.c_int, C.c_int, C.c_int, i32, i32, i32, f64, f64, f64, f64, f64, f64, C.c_int,
                                      i32, i32, C.c_int]
            L.orcf_destroy.argtypes = [P]
            L.orcf_set_solver.argtypes = [P, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int]
            L.orcf_init.argtypes = [P, f64]
            L.orcf_init_hot.argtypes = [P, f64, f64, f64, C.c_void_p]
            L.orcf_step.argtypes = [P, C.c_double, f64, C.c_int, C.POINTER(C.c_int), f64]
            L.orcf_step.restype = C.c_int
            L.orcf_get.argtypes = [P, C.c_int, f64]
            L.orcf_get.restype = C.c_longlong
            L.orcf_solve_iters.argtypes = [P]
            L.orcf_solve_iters.restype = C.c_longlong
            L.orcf_njoint.argtypes = [P]
            L.orcf_set_order.argtypes = [P, i32]
            L.orcf_last_nlist.argtypes = [P]
            L.orcf_set_wetdry.argtypes = [P, C.c_int, C.c_int]
            L.orcf_set_hdry.argtypes = [P, C.c_double]
            L.orcf_set_scheme.argtypes = [P, C.c_int]
            L.orcf_capture.argtypes = [P, C.c_int]
            L.orcf_captured.argtypes = [P, f64, f64, f64, f64]
            L.orcf_captured.restype = C.c_int
            L._flow_bound = True
        g = case.grid
        self.case = case
        self.g = g
        self._h = L.orcf_create(g.ncells, g.ncellsD, g.nmaxfaces, np.ascontiguousarray(g.cell2cell, np.int32),
                                np.ascontiguousarray(g.ncface, np.int32), np.ascontiguousarray(g.idirface, np.int32),
                                np.ascontiguousarray(g.x), np.ascontiguousarray(g.y), np.ascontiguousarray(g.dx),
                                np.ascontiguousarray(g.dy), np.ascontiguousarray(case.zb, np.float64),
                                np.ascontiguousarray(case.coefman, np.float64), int(case.th_cells.size),
                                np.ascontiguousarray(case.th_cells, np.int32),
                                np.ascontiguousarray(case.th_faces, np.int32), int(skewcor))
        self.t = 0.0
        self.steps = 0

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().orcf_destroy(h)
            self._h = None

    def set_solver(self, nsolv=4, precond=PC_ILU0, tol=1e-3, nswp_pp=20, nswp_uv=5, norm=1):
        lib().orcf_set_solver(self._h, nsolv, precond, tol, nswp_pp, nswp_uv, norm)

    def set_order(self, perm):
        """Solve in another unknown order (perm[r] = natural 0-based cell of solver row r)."""
        lib().orcf_set_order(self._h, np.ascontiguousarray(perm, np.int32))

    def set_wetdry(self, ponding=False, narrowchannels=False, hdry=None):
        """The ponding and narrow-channel switches of the wetting and drying
        rules, and the drying depth (hmin = hdry, the one- and two-cell depths
        5 and 2 hdry)."""
        lib().orcf_set_wetdry(self._h, int(ponding), int(narrowchannels))
        if hdry is not None:
            lib().orcf_set_hdry(self._h, float(hdry))

    def set_scheme(self, ndsch):
        """ADVECTION_SCHEME: 0 none, 1 upwind, 2 hybrid, 3 power law, 4 exponential."""
        lib().orcf_set_scheme(self._h, int(ndsch))

    def init(self, eta0=None):
        if eta0 is None:
            eta0 = np.full(self.g.ncellsD, self.case.wse(0.0))
        lib().orcf_init(self._h, np.ascontiguousarray(eta0, np.float64))

    def init_hot(self, p, u, v, t=0.0, flux=None):
        """Hot start from the water pressure and velocities of all ncellsD cells
        (and the face fluxes [ncellsD, nmaxfaces] when the file holds them)."""
        fl = None if flux is None else np.ascontiguousarray(flux, np.float64)
        lib().orcf_init_hot(self._h, *[np.ascontiguousarray(a, np.float64) for a in (p, u, v)],
                            None if fl is None else fl.ctypes.data)
        self.t = t

    def step(self, maxit=None, dt=None):
        dt = self.case.dt if dt is None else dt
        if maxit is None:
            maxit = 20 + self.g.ncells // 10000  # flow.F90:784,792
        wse = np.ascontiguousarray(self.case.wsebnd(self.t + dt), np.float64)
        ni = C.c_int()
        rm = np.zeros(3)
        st = lib().orcf_step(self._h, dt, wse, int(maxit), C.byref(ni), rm)
        self.t += dt
        self.steps += 1
        return dict(status=st, niter=ni.value, rmom=rm.copy())

    def get(self, name):
        g = self.g
        if name in self.CELL:
            out = np.zeros(g.ncellsD)
            lib().orcf_get(self._h, self.CELL[name], out)
            return out
        out = np.zeros(g.ncellsD * g.nmaxfaces)
        lib().orcf_get(self._h, self.FACE[name], out)
        return out.reshape(g.ncellsD, g.nmaxfaces)

    def capture(self, var):
        """Arms the capture of the next solve() of variable var (1 pp, 2 u, 3 v)."""
        lib().orcf_capture(self._h, int(var))

    def captured(self):
        """(acoef [ncellsD, nmaxfaces], ss, sp, phi) of the captured system, as
        solve() received it, natural order; None before the capture."""
        g = self.g
        a = np.zeros(g.ncellsD * g.nmaxfaces)
        ss, sp, phi = np.zeros(g.ncellsD), np.zeros(g.ncellsD), np.zeros(g.ncellsD)
        if not lib().orcf_captured(self._h, a, ss, sp, phi):
            return None
        return a.reshape(g.ncellsD, g.nmaxfaces), ss, sp, phi

    @property
    def solve_iters(self):
        return lib().orcf_solve_iters(self._h)

    @property
    def last_nlist(self):
        """Cells whose gradient weights der_update recomputed at the last step."""
        return lib().orcf_last_nlist(self._h)

    @property
    def njoint(self):
        return lib().orcf_njoint(self._h)
