"""ctypes loader for libcmsgpu.so (the in-tree CUDA library).

The library must exist: nothing here falls back to a CPU path.  Build it with
``python -m cms2d_b200.build`` (``__graft_entry__.build()`` does the same).
"""
from __future__ import annotations

import ctypes as C
import os
import re

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcmsgpu.so")
HEADER = os.path.join(os.path.dirname(_HERE), "include", "cmsgpu.h")

CMS_OK, CMS_NOT_CONVERGED, CMS_NONFINITE, CMS_DEVICE_ERROR, CMS_BAD_ARGUMENT, CMS_UNSUPPORTED = range(6)
STATUS_NAMES = {0: "ok", 1: "not converged", 2: "non-finite", 3: "device error", 4: "bad argument", 5: "unsupported"}
ORDER_MULTICOLOR, ORDER_NATURAL = 0, 1
PREC_FP64, PREC_FP32_REFINE, PREC_FP32 = 0, 1, 2


class SolverOpts(C.Structure):
    _fields_ = [("ordering", C.c_int), ("precision", C.c_int), ("norm", C.c_int), ("tol", C.c_double),
                ("max_iters", C.c_int), ("inner_tol", C.c_double), ("inner_max", C.c_int),
                ("max_refine", C.c_int), ("verify", C.c_int), ("multi_kernel", C.c_int),
                ("inner_relax", C.c_int), ("relaxsor", C.c_double), ("nswp0_vel", C.c_int),
                ("reduced_layout", C.c_int)]


class SolveInfo(C.Structure):
    _fields_ = [("status", C.c_int), ("iters", C.c_int), ("inner", C.c_int), ("refine_steps", C.c_int),
                ("relres", C.c_double), ("true_relres", C.c_double), ("rmom", C.c_double), ("ncolors", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class CmsError(RuntimeError):
    pass


_lib = None


def header_symbols() -> list[str]:
    """Function names declared in include/*.h."""
    inc = os.path.dirname(HEADER)
    names = []
    for f in sorted(os.listdir(inc)):
        if f.endswith(".h"):
            txt = open(os.path.join(inc, f)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names += re.findall(r"\b(cms_\w+)\s*\(", txt)
    return sorted(set(names))


def lib():
    """Loads libcmsgpu.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise CmsError(f"{LIB_PATH} is missing: build it with `python -m cms2d_b200.build`")
    L = C.CDLL(LIB_PATH)
    vp, ip, i = C.c_void_p, C.c_void_p, C.c_int
    d, f = C.c_double, C.c_float
    L.cms_solver_default_opts.argtypes = [C.POINTER(SolverOpts)]
    L.cms_solver_create.argtypes = [i, i, i, ip, ip, ip, C.POINTER(SolverOpts), C.POINTER(vp)]
    L.cms_solver_update_wet.argtypes = [vp, ip]
    L.cms_solver_set_opts.argtypes = [vp, C.POINTER(SolverOpts)]
    for name, real in (("d", d), ("f", f)):
        for dev in ("", "dev_"):
            fn = getattr(L, f"cms_solver_solve_{dev}{name}")
            fn.argtypes = [vp, vp, vp, vp, vp, vp, real, i, i, C.POINTER(SolveInfo)]
            fn = getattr(L, f"cms_solver_solve_{dev}n_{name}")
            fn.argtypes = [vp, i, vp, vp, vp, vp, vp, real, i, i, C.POINTER(SolveInfo)]
    L.cms_solver_ncolors.argtypes = [vp]
    L.cms_solver_device_bytes.argtypes = [vp]
    L.cms_solver_device_bytes.restype = C.c_size_t
    L.cms_solver_get_perm.argtypes = [vp, ip]
    L.cms_solver_launches.argtypes = [vp]
    L.cms_solver_launches.restype = C.c_longlong
    L.cms_solver_profile.argtypes = [vp, i]
    L.cms_solver_wait_selftest.argtypes = [vp, C.c_uint]
    L.cms_solver_refine_fallbacks.argtypes = [vp]
    L.cms_solver_refine_fallbacks.restype = C.c_longlong
    L.cms_solver_persist_wait_selftest.argtypes = [vp, C.c_uint, C.c_int]
    L.cms_solver_profile_read.argtypes = [vp, i, vp, vp, vp]
    L.cms_solver_set_tiles.argtypes = [vp, i]
    L.cms_solver_stream.argtypes = [vp]
    L.cms_solver_stream.restype = vp
    L.cms_solver_destroy.argtypes = [vp]
    L.cms_order_build.argtypes = [i, i, i, ip, ip, i, ip, ip, ip]
    L.cms_gpu_init.argtypes = [i, i, i, ip, ip, ip]
    L.cms_gpu_set_opts.argtypes = [C.POINTER(SolverOpts)]
    L.cms_gpu_update_wet.argtypes = [ip]
    L.cms_gpu_solve_d.argtypes = [i, vp, vp, vp, vp, vp, d, i, i, C.POINTER(d)]
    L.cms_gpu_solve_f.argtypes = [i, vp, vp, vp, vp, vp, f, i, i, C.POINTER(f)]
    L.cms_gpu_last_info.argtypes = [C.POINTER(SolveInfo)]
    L.cms_gpu_version.restype = C.c_char_p
    L.cms_gpu_last_error.restype = C.c_char_p
    _lib = L
    return L


def last_error() -> str:
    return lib().cms_gpu_last_error().decode()


def check(rc: int, what: str, allow=(CMS_OK,)) -> int:
    if rc not in allow:
        raise CmsError(f"{what}: {STATUS_NAMES.get(rc, rc)} ({last_error()})")
    return rc
