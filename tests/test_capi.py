"""C-ABI checks that need no GPU: the library loads and exports what include/*.h declares."""
import ctypes as C
import subprocess

import numpy as np

from cms2d_b200 import _lib
from cms2d_b200 import grid as G


def test_library_exports_every_header_symbol():
    names = _lib.header_symbols()
    assert len(names) >= 20
    L = _lib.lib()
    for name in names:
        assert hasattr(L, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True, check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    missing = [n for n in names if n not in exported]
    assert not missing, missing


def test_version_and_defaults():
    L = _lib.lib()
    assert b"sm_100a" in L.cms_gpu_version()
    o = _lib.SolverOpts()
    L.cms_solver_default_opts(C.byref(o))
    assert o.ordering == 0 and o.precision == 0 and o.norm == 1 and abs(o.tol - 1e-3) < 1e-15


def test_bad_arguments_rejected_before_device_use():
    L = _lib.lib()
    g = G.cartesian_grid(4, 3)
    c2c = np.ascontiguousarray(g.cell2cell, np.int32)
    ncf = np.ascontiguousarray(g.ncface, np.int32)
    h = C.c_void_p()
    # nmaxfaces out of range
    rc = L.cms_solver_create(g.ncells, g.ncellsD, 9, c2c.ctypes.data, ncf.ctypes.data, None, None, C.byref(h))
    assert rc == _lib.CMS_BAD_ARGUMENT
    # neighbour index out of range
    bad = c2c.copy(); bad[0, 0] = g.ncellsD + 5
    rc = L.cms_solver_create(g.ncells, g.ncellsD, g.nmaxfaces, bad.ctypes.data, ncf.ctypes.data, None, None, C.byref(h))
    assert rc == _lib.CMS_BAD_ARGUMENT
    assert "out of range" in _lib.last_error()
    # the global API without init
    d = C.c_double()
    z = np.zeros(4)
    assert L.cms_gpu_solve_d(1, z.ctypes.data, z.ctypes.data, z.ctypes.data, z.ctypes.data, z.ctypes.data, 1.0, 1, 3,
                             C.byref(d)) == _lib.CMS_BAD_ARGUMENT


def test_order_build_host_only():
    from cms2d_b200.solver import order_build
    g = G.cartesian_grid(8, 6)
    perm, gstart, (kl, ku) = order_build(g, "multicolor")
    assert len(gstart) == 3 and gstart[-1] == g.ncells
    # red cells (i+j even) first
    i = perm % 8; j = perm // 8
    assert np.all(((i + j) % 2)[: gstart[1]] == 0)


def test_flow_entry_points_marshal_and_reject_bad_grids():
    """The flow binding's argument lists match the C-ABI (checked without a GPU)."""
    from cms2d_b200 import flow as F
    L = _lib.lib()
    F._bind(L)
    o = F.FlowOpts()
    L.cms_flow_default_opts(C.byref(o))
    assert o.nsolv == 4 and o.nswp_pp == 20 and o.nswp_uv == 5 and o.skewcor == 1
    z = np.zeros(16, np.int32)
    zd = np.zeros(16)
    h = C.c_void_p()
    p = lambda a: a.ctypes.data_as(C.c_void_p)
    rc = L.cms_flow_create(0, 0, 4, p(z), p(z), p(z), p(zd), p(zd), p(zd), p(zd), p(zd), p(zd), 0, None, None,
                           C.byref(o), C.byref(h))
    assert rc == _lib.CMS_BAD_ARGUMENT
    info = F.FlowInfo()
    assert L.cms_flow_step(None, 1.0, None, C.byref(info)) == _lib.CMS_BAD_ARGUMENT


def test_ensemble_entry_points_reject_bad_arguments():
    """cms_ensemble_* argument checks run before any device work."""
    from cms2d_b200 import ensemble as E
    L = _lib.lib()
    E._bind(L)
    h = C.c_void_p()
    assert L.cms_ensemble_create(0, None, C.byref(h)) == _lib.CMS_BAD_ARGUMENT
    arr = (C.c_void_p * 2)(None, None)
    assert L.cms_ensemble_create(2, arr, C.byref(h)) == _lib.CMS_BAD_ARGUMENT
    assert L.cms_ensemble_step(None, 1.0, None, None) == _lib.CMS_BAD_ARGUMENT
    assert L.cms_ensemble_set_tiles(None, 4) == _lib.CMS_BAD_ARGUMENT
    assert L.cms_ensemble_batched(None) == 0
