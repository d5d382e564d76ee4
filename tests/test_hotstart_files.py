"""Hot-start files in the SMS ASCII dataset format (cms2d_b200.hotstart):
written as write_hotstart_sup writes them, read back as hot_read_dat reads
them, and used to restart a model (CPU oracle)."""
import numpy as np

from cms2d_b200 import cases, gridio, hotstart
from cms2d_b200 import grid as G
from oracle import oracle as O


def test_dataset_format(tmp_path):
    hotstart.write_hot_start(tmp_path / "HotStart", p=np.array([9.81, 19.62, np.nan]), eta=[1.0, 2.0, 3.0],
                             u=[0.1, -0.25, 0.0], v=[0.0, 1.5e-7, 2.0], iwet=[1, 1, 0], ncells=3, time_hours=6.5)
    lines = open(tmp_path / "HotStart_p.dat").read().splitlines()
    assert lines[:4] == ["DATASET", 'OBJTYPE "scat2d"', "BEGSCL", "OBJID 17255"]
    assert lines[4].split() == ["ND", "3"] and lines[6] == 'NAME "Water_Pressure"'
    assert lines[9].split() == ["TS", "0", "6.5000"]
    assert lines[10] == " 9.81000E+00" and lines[12].strip() == "-999." and lines[-1] == "ENDDS"
    vel = open(tmp_path / "HotStart_vel.dat").read().splitlines()
    assert vel[2:4] == ["BEGVEC", "VECTYPE 0"] and vel[12] == "-2.50000E-01  1.50000E-07"
    sup = open(tmp_path / "HotStart.sup").read().splitlines()
    assert sup[0] == "SUPER" and 'DATA    "HotStart_vel.dat"' in sup
    ds = hotstart.read_hot_start(tmp_path / "HotStart.sup")
    assert [d.name for d in ds] == ["Water_Pressure", "Water_Elevation", "Current_Velocity", "Wet"]
    assert ds[2].vector and np.allclose(ds[2].values[0][:, 1], [0.0, 1.5e-7, 2.0])
    assert ds[1].times == [6.5]


def test_restart_from_files_on_a_grid_with_land(tmp_path):
    lev = G.refinement_rectangles(10, 8, [(1, 3, 2, 7, 6)])
    act = lambda x, y, s: (x - 120.0) ** 2 + (y - 60.0) ** 2 > 25.0 ** 2  # noqa: E731
    gridio.write_tel(tmp_path / "g.tel", lev, 20.0, lambda x, y: 2.0 + 0.02 * y, active=act)
    gf = gridio.read_tel(tmp_path / "g.tel")
    case = cases.from_grid_file(gf, dt=300.0)
    n = case.grid.ncells
    o = O.FlowOracle(case)
    o.init()
    for _ in range(3):
        o.step()
    hotstart.write_hot_start(tmp_path / "HotStart", o.get("p"), o.get("eta"), o.get("u"), o.get("v"),
                             o.get("iwet"), n, time_hours=o.t / 3600.0)
    p, u, v, t = hotstart.hot_start_fields(hotstart.read_hot_start(tmp_path / "HotStart.sup"), gf)
    assert abs(t - o.t / 3600.0) < 1e-4
    # five significant digits in the files
    assert np.abs(p[:n] / 9.81 - o.get("eta")[:n]).max() <= 1e-5 * np.abs(o.get("eta")[:n]).max() + 1e-12
    h = O.FlowOracle(case)
    h.init_hot(p, u, v, t=o.t)
    for _ in range(2):
        assert o.step()["status"] == 0 and h.step()["status"] == 0
    assert np.abs(o.get("eta")[:n] - h.get("eta")[:n]).max() < 1e-4
