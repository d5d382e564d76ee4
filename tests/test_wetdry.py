"""Wetting and drying rules without a GPU: the library's host rules
(cms_wetdry_rules, a worklist to the fixed point) against the oracle's literal
restatement of flow_wetdry(0) (sweeps in cell order until nothing changes,
then flow_pond's alternating sweeps)."""
import numpy as np
import pytest

from cms2d_b200 import cases
from cms2d_b200 import flow as FL
from oracle import oracle as O


def _oracle_iwet(case, eta, ponding=False, narrow=False):
    f = O.FlowOracle(case)
    f.set_wetdry(ponding=ponding, narrowchannels=narrow)
    f.init(eta)
    return f.get("iwet").astype(np.int32)


def _depth_wet(case, eta, hdry=0.05):
    return (eta * 9.81 * (1.0 / 9.81) - case.zb >= hdry).astype(np.int32)


@pytest.mark.parametrize("refine", [False, True])
def test_rules_match_oracle_over_the_tide(refine):
    c = cases.tidal_flat(refine=refine)
    n = c.grid.ncells
    fired_narrow = fired_pond = 0
    for level in np.linspace(-0.95, 1.0, 14):
        eta = np.full(c.grid.ncellsD, level)
        ours = FL.wetdry_rules(c, eta)
        ref = _oracle_iwet(c, eta)
        assert np.array_equal(ours, ref), (level, np.nonzero(ours != ref)[0][:10])
        assert ours[:n].sum() > 0
        depth = _depth_wet(c, eta)[:n]
        fired_narrow += int((depth.astype(bool) & ~ours[:n].astype(bool)).sum())
        pond = FL.wetdry_rules(c, eta, ponding=True)
        fired_pond += int(pond[:n].sum() - ours[:n].sum())
        assert np.array_equal(pond, _oracle_iwet(c, eta, ponding=True))
    # the case exercises both the narrow-channel rules and flow_pond
    assert fired_narrow > 0 and fired_pond > 0


@pytest.mark.parametrize("seed", [1, 2, 3])
@pytest.mark.parametrize("refine", [False, True])
def test_rules_match_oracle_on_rough_beds(seed, refine):
    """Beds of random relief around the water level: many narrow channels,
    ponds and cascades of removals, where a wrong order would show."""
    c = cases.tidal_flat(nx=40, ny=32, seed=seed, refine=refine)
    rng = np.random.default_rng(seed)
    n = c.grid.ncells
    zb = c.zb.copy()
    zb[:n] = rng.uniform(-0.35, 0.25, n)
    c.zb = zb
    eta = np.zeros(c.grid.ncellsD)
    for narrow in (False, True):
        ours = FL.wetdry_rules(c, eta, narrowchannels=narrow)
        ref = _oracle_iwet(c, eta, narrow=narrow)
        assert np.array_equal(ours, ref), (narrow, np.nonzero(ours != ref)[0][:10])
    depth = _depth_wet(c, eta)[:n]
    assert (depth.sum() - ours[:n].sum()) > 10


def test_closed_dummies_dry_string_dummies_follow_depth():
    c = cases.tidal_flat()
    g = c.grid
    n = g.ncells
    eta = np.full(g.ncellsD, 0.5)
    w = FL.wetdry_rules(c, eta)
    th_d = g.cell2cell[c.th_cells - 1, c.th_faces - 1] - 1
    walls = np.setdiff1d(np.arange(n, g.ncellsD), th_d)
    assert np.all(w[walls] == 0)
    assert np.array_equal(w[th_d], _depth_wet(c, eta)[th_d])


def _dump(case, code, path):
    g = case.grid
    with open(path, "wb") as f:
        np.array([g.ncells, g.ncellsD, g.nmaxfaces], np.int32).tofile(f)
        g.ncface.astype(np.int32).tofile(f)
        (g.cell2cell.astype(np.int32) - 1).tofile(f)
        g.idirface.astype(np.int32).tofile(f)
        code.astype(np.uint8).tofile(f)
        np.array([case.th_cells.size], np.int32).tofile(f)
        d = g.cell2cell[case.th_cells - 1, case.th_faces - 1] - 1
        np.stack([case.th_cells - 1, d], 1).astype(np.int32).tofile(f)


@pytest.mark.parametrize("refine", [False, True])
def test_incremental_narrow_update_equals_full(tmp_path, refine):
    """The step's incremental update of the narrow-channel set against the full
    recomputation, over 300 random batches of depth-class changes per mode."""
    import os
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = str(tmp_path / "wdinc")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(root, "cms2d_b200", "csrc"), "-I",
                    os.path.join(root, "include"), "-o", exe, os.path.join(root, "tests", "wetdry_incremental_check.cpp"),
                    os.path.join(root, "cms2d_b200", "csrc", "cms_flow_wetdry.cpp")], check=True)
    c = cases.tidal_flat(60, 40, seed=3, refine=refine)
    n = c.grid.ncells
    rng = np.random.default_rng(1)
    zb = c.zb.copy()
    zb[:n] = rng.uniform(-0.35, 0.25, n)
    h = 0.0 - zb
    code = (h >= 0.05) * 1 | (h < 0.25) * 2 | (h < 0.1) * 4
    path = str(tmp_path / "grid.bin")
    _dump(c, code, path)
    for narrow in ("0", "1"):
        out = subprocess.run([exe, path, narrow], capture_output=True, text=True)
        assert out.returncode == 0, (narrow, out.stdout, out.stderr)
        assert int(out.stdout.split()[3]) > 1000  # the batches did change the set
