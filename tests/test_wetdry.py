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
