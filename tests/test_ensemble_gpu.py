"""Ensemble stepping (cms_ensemble_*): batched solves give each member the
results of its own flow step.

Same tile count per member as its own solver: identical arithmetic, results
agree to rounding (observed bit-identical).  A different split of the batched
launch changes the block partition of the dot products only: the solves stop
at the same 1e-8 relative residual, results agree within 1e-7 m / 1e-6.
"""
import numpy as np
import pytest

from cms2d_b200 import cases
from cms2d_b200.ensemble import EnsembleModel
from cms2d_b200.flow import FlowModel

pytestmark = pytest.mark.gpu

SET = dict(precision="fp32_refine", nsolv=3, tol=1e-8, norm=2, nswp_pp=400, nswp_uv=400)


def _basins():
    return [cases.tidal_basin(40, 30, seed=1, amp=0.5, manning=0.02),
            cases.tidal_basin(56, 22, seed=2, amp=0.8, manning=0.03, depth_off=7.0),
            cases.tidal_basin(30, 45, seed=3, amp=0.4, manning=0.025, depth_shore=3.0)]


def _solo(cs, steps):
    out = []
    for c in cs:
        m = FlowModel(c, **SET)
        m.init()
        for _ in range(steps):
            info = m.step()
            assert info["status"] == 0, info
        out.append({k: m.get(k)[: c.grid.ncells] for k in ("eta", "u", "v")})
        m.close()
    return out


def _compare(ens, solo, cs, eta_tol, vel_tol):
    for m, ref, c in zip(ens.members, solo, cs):
        n = c.grid.ncells
        assert np.abs(m.get("eta")[:n] - ref["eta"]).max() <= eta_tol
        vmax = np.hypot(ref["u"], ref["v"]).max()
        for k in ("u", "v"):
            assert np.abs(m.get(k)[:n] - ref[k]).max() <= vel_tol * vmax, k


def test_ensemble_matches_member_steps():
    cs = _basins()
    solo = _solo(cs, 2)
    e = EnsembleModel(cs, **{k: v for k, v in SET.items() if k != "precision"})
    assert e.batched
    e.init()
    for _ in range(2):
        infos = e.step()
        assert all(i["status"] == 0 for i in infos), infos
    assert e.launches > 0
    _compare(e, solo, cs, 1e-10, 1e-8)
    e.close()


def test_ensemble_uneven_split():
    cs = [cases.tidal_basin(220, 120, seed=4, amp=0.6), cases.tidal_basin(90, 70, seed=5, amp=0.9)]
    solo = _solo(cs, 2)
    e = EnsembleModel(cs, **{k: v for k, v in SET.items() if k != "precision"})
    e.set_tiles(5)  # 4 + 1 tiles: another dot-product partition than the members' own solvers
    tot, per = e.tiles()
    assert tot == per.sum() <= 5 and per.min() >= 1
    e.init()
    for _ in range(2):
        infos = e.step()
        assert all(i["status"] == 0 for i in infos), infos
    _compare(e, solo, cs, 1e-7, 1e-6)
    e.close()


def test_layout_autotuner_picks_a_candidate():
    cs = _basins()
    e = EnsembleModel(cs, **{k: v for k, v in SET.items() if k != "precision"})
    e.init()
    best = e.tune(candidates=[3, 12], steps=1)
    assert best in (3, 12)
    assert e.tiles()[0] <= best and set(e.tuning["candidates"]) == {3, 12}
    info = e.step()
    assert all(i["status"] == 0 for i in info)
    e.close()


def test_ensemble_wetting_and_drying():
    """Intertidal members (a falling and a rising tide, Cartesian and
    telescoping): each member's wet set and fields follow its own steps."""
    cs = [cases.tidal_flat(seed=1, t0_hours=1.0), cases.tidal_flat(50, 36, seed=2, t0_hours=7.0, refine=True)]
    steps = 4
    solo, wet = [], []
    for c in cs:
        m = FlowModel(c, **SET)
        m.init()
        for _ in range(steps):
            assert m.step()["status"] == 0
        solo.append({k: m.get(k)[: c.grid.ncells] for k in ("eta", "u", "v")})
        wet.append(m.get("iwet"))
        m.close()
    e = EnsembleModel(cs, **{k: v for k, v in SET.items() if k != "precision"})
    e.init()
    changed = 0
    for _ in range(steps):
        infos = e.step()
        assert all(i["status"] == 0 for i in infos), infos
        changed += sum(i["nchanged"] for i in infos)
    assert changed > 0
    for m, w in zip(e.members, wet):
        assert np.array_equal(m.get("iwet"), w)
    _compare(e, solo, cs, 1e-10, 1e-8)
    e.close()


def test_stage_graphs_match_direct_launches():
    """A flow model whose stage kernel sequences replay as CUDA graphs gives
    the same bits as direct launches, through wet/dry changes on an
    intertidal flat (each change makes the graphs be captured again)."""
    c = cases.tidal_flat(60, 40, seed=2, t0_hours=2.0)
    out = []
    for graphs in (False, True):
        m = FlowModel(c, precision="fp64", nsolv=3, tol=1e-8, norm=2, nswp_pp=400, nswp_uv=400)
        m.set_graphs(graphs)
        m.init()
        changed = 0
        for _ in range(6):
            info = m.step()
            assert info["status"] == 0, info
            changed += info["nchanged"]
        out.append((m.get("eta").copy(), m.get("u").copy(), m.get("v").copy(), m.graph_stats(), changed))
        m.close()
    (e0, u0, v0, s0, c0), (e1, u1, v1, s1, c1) = out
    assert s0 == (0, 0)
    assert c0 == c1 > 0
    replays, captures = s1
    assert replays > 0 and captures > 4, s1  # two stages, re-captured after wet-set changes
    np.testing.assert_array_equal(e0, e1)
    np.testing.assert_array_equal(u0, u1)
    np.testing.assert_array_equal(v0, v1)


def test_ensemble_replays_stage_graphs():
    cs = _basins()
    e = EnsembleModel(cs, **{k: v for k, v in SET.items() if k != "precision"})
    e.init()
    for _ in range(2):
        assert all(i["status"] == 0 for i in e.step())
    for m in e.members:
        replays, captures = m.graph_stats()
        assert replays > captures > 0
    e.close()
