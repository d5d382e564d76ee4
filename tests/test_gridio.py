"""Grid file readers and writers (read_tel / read_grid_cart + geo_cart).

* Telescoping files written from parent-level maps (with land, refinement
  interfaces and split sides next to land) read back to exactly the grid the
  generator builds with read_tel's rules.
* Cartesian files (resolution and coordinate blocks, land, rectilinear
  spacing) read back to the generator's Cartesian grid, numbering
  id = i + (j-1)*maxcol, dummies N, E, S, W per cell.
* The reference's own test grids (testing/tests_flow/*/*.tel), from the
  committed fixture: structural checks (every internal face has its back
  face, every dummy its back link, no isolated cells); where the reference
  tree is present ($CMS_REFERENCE_DIR), read in place and compared with the
  fixture.
"""
import glob
import os

import numpy as np
import pytest

from cms2d_b200 import grid as G
from cms2d_b200 import gridio
from tests import reference_cases as RC

REF_TEL = sorted(glob.glob(os.path.join(RC.REF_DIR, "testing/tests_flow/*/*.tel"))) if RC.REF_DIR else []


def _same_grid(a, b, xy_tol=1e-12):
    assert (a.ncells, a.ncellsD, a.nmaxfaces) == (b.ncells, b.ncellsD, b.nmaxfaces)
    for k in ("cell2cell", "ncface", "idirface"):
        np.testing.assert_array_equal(getattr(a, k), getattr(b, k), err_msg=k)
    for k in ("x", "y", "dx", "dy"):
        np.testing.assert_allclose(getattr(a, k), getattr(b, k), rtol=0, atol=xy_tol * 1e3, err_msg=k)


def _levels():
    lev2 = G.refinement_rectangles(14, 11, [(1, 2, 2, 10, 8), (2, 4, 3, 8, 6)])
    return [
        ("cartesian", np.zeros((9, 13), dtype=np.int64), None),
        ("two-level", G.refinement_rectangles(12, 10, [(1, 3, 2, 9, 7)]), None),
        ("three-level", lev2, None),
        ("land", lev2, lambda x, y, s: (x - 140.0) ** 2 + (y - 110.0) ** 2 > 45.0 ** 2),
        ("land-strip", G.refinement_rectangles(12, 10, [(1, 3, 2, 9, 7)]), lambda x, y, s: np.abs(y - 100.0) > 12.0),
    ]


@pytest.mark.parametrize("name,lev,active", _levels(), ids=[c[0] for c in _levels()])
def test_tel_roundtrip(tmp_path, name, lev, active):
    dx0 = 20.0
    depth = lambda x, y: 2.0 + 0.01 * x + 0.003 * y  # noqa: E731
    p = tmp_path / f"{name}.tel"
    gridio.write_tel(p, lev, dx0, depth, active=active, angle=12.5, xorigin=1000.0, yorigin=-50.0)
    gf = gridio.read_tel(p)
    ref = G.telescoping_grid(lev, dx0, active=active, nmaxfaces=6)
    _same_grid(gf.grid, ref)
    n = ref.ncells
    np.testing.assert_allclose(gf.zb[:n], -(2.0 + 0.01 * ref.x[:n] + 0.003 * ref.y[:n]), rtol=1e-14)
    # dummies take the bed of the cell they hang off
    for d in range(n, ref.ncellsD):
        c = ref.cell2cell[d][ref.cell2cell[d] > 0][0] - 1
        assert gf.zb[d] == gf.zb[c]
    assert (gf.angle, gf.xorigin, gf.yorigin) == (12.5, 1000.0, -50.0)


def test_tel_rows_may_wrap_and_carry_extra_items(tmp_path):
    lev = np.zeros((3, 4), dtype=np.int64)
    p = tmp_path / "a.tel"
    gridio.write_tel(p, lev, 10.0, lambda x, y: 1.0 + 0 * x)
    lines = open(p).read().splitlines()
    out = lines[:2]
    for i, ln in enumerate(lines[2:]):
        t = ln.split()
        if i % 2:  # wrap the row over two records
            out += [" ".join(t[:6]), " ".join(t[6:])]
        else:  # trailing items after the 14th are ignored
            out.append(ln + " 0 7")
    q = tmp_path / "b.tel"
    q.write_text("\n".join(out) + "\n")
    _same_grid(gridio.read_tel(q).grid, gridio.read_tel(p).grid)


def test_tel_isolated_cell_rejected(tmp_path):
    lev = np.zeros((5, 5), dtype=np.int64)
    # one wet cell surrounded by land
    act = lambda x, y, s: ((np.abs(x - 50.0) < 1) & (np.abs(y - 50.0) < 1)) | (x < 20.0)  # noqa: E731
    p = tmp_path / "iso.tel"
    gridio.write_tel(p, lev, 20.0, lambda x, y: 1.0 + 0 * x, active=act)
    with pytest.raises(ValueError, match="isolated"):
        gridio.read_tel(p)


@pytest.mark.parametrize("coords", [False, True])
def test_cart_roundtrip_uniform_with_land(tmp_path, coords):
    nx, ny, dx = 17, 11, 25.0
    jj, ii = np.mgrid[0:ny, 0:nx]
    active = ~((ii - 8) ** 2 + (jj - 5) ** 2 < 6)  # a round island
    depth = 1.0 + 0.1 * ii + 0.05 * jj
    p = tmp_path / "g.cart"
    gridio.write_cart(p, np.full(nx, dx), np.full(ny, dx), depth, active=active, angle=30.0, coords=coords)
    gf = gridio.read_cart(p)
    ref = G.cartesian_grid(nx, ny, dx, active=lambda x, y, s: active[(y // dx).astype(int), (x // dx).astype(int)])
    _same_grid(gf.grid, ref, xy_tol=1e-12)
    n = ref.ncells
    np.testing.assert_allclose(gf.zb[:n], -depth[active], rtol=1e-14)
    assert np.array_equal(gf.mapid, (ii + 1 + jj * nx)[active])


def test_cart_rectilinear(tmp_path):
    dxs = np.array([10.0, 10.0, 15.0, 22.5, 30.0, 30.0])
    dys = np.array([5.0, 8.0, 8.0, 12.0])
    depth = np.full((4, 6), 3.0)
    p = tmp_path / "r.cart"
    gridio.write_cart(p, dxs, dys, depth)
    g = gridio.read_cart(p).grid
    ref = G.cartesian_grid(6, 4, 1.0)
    for k in ("cell2cell", "ncface", "idirface"):
        np.testing.assert_array_equal(getattr(g, k), getattr(ref, k))
    n = g.ncells
    xe, ye = np.cumsum(dxs), np.cumsum(dys)
    np.testing.assert_allclose(g.x[:n].reshape(4, 6), np.broadcast_to(xe - 0.5 * dxs, (4, 6)))
    np.testing.assert_allclose(g.y[:n].reshape(4, 6), np.broadcast_to((ye - 0.5 * dys)[:, None], (4, 6)))
    np.testing.assert_allclose(g.dx[:n].reshape(4, 6), np.broadcast_to(dxs, (4, 6)))
    # a dummy east of the last column is as wide as that column
    c = int(g.cell2cell[5, 1]) - 1
    assert c >= n and g.dx[c] == 30.0 and g.x[c] == g.x[5] + 30.0


def test_cart_without_activity_block_follows_the_last_depth(tmp_path):
    """read_grid_cart sets the whole activity array inside its per-cell loop:
    without an activity block the last cell's depth decides for every cell."""
    depth = np.full((3, 4), 2.0)
    depth[0, 0] = -999.0
    for last, expect in ((2.0, 12), (-999.0, 0)):
        depth[-1, -1] = last
        p = tmp_path / "n.cart"
        gridio.write_cart(p, np.full(4, 5.0), np.full(3, 5.0), depth)
        txt = open(p).read()
        i = txt.index("GRID_ACTIVITY_BEGIN")
        p.write_text(txt[:i])
        if expect == 0:
            with pytest.raises(ValueError, match="no active cells"):
                gridio.read_cart(p)
        else:
            assert gridio.read_cart(p).grid.ncells == expect


@pytest.mark.skipif(not REF_TEL, reason="reference tree not present (set CMS_REFERENCE_DIR)")
@pytest.mark.parametrize("path", REF_TEL, ids=[os.path.basename(p) for p in REF_TEL])
def test_reference_test_grids_match_fixture(path):
    gf = gridio.read_tel(path)
    with open(path) as f:
        f.readline()
        nfull = int(float(f.readline().split()[3]))
    assert 0 < gf.grid.ncells <= nfull and gf.grid.ncellsD > gf.grid.ncells
    name = os.path.basename(os.path.dirname(path))
    fx, _, _ = RC.load(name)
    _same_grid(gf.grid, fx.grid, xy_tol=0.0)
    np.testing.assert_array_equal(gf.zb, fx.zb)


@pytest.mark.parametrize("name", RC.names())
def test_reference_test_grids(name):
    g = RC.load(name)[0].grid
    n = g.ncells
    assert 0 < n and g.ncellsD > n
    back = {1: 3, 2: 4, 3: 1, 4: 2}
    for i in range(n):
        for k in range(int(g.ncface[i])):
            j = int(g.cell2cell[i, k]) - 1
            d = int(g.idirface[i, k])
            assert 1 <= d <= 4 and j >= 0
            if j < n:  # internal: the neighbour has a face back with the opposite direction
                kk = [q for q in range(int(g.ncface[j])) if int(g.cell2cell[j, q]) - 1 == i]
                assert len(kk) == 1 and int(g.idirface[j, kk[0]]) == back[d]
            else:  # dummy: its back link on the opposite face
                assert int(g.cell2cell[j, back[d] - 1]) - 1 == i and int(g.ncface[j]) == 4


def test_case_from_grid_file_steps(tmp_path):
    """A telescoping file read back and run: the oracle's flow steps finish and
    follow the tide, identical to the same case built from the level map."""
    from cms2d_b200 import cases
    from oracle import oracle as O
    lev = G.refinement_rectangles(10, 8, [(1, 3, 2, 7, 6)])
    depth = lambda x, y: 2.0 + 0.02 * y  # noqa: E731
    p = tmp_path / "basin.tel"
    gridio.write_tel(p, lev, 20.0, depth)
    c = cases.from_grid_file(gridio.read_tel(p), dt=300.0)
    g2 = G.telescoping_grid(lev, 20.0, nmaxfaces=6)
    zb2 = cases._fill_dummies(g2, -(2.0 + 0.02 * g2.y[: g2.ncells]))
    c2 = cases.Case("ref", g2, zb2, np.full(g2.ncells, 0.025), *cases._north_string(g2), [(0.5, cases.M2_HOURS)],
                    300.0, 10)
    runs = []
    for case in (c, c2):
        f = O.FlowOracle(case)
        f.init()
        for _ in range(3):
            assert f.step()["status"] == 0
        runs.append(f.get("eta")[: g2.ncells])
    np.testing.assert_allclose(runs[0], runs[1], rtol=0, atol=1e-12)
    assert abs(runs[0].mean() - c.wse(900.0)) < 0.02
