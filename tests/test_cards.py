"""Card files (*.cmcards): the cards the implicit flow step serves, read as
flow_cards reads them, and the reference's own test cases (grid and cards,
from the committed fixture; read in place and compared with it where the
reference tree is present, $CMS_REFERENCE_DIR) run through the oracle."""
import glob
import os

import pytest

from cms2d_b200 import cards, gridio
from cms2d_b200 import solver as S
from oracle import oracle as O
from tests import reference_cases as RC

REF_CARDS = sorted(glob.glob(os.path.join(RC.REF_DIR, "testing/tests_flow/*/*.cmcards"))) if RC.REF_DIR else []


def test_flow_settings(tmp_path):
    p = tmp_path / "a.cmcards"
    p.write_text("""! comment line
CMS_VERSION        5.3
TELESCOPING        "grid one.tel"
SOLUTION_SCHEME    IMPLICIT
MATRIX_SOLVER      GAUSS-SEIDEL-SOR   ! trailing comment
SOR_CONSTANT       1.6
PRESSURE_ITERATIONS 60
VEL_ITER           12
HYDRO_MAX_ITER     25
DRYING_DEPTH       5 'cm'
WATER_PONDING      ON
NARROW_CHANNELS    OFF
SKEWNESS_CORRECTION OFF
HYDRO_TIMESTEP     10 'min'
MATRIX_SOLVER      HYBRID
""")
    kw, dt, grid = cards.flow_settings(cards.read_cards(p), str(tmp_path))
    assert kw == dict(nsolv=5, nswp_pp=60, nswp_uv=12, maxit=25, relaxsor=1.6, hdry=0.05, ponding=True,
                      narrowchannels=False, skewcor=False)
    assert dt == 600.0 and grid == os.path.join(str(tmp_path), "grid one.tel")
    p.write_text("SOLUTION_SCHEME EXPLICIT\n")
    with pytest.raises(ValueError, match="implicit"):
        cards.flow_settings(cards.read_cards(p))


def test_card_aliases_last_in_file_wins(tmp_path):
    p = tmp_path / "b.cmcards"
    p.write_text("SOLVER_TYPE GMRES\nMATRIX_SOLVER BICGSTAB\nPRES_ITER 9\nPRESSURE_ITERATIONS 7\n"
                 "DRYING_DEPTH_ONE_CELL 0.3\nTWO_CELL_DRYING_DEPTH 0.2\n")
    kw, _, _ = cards.flow_settings(cards.read_cards(p))
    assert kw["nsolv"] == S.SOLVER_NAMES["BICGSTAB"] and kw["nswp_pp"] == 7
    p.write_text("MATRIX_SOLVER BICGSTAB\nPRESSURE_ITERATIONS 7\nSOLVER_TYPE GMRES\nPRES_ITER 9\n")
    kw, _, _ = cards.flow_settings(cards.read_cards(p))
    assert kw["nsolv"] == S.SOLVER_NAMES["GMRES"] and kw["nswp_pp"] == 9


@pytest.mark.skipif(not REF_CARDS, reason="reference tree not present (set CMS_REFERENCE_DIR)")
@pytest.mark.parametrize("path", REF_CARDS, ids=[os.path.basename(p) for p in REF_CARDS])
def test_reference_cards_match_fixture(path):
    kw, dt, grid = cards.flow_settings(cards.read_cards(path), os.path.dirname(path))
    assert kw["nsolv"] in S.SOLVER_NAMES.values() and 0 < kw["hdry"] < 1 and dt > 0
    assert gridio.read_tel(grid).grid.ncells > 0
    _, kw2, dt2 = RC.load(os.path.basename(os.path.dirname(path)))
    assert kw2 == kw and dt2 == dt


@pytest.mark.parametrize("name", RC.names())
def test_reference_test_case_runs_from_its_cards(name):
    case, kw = RC.case(name)
    assert kw["nsolv"] == S.SOLVER_NAMES["GMRES"] and kw["skewcor"] is True
    assert case.dt == 60.0
    d = S.NSWP_DEFAULT[kw["nsolv"]]
    f = O.FlowOracle(case)
    f.set_solver(nsolv=kw["nsolv"], precond=O.PC_ILU0, tol=1e-3, nswp_pp=d[1], nswp_uv=d[2])
    f.set_wetdry(ponding=kw.get("ponding", False), narrowchannels=kw.get("narrowchannels", False),
                 hdry=kw["hdry"])
    f.init()
    for _ in range(3):
        assert f.step()["status"] == 0
