"""Reader of the reference's card files (*.cmcards) for the cards the implicit
flow step reads.

A card line is a name followed by values, a value optionally followed by its
unit in quotes (``HYDRO_TIMESTEP  60 'sec'``); quoted strings are file names;
``!`` starts a comment.  The reference reads cards in one loop, each module
claiming its own (flow_cards, source/flow/flow.F90:171-589; the grid file
cards, source/geospatial/geospatial.F90:170-200), so a card given twice takes
its last value.  flow_settings maps the cards this library serves onto the
arguments of cms2d_b200.flow.FlowModel:

  MATRIX_SOLVER / SOLVER_TYPE            nsolv (solvers.f90:9-17 names)
  PRESSURE_ITERATIONS (and aliases)      nswp_pp
  VELOCITY_ITERATIONS (and aliases)      nswp_uv
  HYDRO_MAX_ITERATIONS (and aliases)     maxit
  SUCCESSIVE_OVER_RELAXATION_CONSTANT    relaxsor
  DRYING_DEPTH                           hdry
  DRYING_DEPTH_ONE_CELL / _TWO_CELL      read, no effect on the step (below)
  WATER_PONDING                          ponding
  NARROW_CHANNELS (and aliases)          narrowchannels
  SKEWNESS_CORRECTION                    skewcor
  ADVECTION_SCHEME                       ndsch (NONE .. EXPONENTIAL, definitions.F90:166-171)
  HYDRO_TIMESTEP                         the time step (seconds)
  TELESCOPING / GRID_FILE                the grid file

SOLUTION_SCHEME other than IMPLICIT is rejected: only the implicit step is
served.

The one- and two-cell drying depths (DRYING_DEPTH_ONE_CELL /
ONE_CELL_DRYING_DEPTH, DRYING_DEPTH_TWO_CELL / TWO_CELL_DRYING_DEPTH,
flow.F90:248-252) are accepted and validated, but they never change the wet set: with narrow
channels off the reference resets them to 5 and 2 times DRYING_DEPTH
(flow.F90:686-689) before the rules that read them (flow.F90:1340-1424), and
with narrow channels on only the isolated-cell rule runs (flow.F90:1324-1338),
which reads neither.  The flow model therefore takes hdry alone.
"""
from __future__ import annotations

import os
import shlex

from .solver import SOLVER_NAMES

_TIME = {"sec": 1.0, "s": 1.0, "second": 1.0, "seconds": 1.0, "min": 60.0, "minutes": 60.0, "hr": 3600.0,
         "hrs": 3600.0, "hour": 3600.0, "hours": 3600.0, "day": 86400.0, "days": 86400.0}
_LENGTH = {"m": 1.0, "cm": 0.01, "mm": 0.001, "ft": 0.3048}
# the first-order entries of the reference's scheme list (advsc, definitions.F90:166-171)
ADVECTION_SCHEMES = {"NONE": 0, "UPWIND": 1, "HYBRID": 2, "POWERLAW": 3, "EXPONENTIAL": 4}
_TRUE = {"ON", "TRUE", "T", "YES", "1", ".TRUE."}
_FALSE = {"OFF", "FALSE", "F", "NO", "0", ".FALSE."}


class Cards(dict):
    """Card name -> list of value tokens (quotes removed) of its last
    occurrence; .line[name] is the line number of that occurrence, so that of
    several aliases of one setting the one given last in the file wins, as in
    the reference's single reading loop."""

    def __init__(self):
        super().__init__()
        self.line = {}


def read_cards(path) -> Cards:
    """Card name -> list of value tokens (quotes removed), last occurrence."""
    cards = Cards()
    with open(path) as f:
        for lineno, ln in enumerate(f, 1):
            ln = ln.split("!", 1)[0].strip()
            if not ln:
                continue
            try:
                toks = shlex.split(ln, posix=True)
            except ValueError:
                toks = ln.split()
            name = toks[0].upper()
            cards[name] = toks[1:]
            cards.line[name] = lineno
    return cards


def _scalar(vals, table):
    v = float(vals[0])
    if len(vals) > 1 and vals[1].lower() in table:
        v *= table[vals[1].lower()]
    return v


def _boolean(vals):
    t = vals[0].upper()
    if t in _TRUE:
        return True
    if t in _FALSE:
        return False
    raise ValueError(f"not a boolean card value: {vals[0]}")


def _first(cards, *names):
    """Values of the alias of one setting given last in the file (plain dicts
    without line numbers: the first alias present)."""
    lines = getattr(cards, "line", {})
    best, best_line = None, -1
    for n in names:
        if n in cards and cards[n]:
            ln = lines.get(n, 0)
            if best is None or ln > best_line:
                best, best_line = cards[n], ln
    return best


def flow_settings(cards: dict, base_dir: str = "."):
    """(FlowModel keyword arguments, time step in seconds or None, grid file
    path or None) from the cards of read_cards."""
    kw = {}
    v = _first(cards, "SOLUTION_SCHEME")
    if v and v[0].upper() != "IMPLICIT":
        raise ValueError(f"SOLUTION_SCHEME {v[0]}: only the implicit flow step is served")
    v = _first(cards, "MATRIX_SOLVER", "SOLVER_TYPE")
    if v:
        name = v[0].upper()
        if name not in SOLVER_NAMES:
            raise ValueError(f"unknown MATRIX_SOLVER {v[0]}")
        kw["nsolv"] = SOLVER_NAMES[name]
    v = _first(cards, "PRESSURE_ITERATIONS", "PRESSURE_ITER", "PRES_ITER", "PRESS_ITER")
    if v:
        kw["nswp_pp"] = int(float(v[0]))
    v = _first(cards, "VELOCITY_ITERATIONS", "VELOCITY_ITER", "VEL_ITER")
    if v:
        kw["nswp_uv"] = int(float(v[0]))
    v = _first(cards, "HYDRO_MAX_ITERATIONS", "HYDRO_MAX_ITER", "SOLVER_MAX_ITER")
    if v:
        kw["maxit"] = int(float(v[0]))
    v = _first(cards, "SUCCESSIVE_OVER_RELAXATION_CONSTANT", "SOR_CONSTANT")
    if v:
        kw["relaxsor"] = float(v[0])
    v = _first(cards, "DRYING_DEPTH")
    if v:
        kw["hdry"] = _scalar(v, _LENGTH)
    for key, names in (("hdry1", ("DRYING_DEPTH_ONE_CELL", "ONE_CELL_DRYING_DEPTH")),
                       ("hdry2", ("DRYING_DEPTH_TWO_CELL", "TWO_CELL_DRYING_DEPTH"))):
        v = _first(cards, *names)
        if v:
            _scalar(v, _LENGTH)  # validated; without effect on the wet set (module docstring)
    v = _first(cards, "WATER_PONDING")
    if v:
        kw["ponding"] = _boolean(v)
    v = _first(cards, "ONE_CELL_WIDE_CHANNELS", "ONE-CELL-WIDE_CHANNELS", "NARROW_CHANNELS")
    if v:
        kw["narrowchannels"] = _boolean(v)
    v = _first(cards, "ADVECTION_SCHEME")
    if v:
        name = v[0].upper()
        if name not in ADVECTION_SCHEMES:
            raise ValueError(f"ADVECTION_SCHEME {v[0]}: only NONE, UPWIND, HYBRID, POWERLAW and EXPONENTIAL "
                             f"are served")
        kw["ndsch"] = ADVECTION_SCHEMES[name]
    v = _first(cards, "SKEWNESS_CORRECTION")
    if v:
        kw["skewcor"] = _boolean(v)
    dt = None
    v = _first(cards, "HYDRO_TIMESTEP")
    if v:
        dt = _scalar(v, _TIME)
    grid = None
    v = _first(cards, "TELESCOPING", "TELESCOPING_FILE", "GRID_FILE")
    if v:
        grid = v[0] if os.path.isabs(v[0]) else os.path.join(base_dir, v[0])
    return kw, dt, grid
