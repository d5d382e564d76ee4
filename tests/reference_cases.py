"""The reference's three flow test cases (L05, L08, L10) from the committed
fixture tests/golden/reference_test_cases.npz (made by
tests/golden/make_reference_cases.py from their .tel and .cmcards files).

REF_DIR: the reference tree, from $CMS_REFERENCE_DIR (tests that read the
reference's files in place skip when it is unset or missing)."""
from __future__ import annotations

import json
import os

import numpy as np

from cms2d_b200 import cases, gridio

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "golden", "reference_test_cases.npz")
REF_DIR = os.environ.get("CMS_REFERENCE_DIR", "")
if REF_DIR and not os.path.isdir(REF_DIR):
    REF_DIR = ""


def names():
    with np.load(FIXTURE) as z:
        return [str(s) for s in z["cases"]]


def load(name):
    """(GridFile, flow settings dict, time step s) of one test case."""
    with np.load(FIXTURE) as z:
        rows = z[f"{name}/rows"]
        angle, x0, y0 = (float(v) for v in z[f"{name}/origin"])
        st = json.loads(str(z[f"{name}/settings"]))
    return gridio.tel_grid(rows, angle, x0, y0, name), st["flow"], st["dt"]


def case(name, amp=0.02):
    """The test case's grid with a north water-level string (M2 of amplitude
    amp) and uniform Manning n: the cases' own strings and roughness fields
    are in HDF5 files, which nothing here reads."""
    gf, kw, dt = load(name)
    return cases.from_grid_file(gf, tide=((amp, cases.M2_HOURS),), dt=dt), kw
