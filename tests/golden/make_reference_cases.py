"""Writes reference_test_cases.npz: the reference's three flow test cases
(testing/tests_flow/{L05_Implicit_Test01, L08_Sed_LSTF,
L10_Sed_BedAggradation_SedSorting}) as the flow step reads them -- each
grid's cell rows as parsed from its .tel file (cms2d_b200.gridio.parse_tel)
and the flow settings of its .cmcards (cms2d_b200.cards.flow_settings).

The GPU tests run these cases where the reference tree is absent.  Run from
the repository root:

    python tests/golden/make_reference_cases.py [REFERENCE_DIR]

REFERENCE_DIR defaults to $CMS_REFERENCE_DIR, else /root/reference.
"""
from __future__ import annotations

import glob
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from cms2d_b200 import cards, gridio  # noqa: E402


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CMS_REFERENCE_DIR", "/root/reference")
    out = {}
    names = []
    for cm in sorted(glob.glob(os.path.join(ref, "testing", "tests_flow", "*", "*.cmcards"))):
        case = os.path.basename(os.path.dirname(cm))
        kw, dt, grid = cards.flow_settings(cards.read_cards(cm), os.path.dirname(cm))
        angle, x0, y0, rows = gridio.parse_tel(grid)
        names.append(case)
        out[f"{case}/rows"] = rows
        out[f"{case}/origin"] = np.array([angle, x0, y0])
        out[f"{case}/settings"] = np.array(json.dumps({"flow": kw, "dt": dt,
                                                       "grid": os.path.basename(grid)}))
    out["cases"] = np.array(names)
    np.savez_compressed(os.path.join(HERE, "reference_test_cases.npz"), **out)
    print(f"wrote {len(names)} cases: {', '.join(names)}")


if __name__ == "__main__":
    main()
