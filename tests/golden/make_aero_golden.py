"""Generates tests/golden/aero_golden.json with FlowCraft's own code only:
LbmReference steps the case (oracle/_ref/libfcref.so), then
FieldOverlay::ComputeAerodynamicForces (FieldOverlay.cpp:469-621, compiled
into the same library) integrates the field, on the grid's own spacing and on
a shifted, scaled one. Run here (where the reference tree exists):
python tests/golden/make_aero_golden.py
"""
from __future__ import annotations

import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.abspath(os.path.join(HERE, "..", "..")))
sys.path.insert(0, HERE)

from cases import CASES, OracleAdapter, geometry  # noqa: E402
from oracle import oracle as orc  # noqa: E402

# (case, steps, cell size, origin)
AERO_CASES = [
    ("wing_q19", 60, 1.0, (0.0, 0.0, 0.0)),
    ("wing_q19", 200, 0.37, (-3.5, 2.25, 10.0)),
    ("sphere48_q19", 60, 1.0, (0.0, 0.0, 0.0)),
    ("ground_q15", 100, 0.5, (1.0, -2.0, 0.25)),
]


def main():
    orc.build()
    if not orc.available("ref"):
        raise SystemExit("oracle/_ref/libfcref.so missing: the reference tree is needed to generate fixtures")
    out = {"generator": "FlowCraft LbmReference + FieldOverlay::ComputeAerodynamicForces via oracle/_ref",
           "cases": []}
    for name, steps, cs, origin in AERO_CASES:
        case = CASES[name]
        solid, _ = geometry(case["geom"])
        sim = OracleAdapter(case, precision="ref")
        sim.step(steps)
        field = sim.readback_field()
        r = orc.aero_forces_reference(solid, field, cs, origin)
        out["cases"].append({"case": name, "steps": steps, "cell_size": cs, "origin": list(origin),
                             **{k: (list(v) if isinstance(v, tuple) else v) for k, v in r.items()}})
        print(name, steps, r["force"], r["center_of_pressure"])
    with open(os.path.join(HERE, "aero_golden.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
