"""Generates the golden fixtures in tests/golden/*.json by running FlowCraft's
own CPU solver, LbmReference (FlowCraft/LbmReference.cpp, compiled unmodified
from the reference tree into oracle/_ref/libfcref.so by oracle/Makefile), on
every case of cases.py.

Each fixture records, per checkpoint of the case's step schedule: the SHA-256
of the full 4-float-per-cell field (bit-exact pin), the float32 bit patterns
of a fixed random subsample of cells, and LbmReference::ComputeStats. Run
here (where the reference tree exists):  python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.abspath(os.path.join(HERE, "..", "..")))
sys.path.insert(0, HERE)

from cases import CASES, OracleAdapter, field_digest, geometry, input_digest, run_schedule, sample_indices  # noqa
from oracle import oracle as orc  # noqa: E402


def main(names=None):
    orc.build()
    if not orc.available("ref"):
        raise SystemExit("oracle/_ref/libfcref.so missing: the reference tree is needed to generate fixtures")
    for name, case in CASES.items():
        if names and name not in names:
            continue
        t0 = time.time()
        solid, sdf = geometry(case["geom"])
        sim = OracleAdapter(case, precision="ref")
        n = solid.size
        idx = sample_indices(n)
        cps = []

        def on_cp(step, field):
            bits = field.view(np.uint32).reshape(n, 4)[idx]
            cps.append({"step": step, "field_sha256": field_digest(field),
                        "sample_bits": bits.tolist(), "stats": sim.stats(),
                        "diverged": bool(sim.o.has_diverged())})

        run_schedule(sim, case, on_cp)
        fx = {"case": name, "generator": "FlowCraft LbmReference via oracle/_ref/libfcref.so",
              "dims": case["geom"]["dims"], "q": case["q"], "input_sha256": input_digest(solid, sdf),
              "sample_idx": idx.tolist(), "checkpoints": cps}
        with open(os.path.join(HERE, f"{name}.json"), "w") as f:
            json.dump(fx, f, separators=(",", ":"))
        print(f"{name}: {len(cps)} checkpoints, {time.time() - t0:.1f}s")


if __name__ == "__main__":
    main(sys.argv[1:] or None)
