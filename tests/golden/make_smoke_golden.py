"""Generates tests/golden/smoke_golden.json with FlowCraft's own code only:
LbmReference steps the 48x24x24 sphere case 60 steps (oracle/_ref), then
SmokeTrailSystem::Step (FlowCraft/SmokeTrail.cpp:278-343, compiled into the
same library) advects seeded particles through that field, free and
confined to a z plane. The numpy restatement (oracle/smoke_oracle.py) must
reproduce every trail bit for bit before the file is written. Run here
(where the reference tree exists): python tests/golden/make_smoke_golden.py
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.abspath(os.path.join(HERE, "..", "..")))
sys.path.insert(0, HERE)

from cases import CASES, field_digest, geometry, params_for  # noqa: E402
from oracle import oracle as orc  # noqa: E402
from oracle import smoke_oracle as so  # noqa: E402

CASE, CASE_STEPS = "sphere48_q19", 60
TRAIL, STEPS = 8, 7
RUNS = [  # (name, mm per second per lattice unit, dt, confine axis, confine index)
    ("free", 40.0, 0.05, -1, 0),
    ("plane_z", 25.0, 0.3, 2, 12),  # dt above the 0.1 s cap
]


def positions(solid, dims, rng, count, z_plane=None):
    nx, ny, nz = dims
    sd = solid.reshape(nz, ny, nx)
    out = []
    while len(out) < count:
        gx = rng.uniform(6.0, nx - 8.0)
        gy = rng.uniform(2.0, ny - 2.0)
        gz = z_plane + 0.5 if z_plane is not None else rng.uniform(2.0, nz - 2.0)
        if sd[int(gz), int(gy), int(gx)]:
            continue
        out.append((gy, gx, gz))  # world (x, y, z) = grid (y, x, z)
    return np.array(out, dtype=np.float32)


def main():
    case = CASES[CASE]
    solid, sdf = geometry(case["geom"])
    nz, ny, nx = solid.shape
    dims = (nx, ny, nz)
    o = orc.Oracle(solid, sdf, case["q"], params_for(case), case["seed_mid"], "ref")
    o.step(CASE_STEPS)
    field = o.readback_field()
    o.close()
    rng = np.random.default_rng(20261203)
    out = {"case": CASE, "case_steps": CASE_STEPS, "field_sha256": field_digest(field), "trail_length": TRAIL,
           "steps": STEPS, "cell_size": 1.0, "origin": [0.0, 0.0, 0.0], "runs": []}
    for name, mm, dt, axis, index in RUNS:
        pos = positions(solid, dims, rng, 48, z_plane=index if axis == 2 else None)
        trails, lens = so.step_reference(solid, field, dims, 1.0, (0.0, 0.0, 0.0), pos, TRAIL, STEPS, mm, dt,
                                         False, axis, index)
        mine, ok = so.advect(field, solid, dims, 1.0, (0.0, 0.0, 0.0), pos, STEPS, mm, dt, axis)
        keep = ok & (lens == min(STEPS + 1, TRAIL))
        assert keep.sum() >= 40, keep.sum()
        for p in np.nonzero(keep)[0]:
            want = trails[p, :lens[p]]
            got = mine[p, STEPS + 1 - lens[p]:]
            assert np.array_equal(want.view(np.uint32), got.view(np.uint32)), (name, p)
        out["runs"].append({"name": name, "mm_per_sec": mm, "dt": dt, "confine_axis": axis, "confine_index": index,
                            "positions": pos.tolist(), "keep": keep.astype(int).tolist(),
                            "trail_bits": trails.view(np.uint32).tolist(), "lens": lens.tolist()})
        print(name, "particles kept", int(keep.sum()), "of", len(pos))
    with open(os.path.join(HERE, "smoke_golden.json"), "w") as f:
        json.dump(out, f)


if __name__ == "__main__":
    main()
