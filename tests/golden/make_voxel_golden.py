"""Generates tests/golden/voxel_golden.json by running FlowCraft's own CPU
voxelizer, Voxelizer::Voxelize (FlowCraft/Voxelizer.cpp, compiled unmodified
from the reference tree into oracle/_ref/libfcref.so by oracle/Makefile), on
every GOLDEN case of voxel_cases.py. Each entry records the mesh digest, the
derived grid (dims, cell size, origin as float32 bit patterns) and SHA-256
digests of the solid mask and of the signed-distance floats. Run here (where
the reference tree exists):  python tests/golden/make_voxel_golden.py
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.abspath(os.path.join(HERE, "..", "..")))
sys.path.insert(0, HERE)

from voxel_cases import GOLDEN, digest, mesh, mesh_digest  # noqa: E402
from oracle import oracle as orc  # noqa: E402


def main():
    orc.build()
    if not orc.available("ref"):
        raise SystemExit("oracle/_ref/libfcref.so missing: the reference tree is needed to generate fixtures")
    out = {"generator": "FlowCraft Voxelizer::Voxelize via oracle/_ref/libfcref.so", "cases": {}}
    for name, case in GOLDEN.items():
        pos, idx = mesh(case["mesh"])
        pad = case.get("padding", (0.3, 1.0, 0.5))
        dims, cell, origin, solid, sdf = orc.voxelize_reference(pos, idx, case["res"], pad)
        out["cases"][name] = {
            "mesh_sha256": mesh_digest(pos, idx), "triangles": int(idx.size // 3), "dims": list(dims),
            "cell_bits": int(np.float32(cell).view(np.uint32)),
            "origin_bits": [int(v) for v in np.asarray(origin, np.float32).view(np.uint32)],
            "solid_sha256": digest(solid), "sdf_sha256": digest(sdf), "solid_cells": int(solid.sum()),
            "finite_sdf_cells": int(np.isfinite(sdf).sum()),
        }
        print(name, dims, int(solid.sum()))
    with open(os.path.join(HERE, "voxel_golden.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
