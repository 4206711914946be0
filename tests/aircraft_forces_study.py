"""Drag and lift of the large benchmark configuration: the procedural
high-wing aircraft on 1024x512x512 (268M cells), U 0.05, Re 1e5 on the
60-cell root chord, Cs 0.1, mid-speed seed, 3000 steps. The configuration's
own run, with the learned closure in FP16 offset storage, against the FP32
Smagorinsky GPU run (the accuracy target: Cd and Cl within 1 %), and FP16
Smagorinsky for context.

Drag and lift are the x and z sums of the solid cells' momentum-exchange
force (the device FP64 integral, AerodynamicForces), averaged every 10 steps
over the last fifth of the run, as the polar sweep averages them. Ratios of
forces are ratios of coefficients (same reference area and dynamic
pressure).

Not collected by pytest; run on a GPU machine:  python tests/aircraft_forces_study.py
It prints one JSON object and a markdown table. STUDY_STEPS overrides 3000.
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
sys.path.insert(0, ROOT)

STEPS = int(os.environ.get("STUDY_STEPS", "3000"))
AVG_FROM = STEPS - STEPS // 5


def run(cfg, solid, sdf, storage, learned):
    import bench
    from flowcraft_b200 import LatticeModel, LbmSolver, Params, Storage, VoxelGrid
    from flowcraft_b200.closure import ClosureWeights
    s = LbmSolver()
    grid = VoxelGrid(cfg["nx"], cfg["ny"], cfg["nz"], solid=solid, signedDistance=sdf)
    assert s.Init(0, grid, LatticeModel.D3Q19, Storage[storage]), s.LastError()
    s.Reset(Params(tau=bench.tau_for(cfg), inletVelocity=cfg["u"], smagorinskyCs=cfg["cs"]), True)
    if learned:
        s.SetClosure(ClosureWeights.load(bench.CLOSURE_WEIGHTS))
    t0 = time.perf_counter()
    s.Step(None, AVG_FROM)
    acc, n = np.zeros(3), 0
    for _ in range(AVG_FROM, STEPS, 10):
        s.Step(None, 10)
        acc += np.asarray(s.AerodynamicForces().forceSum, dtype=np.float64)
        n += 1
    last = np.asarray(s.AerodynamicForces().forceSum, dtype=np.float64)
    cov = s.ClosureCoverage() if learned else None
    diverged = s.HasDiverged()
    s.close()
    return {"avg": (acc / n).tolist(), "last": last.tolist(), "seconds": time.perf_counter() - t0,
            "diverged": diverged, "coverage": cov}


def main():
    import bench
    import torch
    cfg = bench.CONFIGS["large"]
    solid_t, sdf_t = bench.build_geometry(cfg, "cuda:0")
    solid, sdf = solid_t.cpu().numpy(), sdf_t.cpu().numpy()
    del solid_t, sdf_t
    torch.cuda.empty_cache()
    res = {}
    for name, storage, learned in (("fp32_smagorinsky", "FP32", False), ("fp16_learned", "FP16_OFFSET", True),
                                   ("fp16_smagorinsky", "FP16_OFFSET", False)):
        res[name] = run(cfg, solid, sdf, storage, learned)
        torch.cuda.empty_cache()
    ref = np.asarray(res["fp32_smagorinsky"]["avg"])
    ref_last = np.asarray(res["fp32_smagorinsky"]["last"])
    for name, r in res.items():
        a, l = np.asarray(r["avg"]), np.asarray(r["last"])
        r["drag_vs_fp32"] = a[0] / ref[0] - 1.0
        r["lift_vs_fp32"] = a[2] / ref[2] - 1.0
        r["drag_vs_fp32_last"] = l[0] / ref_last[0] - 1.0
        r["lift_vs_fp32_last"] = l[2] / ref_last[2] - 1.0
    print(json.dumps({"steps": STEPS, "avg_from": AVG_FROM, "runs": res}))
    print()
    print("| run | drag (avg) | lift (avg) | drag vs FP32 | lift vs FP32 | last step: drag / lift vs FP32 |")
    print("|---|---|---|---|---|---|")
    for name, r in res.items():
        a = r["avg"]
        print(f"| {name} | {a[0]:.5g} | {a[2]:.5g} | {100 * r['drag_vs_fp32']:+.2f} % | "
              f"{100 * r['lift_vs_fp32']:+.2f} % | {100 * r['drag_vs_fp32_last']:+.2f} % / "
              f"{100 * r['lift_vs_fp32_last']:+.2f} % |")


if __name__ == "__main__":
    main()
