"""Precision study (the 384x192x192 NACA 0012 precision configuration at
half size): the GPU storage formats and the learned closure against the FP64
oracle, and the learned closure's drag and lift against the FP32 Smagorinsky
GPU run.

Case: NACA 0012 wing, chord 48, span 64, 4 deg, on 192x96x96 (the full-size
case halved, so nu and tau are the full-size case's: U 0.06, Re 5e3 on the
chord, tau 0.50173), Smagorinsky Cs 0.1, mid-speed seed, 1000 steps, D3Q19
and D3Q15. Drag and lift are the x and z sums of the solid cells'
momentum-exchange force (the device FP64 integral), normalized by
0.5 rho U^2 chord span.

Not collected by pytest; run on a GPU machine:  python tests/precision_study.py
It prints one JSON object and a markdown table. Cd and Cl are reported at
the last step and averaged over the last fifth of the steps (as the polar
sweep averages them). STUDY_GPU_ONLY=1 skips the FP64 oracle runs and
compares the GPU variants with each other only.
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
sys.path.insert(0, ROOT)

NX, NY, NZ, CHORD, SPAN, AOA, U = 192, 96, 96, 48.0, 64.0, 4.0, 0.06
STEPS = int(os.environ.get("STUDY_STEPS", "1000"))
AVG_FROM = STEPS - STEPS // 5
GPU_ONLY = os.environ.get("STUDY_GPU_ONLY", "0") == "1"
TAU = 0.5 + 3.0 * U * CHORD / 5e3
CS = 0.1


def geometry():
    from flowcraft_b200 import geometry as geo
    solid, sdf = geo.naca_wing_grid(NX, NY, NZ, chord=CHORD, span=SPAN, aoa_deg=AOA, digits="0012")
    return np.ascontiguousarray(solid, np.uint8), np.ascontiguousarray(sdf, np.float32)


def coeffs(force):
    q = 0.5 * U * U * CHORD * SPAN
    return force[0] / q, force[2] / q


def run_oracle(solid, sdf, q, closure=None):
    from oracle import oracle as orc
    p = orc.Params(TAU, U, False, True, True, CS)
    o = orc.Oracle(solid, sdf, q, p, seed_mid=True, precision="f64")
    if closure is not None:
        o.set_closure(closure)
    o.step(STEPS)
    f = o.readback_field_f64().reshape(-1, 4)
    o.close()
    s = solid.ravel().astype(bool)
    force = f[s][:, 1:4].sum(axis=0)
    return f, force


def run_gpu(solid, sdf, q, storage, closure=None):
    from flowcraft_b200.lbm import LatticeModel, LbmSolver, Params, Storage, VoxelGrid
    s = LbmSolver()
    g = VoxelGrid(NX, NY, NZ, solid=solid.ravel(), signedDistance=sdf.ravel())
    assert s.Init(0, g, LatticeModel.D3Q19 if q == 19 else LatticeModel.D3Q15, Storage[storage]), s.LastError()
    s.Reset(Params(tau=TAU, inletVelocity=U, smagorinskyCs=CS), True)
    if closure is not None:
        s.SetClosure(closure)
    s.Step(None, AVG_FROM)
    acc, n = np.zeros(3), 0
    for _ in range(AVG_FROM, STEPS, 10):
        s.Step(None, 10)
        acc += np.asarray(s.AerodynamicForces().forceSum)
        n += 1
    f = s.ReadbackField().reshape(-1, 4).astype(np.float64)
    a = s.AerodynamicForces()
    s.close()
    return f, np.asarray(a.forceSum), acc / max(n, 1)


def errors(f, ref, solid):
    fl = ~solid.ravel().astype(bool)
    d = np.abs(f - ref)[fl]
    ua, ub = np.linalg.norm(f[fl][:, 1:], axis=1), np.linalg.norm(ref[fl][:, 1:], axis=1)
    return {"max_drho": float(d[:, 0].max()), "max_du": float(np.abs(ua - ub).max()),
            "rms_du": float(np.sqrt(np.mean((ua - ub) ** 2))), "umax": float(ub.max())}


def main():
    from flowcraft_b200.closure import ClosureWeights
    cw = ClosureWeights.load(os.path.join(ROOT, "flowcraft_b200", "data", "closure_c4.json"))
    solid, sdf = geometry()
    out = {"case": f"NACA 0012 {NX}x{NY}x{NZ}, chord {CHORD}, span {SPAN}, {AOA} deg, U {U}, tau {TAU:.5f}, "
                   f"Cs {CS}, {STEPS} steps, forces averaged over steps {AVG_FROM}-{STEPS}", "rows": []}
    for q in ((19,) if GPU_ONLY else (19, 15)):
        t0 = time.time()
        if not GPU_ONLY:
            ref, fref = run_oracle(solid, sdf, q)
            cd0, cl0 = coeffs(fref)
            refl, frefl = (run_oracle(solid, sdf, q, cw) if q == 19 else (None, None))
        t1 = time.time()
        gpu = {st: run_gpu(solid, sdf, q, st) for st in ("FP32", "FP16_OFFSET", "BF16_OFFSET")}
        if q == 19:
            gpu["FP16_OFFSET+learned"] = run_gpu(solid, sdf, q, "FP16_OFFSET", cw)
        cd32, cl32 = coeffs(gpu["FP32"][1])
        acd32, acl32 = coeffs(gpu["FP32"][2])
        for name, (f, force, avg) in gpu.items():
            learned = name.endswith("learned")
            cd, cl = coeffs(force)
            acd, acl = coeffs(avg)
            row = {"lattice": f"D3Q{q}", "variant": name, "Cd": cd, "Cl": cl, "Cd_avg": acd, "Cl_avg": acl,
                   "dCd_rel_fp32_smag": (cd - cd32) / abs(cd32), "dCl_rel_fp32_smag": (cl - cl32) / abs(cl32),
                   "dCd_avg_rel_fp32_smag": (acd - acd32) / abs(acd32),
                   "dCl_avg_rel_fp32_smag": (acl - acl32) / abs(acl32)}
            if not GPU_ONLY:
                r = refl if learned else ref
                fr = frefl if learned else fref
                cdr, clr = coeffs(fr)
                row.update({"reference": "FP64 oracle" + (" + same closure" if learned else ""),
                            **errors(f, r, solid), "Cd_fp64": cdr, "Cl_fp64": clr,
                            "dCd_rel_fp64": (cd - cdr) / abs(cdr), "dCl_rel_fp64": (cl - clr) / abs(clr)})
            out["rows"].append(row)
        if not GPU_ONLY:
            out[f"oracle_seconds_q{q}"] = round(t1 - t0, 1)
            out[f"fp64_smagorinsky_q{q}"] = {"Cd": cd0, "Cl": cl0}
    print(json.dumps(out))
    print("\n| lattice | variant | Cd | Cl | dCd vs FP32 Smag | dCl vs FP32 Smag | Cd avg | Cl avg | "
          "dCd avg vs FP32 Smag | dCl avg vs FP32 Smag |")
    print("|---|---|---|---|---|---|---|---|---|---|")
    for r in out["rows"]:
        print(f"| {r['lattice']} | {r['variant']} | {r['Cd']:.5f} | {r['Cl']:.5f} | "
              f"{100 * r['dCd_rel_fp32_smag']:+.3f} % | {100 * r['dCl_rel_fp32_smag']:+.3f} % | {r['Cd_avg']:.5f} | "
              f"{r['Cl_avg']:.5f} | {100 * r['dCd_avg_rel_fp32_smag']:+.3f} % | {100 * r['dCl_avg_rel_fp32_smag']:+.3f} % |")
    if not GPU_ONLY:
        print("\n| lattice | variant | max|drho| | max|du| | rms|du| | dCd vs FP64 | dCl vs FP64 |")
        print("|---|---|---|---|---|---|---|")
        for r in out["rows"]:
            print(f"| {r['lattice']} | {r['variant']} | {r['max_drho']:.2e} | {r['max_du']:.2e} | {r['rms_du']:.2e} | "
                  f"{100 * r['dCd_rel_fp64']:+.3f} % | {100 * r['dCl_rel_fp64']:+.3f} % |")


if __name__ == "__main__":
    main()
