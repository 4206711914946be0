"""Precision study of the storage formats (the 384x192x192 NACA 0012
precision configuration): the GPU's FP32, FP16-offset and BF16-offset
storage, and FP16 with the learned closure, against the FP64 oracle, on
D3Q19 and D3Q15.

Case: NACA 0012 wing, chord 96, span 128, 4 deg, on 384x192x192 (14.2M
cells), U 0.06, Re 1e4 on the chord (tau 0.50173), mid-speed seed, 5000
steps, Smagorinsky Cs 0.1. D3Q15 with the regularized collision does not
hold this viscosity: from the mid-speed start it diverges within 100-400
steps at every tau up to 0.55 (Re 1e4 down to 290, Cs 0.1 to 0.25, U 0.06
or 0.03, with or without the signed distance), in FP32, which reproduces the
reference's CPU solver bit for bit, and in FP64. It is stable for the 5000
steps at tau 0.6 (Re 173 on the chord), so D3Q15 runs there (D3Q15_TAU).
Drag and lift are the x and z sums of the
solid cells' momentum-exchange force, normalized by 0.5 rho U^2 chord
span, averaged every 10 steps over the last fifth of the run.

The oracle runs take hours of host CPU and the GPU runs seconds, so the
study runs in three phases that share a directory (not collected by
pytest):

  python tests/precision_study.py oracle --lattice 19 --out DIR   (host CPU)
  python tests/precision_study.py gpu --out DIR                   (a B200)
  python tests/precision_study.py compare --out DIR

Fields are compared on every 4th cell along each axis (96x48x48 cells, the
fluid ones), which keeps the GPU phase's output small; forces use the whole
lattice. ``--half`` runs the same case at half size (192x96x96, chord 48,
span 64, the same tau) for 1000 steps.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
sys.path.insert(0, ROOT)

U = 0.06
D3Q19_CS = 0.1
D3Q15_CS = 0.1
D3Q15_TAU = 0.6
SUB = 4  # field comparison on every SUB-th cell per axis


def case(half: bool):
    if half:
        return dict(nx=192, ny=96, nz=96, chord=48.0, span=64.0, aoa=4.0, steps=1000)
    return dict(nx=384, ny=192, nz=192, chord=96.0, span=128.0, aoa=4.0, steps=5000)


def tau_of(c, q=19):
    """The full-size case's viscosity at either size (D3Q15: D3Q15_TAU)."""
    return 0.5 + 3.0 * U * 96.0 / 1e4 if q == 19 else D3Q15_TAU


def cs_of(q):
    return D3Q19_CS if q == 19 else D3Q15_CS


def geometry(c):
    from flowcraft_b200 import geometry as geo
    solid, sdf = geo.naca_wing_grid(c["nx"], c["ny"], c["nz"], chord=c["chord"], span=c["span"], aoa_deg=c["aoa"],
                                    digits="0012")
    return np.ascontiguousarray(solid, np.uint8), np.ascontiguousarray(sdf, np.float32)


def coeffs(force, c):
    q = 0.5 * U * U * c["chord"] * c["span"]
    return float(force[0] / q), float(force[2] / q)


def subsample(field, c):
    f = np.asarray(field).reshape(c["nz"], c["ny"], c["nx"], 4)
    return np.ascontiguousarray(f[::SUB, ::SUB, ::SUB])


def run_oracle(c, q, threads, out):
    from oracle import oracle as orc
    solid, sdf = geometry(c)
    p = orc.Params(tau_of(c, q), U, False, True, True, cs_of(q))
    o = orc.Oracle(solid, sdf, q, p, seed_mid=True, precision="f64", threads=threads)
    steps = c["steps"]
    avg_from = steps - steps // 5
    t0 = time.time()
    o.step(avg_from)
    acc, n = np.zeros(3), 0
    s = solid.ravel().astype(bool)
    f = None
    for _ in range(avg_from, steps, 10):
        o.step(10)
        f = o.readback_field_f64().reshape(-1, 4)
        acc += f[s][:, 1:4].sum(axis=0)
        n += 1
    np.savez(os.path.join(out, f"fp64_q{q}.npz"), sub=subsample(f, c), force=f[s][:, 1:4].sum(axis=0),
             force_avg=acc / n, diverged=o.has_diverged(), seconds=time.time() - t0)
    o.close()


def run_gpu_variant(c, q, storage, closure, solid, sdf):
    from flowcraft_b200.lbm import LatticeModel, LbmSolver, Params, Storage, VoxelGrid
    s = LbmSolver()
    g = VoxelGrid(c["nx"], c["ny"], c["nz"], solid=solid.ravel(), signedDistance=sdf.ravel())
    assert s.Init(0, g, LatticeModel.D3Q19 if q == 19 else LatticeModel.D3Q15, Storage[storage]), s.LastError()
    s.Reset(Params(tau=tau_of(c, q), inletVelocity=U, smagorinskyCs=cs_of(q)), True)
    if closure is not None:
        s.SetClosure(closure)
    steps = c["steps"]
    avg_from = steps - steps // 5
    s.Step(None, avg_from)
    acc, n = np.zeros(3), 0
    for _ in range(avg_from, steps, 10):
        s.Step(None, 10)
        acc += np.asarray(s.AerodynamicForces().forceSum)
        n += 1
    f = s.ReadbackField()
    force = np.asarray(s.AerodynamicForces().forceSum)
    diverged = s.HasDiverged()
    s.close()
    return dict(sub=subsample(f, c), force=force, force_avg=acc / n, diverged=diverged)


def run_gpu(c, out):
    from flowcraft_b200.closure import ClosureWeights
    cw = ClosureWeights.load(os.path.join(ROOT, "flowcraft_b200", "data", "closure_c4.json"))
    solid, sdf = geometry(c)
    for q in (19, 15):
        for name, storage, closure in (("FP32", "FP32", None), ("FP16_OFFSET", "FP16_OFFSET", None),
                                       ("BF16_OFFSET", "BF16_OFFSET", None),
                                       ("FP16_OFFSET+learned", "FP16_OFFSET", cw)):
            if closure is not None and q != 19:
                continue
            t0 = time.time()
            r = run_gpu_variant(c, q, storage, closure, solid, sdf)
            np.savez(os.path.join(out, f"gpu_q{q}_{name}.npz"), seconds=time.time() - t0, **r)
            print(f"D3Q{q} {name}: diverged={r['diverged']} {time.time() - t0:.1f}s", flush=True)


def errors(sub, ref, solid_sub):
    fl = ~solid_sub.astype(bool).ravel()
    a, b = sub.reshape(-1, 4)[fl].astype(np.float64), ref.reshape(-1, 4)[fl]
    ua, ub = np.linalg.norm(a[:, 1:], axis=1), np.linalg.norm(b[:, 1:], axis=1)
    return {"max_drho": float(np.abs(a[:, 0] - b[:, 0]).max()), "max_du": float(np.abs(ua - ub).max()),
            "rms_du": float(np.sqrt(np.mean((ua - ub) ** 2))), "umax": float(ub.max()), "cells": int(fl.sum())}


def compare(c, out):
    solid, _ = geometry(c)
    solid_sub = solid[::SUB, ::SUB, ::SUB]
    rows = []
    for q in (19, 15):
        ref_path = os.path.join(out, f"fp64_q{q}.npz")
        ref = np.load(ref_path) if os.path.exists(ref_path) else None
        g32 = np.load(os.path.join(out, f"gpu_q{q}_FP32.npz"))
        acd32, acl32 = coeffs(g32["force_avg"], c)
        for name in ("FP32", "FP16_OFFSET", "BF16_OFFSET", "FP16_OFFSET+learned"):
            path = os.path.join(out, f"gpu_q{q}_{name}.npz")
            if not os.path.exists(path):
                continue
            g = np.load(path)
            cd, cl = coeffs(g["force_avg"], c)
            row = {"lattice": f"D3Q{q}", "Cs": cs_of(q), "tau": tau_of(c, q), "variant": name,
                   "diverged": bool(g["diverged"]),
                   "Cd_avg": cd, "Cl_avg": cl, "dCd_vs_fp32_smag": cd / acd32 - 1.0,
                   "dCl_vs_fp32_smag": cl / acl32 - 1.0}
            if ref is not None:
                rcd, rcl = coeffs(ref["force_avg"], c)
                row.update(errors(g["sub"], ref["sub"], solid_sub))
                row.update({"Cd_fp64": rcd, "Cl_fp64": rcl, "dCd_vs_fp64": cd / rcd - 1.0,
                            "dCl_vs_fp64": cl / rcl - 1.0, "fp64_diverged": bool(ref["diverged"]),
                            "reference": "FP64 oracle, Smagorinsky"})
            rows.append(row)
    res = {"case": {**c, "tau": tau_of(c), "tau_d3q15": D3Q15_TAU, "U": U, "sub": SUB}, "rows": rows}
    print(json.dumps(res))
    print("\n| lattice (tau, Cs) | variant | max abs drho | max abs d|u| | rms d|u| | Cd avg | Cl avg | dCd vs FP64 | "
          "dCl vs FP64 | dCd vs FP32 Smag | dCl vs FP32 Smag |")
    print("|---|---|---|---|---|---|---|---|---|---|---|")
    for r in rows:
        e = (f"{r['max_drho']:.1e} | {r['max_du']:.1e} | {r['rms_du']:.1e}" if "max_drho" in r else "- | - | -")
        f64 = (f"{100 * r['dCd_vs_fp64']:+.2f} % | {100 * r['dCl_vs_fp64']:+.2f} %" if "dCd_vs_fp64" in r
               else "- | -")
        print(f"| {r['lattice']} ({r['tau']:.5f}, {r['Cs']}) | {r['variant']} | {e} | {r['Cd_avg']:.5f} | {r['Cl_avg']:.5f} | {f64} | "
              f"{100 * r['dCd_vs_fp32_smag']:+.2f} % | {100 * r['dCl_vs_fp32_smag']:+.2f} % |")
    return res


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("phase", choices=["oracle", "gpu", "compare"])
    ap.add_argument("--out", required=True)
    ap.add_argument("--lattice", type=int, default=19, choices=[19, 15])
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--half", action="store_true")
    a = ap.parse_args(argv)
    os.makedirs(a.out, exist_ok=True)
    c = case(a.half)
    if a.phase == "oracle":
        run_oracle(c, a.lattice, a.threads, a.out)
    elif a.phase == "gpu":
        run_gpu(c, a.out)
    else:
        compare(c, a.out)


if __name__ == "__main__":
    main()
