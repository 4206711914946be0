"""A-posteriori evaluation of the learned closure.

The reference is a fine Smagorinsky run (FP32, twice the resolution), whose
time-averaged velocity field is box-filtered 2x onto the coarse lattice and
whose time-averaged forces are scaled to it. The coarse lattice is run twice
from the same seed, with the Smagorinsky closure and with the learned
closure, in the same storage format (FP16 offsets, the format the learned
closure runs in), so the two coarse runs differ only in the closure. Each is
compared with the filtered fine run:

* the time-averaged drag and lift (the device FP64 force integral); a fine
  force is 4x the coarse one for the same coefficient (area scales with the
  square of the resolution at the same lattice velocity);
* the time-averaged velocity in the wake (every coarse fluid cell downstream
  of the body whose 8 fine cells are fluid), as an rms error over U.

Time: at the same lattice velocity one coarse step spans two fine steps, so
the fine run takes twice the steps and samples at twice the interval.

``evaluate`` returns a dict; ``python -m flowcraft_b200.closure_eval`` runs
the closure configuration's own evaluation (512x256x256 fine, 256x128x128
coarse) and prints it as JSON.
"""
from __future__ import annotations

import json
from dataclasses import dataclass

import numpy as np


@dataclass
class EvalCase:
    name: str
    geom: str            # "sphere" or "wing"
    re: float            # on the sphere diameter / the wing chord
    nx: int = 256        # coarse lattice; the fine one is 2x per axis
    ny: int = 128
    nz: int = 128
    u: float = 0.06
    coarse_steps: int = 2000
    avg_from: float = 0.6  # fraction of the run where averaging starts
    every: int = 50        # coarse steps between samples


def case_geometry(kind: str, nx: int, ny: int, nz: int):
    """(solid, sdf, reference length) of the training geometries (the
    placement of flowcraft_b200.closure_train.c4_cases) on an nx x ny x nz
    lattice."""
    from . import geometry
    if kind == "sphere":
        r = nz * 0.09
        solid, sdf = geometry.sphere_grid(nx, ny, nz, nx * 0.3, ny * 0.5, nz * 0.5, r)
        return solid, sdf, 2.0 * r
    chord = 0.375 * nx / 2
    solid, sdf = geometry.naca_wing_grid(nx, ny, nz, chord=chord, span=ny * 0.6, aoa_deg=6, digits="2412")
    return solid, sdf, chord


def _run(solid, sdf, tau, u, storage, closure, steps, avg_start, every, device):
    """Force and velocity field averaged over samples at avg_start, avg_start
    + every, ... < steps (taken after those many steps)."""
    from .lbm import LatticeModel, LbmSolver, Params, Storage, VoxelGrid
    nz, ny, nx = solid.shape
    s = LbmSolver()
    ok = s.Init(device, VoxelGrid(nx, ny, nz, solid=solid.ravel(), signedDistance=np.asarray(sdf).ravel()),
                LatticeModel.D3Q19, Storage[storage])
    if not ok:
        raise RuntimeError(s.LastError())
    s.Reset(Params(tau=tau, inletVelocity=u, smagorinskyCs=0.1), True)
    if closure is not None:
        s.SetClosure(closure)
    s.Step(None, avg_start)
    force = np.zeros(3)
    vel = np.zeros((nz, ny, nx, 3))
    n = 0
    done = avg_start
    while done < steps:
        force += np.asarray(s.AerodynamicForces().forceSum, dtype=np.float64)
        vel += s.ReadbackField().reshape(nz, ny, nx, 4)[..., 1:4]
        n += 1
        s.Step(None, every)
        done += every
    diverged = s.HasDiverged()
    cov = s.ClosureCoverage() if closure is not None else None
    s.close()
    return {"force": force / n, "vel": vel / n, "samples": n, "diverged": diverged, "coverage": cov}


def box_filter2(vel_fine, solid_fine):
    """2x box filter of a fine field (nz, ny, nx, 3) onto the coarse lattice,
    and the coarse cells whose 8 fine cells are all fluid."""
    nz, ny, nx, _ = vel_fine.shape
    v = vel_fine.reshape(nz // 2, 2, ny // 2, 2, nx // 2, 2, 3).mean(axis=(1, 3, 5))
    fluid = (solid_fine == 0).reshape(nz // 2, 2, ny // 2, 2, nx // 2, 2).all(axis=(1, 3, 5))
    return v, fluid


def evaluate(case: EvalCase, closure, device: int = 0) -> dict:
    fine_solid, fine_sdf, lref_f = case_geometry(case.geom, 2 * case.nx, 2 * case.ny, 2 * case.nz)
    solid, sdf, lref = case_geometry(case.geom, case.nx, case.ny, case.nz)
    tau_f = 0.5 + 3.0 * case.u * lref_f / case.re
    tau_c = 0.5 + 3.0 * case.u * lref / case.re
    start = int(case.avg_from * case.coarse_steps)
    fine = _run(fine_solid, fine_sdf, tau_f, case.u, "FP32", None, 2 * case.coarse_steps, 2 * start,
                2 * case.every, device)
    vf, valid = box_filter2(fine["vel"], fine_solid)
    ref_force = fine["force"] / 4.0
    del fine["vel"]
    # the wake: coarse fluid cells downstream of the body's last solid cell
    xs = np.nonzero(solid.any(axis=(0, 1)))[0]
    wake = valid & (solid == 0)
    wake[:, :, :xs.max() + 2] = False
    out = {"case": case.__dict__, "tau_fine": tau_f, "tau_coarse": tau_c, "wake_cells": int(wake.sum()),
           "fine": {"force": ref_force.tolist(), "samples": fine["samples"], "diverged": fine["diverged"]}}
    for name, cl in (("smagorinsky", None), ("learned", closure)):
        r = _run(solid, sdf, tau_c, case.u, "FP16_OFFSET", cl, case.coarse_steps, start, case.every, device)
        d = r["vel"] - vf
        rms = float(np.sqrt((d[wake] ** 2).sum(axis=-1).mean()) / case.u)
        out[name] = {"force": r["force"].tolist(), "drag_vs_fine": float(r["force"][0] / ref_force[0] - 1.0),
                     "lift_vs_fine": float(r["force"][2] / ref_force[2] - 1.0) if abs(ref_force[2]) > 0 else None,
                     "wake_rms_du_over_u": rms, "diverged": r["diverged"], "coverage": r["coverage"]}
    s, l = out["smagorinsky"], out["learned"]
    out["learned_closer_in_wake"] = l["wake_rms_du_over_u"] < s["wake_rms_du_over_u"]
    out["learned_closer_in_drag"] = abs(l["drag_vs_fine"]) < abs(s["drag_vs_fine"])
    return out


C4_EVAL_CASES = [EvalCase("sphere_re2e4", "sphere", 2e4), EvalCase("wing2412_re1e4", "wing", 1e4)]


def main(argv=None):
    import argparse
    import os

    from .closure import ClosureWeights
    ap = argparse.ArgumentParser(description="a-posteriori evaluation of the learned closure")
    ap.add_argument("--weights", default=os.path.join(os.path.dirname(__file__), "data", "closure_c4.json"))
    ap.add_argument("--scale", type=int, default=1, help="divide the coarse lattice by this per axis")
    ap.add_argument("--steps", type=int, default=2000)
    a = ap.parse_args(argv)
    cw = ClosureWeights.load(a.weights)
    res = []
    for c in C4_EVAL_CASES:
        c = EvalCase(c.name, c.geom, c.re, c.nx // a.scale, c.ny // a.scale, c.nz // a.scale,
                     coarse_steps=a.steps // a.scale)
        res.append(evaluate(c, cw))
        print(json.dumps(res[-1]), flush=True)
    return res


if __name__ == "__main__":
    main()
