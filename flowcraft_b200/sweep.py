"""Angle-of-attack sweeps on the GPU: many wing lattices stepped as one batch
(flowcraft_b200.batch) and their forces reduced to an aerodynamic polar in
the fields of the reference's XFLR5-style polar sweep
(PanelSolver::PolarPoint / PolarSweepResult, FlowCraft/PanelSolver.h:100-141).

* ``c3_lattices(seed)``: the batched-throughput set: 16 NACA 2412 lattices
  with sizes from 64x32x32 to 256x128x128 (2:1:1), chord 0.375 nx, angles
  linspace(-8, 14, 16), U in [0.04, 0.08] and Re in [1e3, 2e4], all drawn
  from one seeded generator.
* ``polar_sweep(...)``: one wing at one lattice size and Reynolds number over
  a list of angles, each angle a batch member; forces are averaged over the
  last fifth of the steps.

Forces and lengths are in lattice units (cells, lattice force); the
coefficients are normalized by 0.5 rho U^2 chord span with rho = 1.
"""
from __future__ import annotations

import math
from dataclasses import asdict, dataclass, field

import numpy as np

OSWALD = 0.85  # PanelSolver::PolarSweepResult::oswaldEfficiency default


@dataclass
class PolarPoint:
    alphaDeg: float = 0.0
    cl: float = 0.0
    cd: float = 0.0
    cdi: float = 0.0
    cd0: float = 0.0
    cm: float = 0.0
    ld: float = 0.0
    liftN: float = 0.0   # lattice force units here
    dragN: float = 0.0
    cpX_mm: float = 0.0  # centre of pressure behind the leading edge, in cells


@dataclass
class PolarSweepResult:
    points: list = field(default_factory=list)
    clAlphaPerDeg: float = 0.0
    clAlphaPerRad: float = 0.0
    alphaZeroLiftDeg: float = 0.0
    maxLD: float = 0.0
    alphaAtMaxLD: float = 0.0
    minCD0: float = 0.0
    oswaldEfficiency: float = OSWALD
    refArea: float = 0.0   # chord x span, cells^2
    refChord: float = 0.0
    refSpan: float = 0.0
    aspectRatio: float = 0.0
    valid: bool = False
    meta: dict = field(default_factory=dict)

    def to_dict(self) -> dict:
        d = asdict(self)
        d["points"] = [asdict(p) if not isinstance(p, dict) else p for p in self.points]
        return d

    def markdown(self) -> str:
        rows = ["| alpha (deg) | Cl | Cd | Cdi | Cd0 | Cm(c/4) | L/D | x_cp / c |", "|---|---|---|---|---|---|---|---|"]
        for p in self.points:
            rows.append(f"| {p.alphaDeg:.1f} | {p.cl:.4f} | {p.cd:.4f} | {p.cdi:.4f} | {p.cd0:.4f} | {p.cm:.4f} | "
                        f"{p.ld:.2f} | {p.cpX_mm / self.refChord:.3f} |")
        return "\n".join(rows)


def wing_lattice(nx: int, aoa_deg: float, device: int = 0, digits: str = "2412"):
    """(solid, sdf, chord, span, leading-edge x) of a 2:1:1 wing lattice."""
    import torch

    from . import geometry
    ny, nz = nx // 2, nx // 2
    chord = 0.375 * nx
    span = 0.75 * ny
    le_x = 0.25 * nx
    solid, sdf = geometry.naca_wing_grid(nx, ny, nz, chord=chord, span=span, aoa_deg=aoa_deg, digits=digits,
                                         le_x=le_x, xp=torch, device=f"cuda:{device}")
    return solid.contiguous(), sdf.contiguous(), chord, span, le_x


def c3_lattices(seed: int = 20261203):
    """The 16 (nx, alpha, U, Re) of the batched-throughput set."""
    rng = np.random.default_rng(seed)
    sizes = 2 * rng.integers(32, 129, size=16)          # nx in [64, 256], even
    alphas = np.linspace(-8.0, 14.0, 16)
    us = rng.uniform(0.04, 0.08, size=16)
    res = rng.uniform(1e3, 2e4, size=16)
    return [dict(nx=int(n), alpha=float(a), u=float(u), re=float(r)) for n, a, u, r in zip(sizes, alphas, us, res)]


def make_members(specs, storage="FP16_OFFSET", cs=0.1, device=0):
    """LbmSolver objects for (nx, alpha, u, re) specs, reset with the mid-speed seed."""
    from .lbm import LatticeModel, LbmSolver, Params, Storage, VoxelGrid
    out = []
    for sp in specs:
        solid, sdf, chord, span, le_x = wing_lattice(sp["nx"], sp["alpha"], device)
        nx = sp["nx"]
        s = LbmSolver()
        if not s.Init(device, VoxelGrid(nx, nx // 2, nx // 2, solid=solid, signedDistance=sdf), LatticeModel.D3Q19,
                      Storage[storage]):
            raise RuntimeError(s.LastError())
        tau = 0.5 + 3.0 * sp["u"] * chord / sp["re"]
        s.Reset(Params(tau=tau, inletVelocity=sp["u"], smagorinskyCs=cs), True)
        out.append((s, dict(sp, chord=chord, span=span, le_x=le_x, tau=tau)))
    return out


def polar_sweep(nx: int = 128, alphas=None, re: float = 5e3, u: float = 0.06, steps: int = 2000,
                storage: str = "FP16_OFFSET", cs: float = 0.1, device: int = 0, tune: bool = True,
                chunk: int = 50) -> PolarSweepResult:
    """Steps one lattice per angle as a batch and reduces the forces."""
    from .batch import CANDIDATES, LbmBatch
    alphas = list(np.linspace(-4.0, 12.0, 9) if alphas is None else alphas)
    mem = make_members([dict(nx=nx, alpha=a, u=u, re=re) for a in alphas], storage, cs, device)
    solvers = [m[0] for m in mem]
    batch = LbmBatch(solvers)
    tuned = batch.Tune(4) if tune else None
    done = len(CANDIDATES) * (4 + 2) if tune else 0
    avg_from = int(0.8 * steps)
    acc = np.zeros((len(alphas), 4))  # Fx, Fz, Fz * x_cp, count
    while done < steps:
        k = min(chunk, steps - done)
        k += k & 1
        batch.Step(k)
        done += k
        if done >= avg_from:
            for j, s in enumerate(solvers):
                a = s.AerodynamicForces()
                acc[j, 0] += a.forceSum[0]
                acc[j, 1] += a.forceSum[2]
                # world y is the flow axis (grid x): cell centres at x + 0.5, like le_x
                acc[j, 2] += a.forceSum[2] * a.centerOfPressure[1]
                acc[j, 3] += 1
    diverged = [s.HasDiverged() for s in solvers]
    batch.close()
    info = mem[0][1]
    chord, span, le_x = info["chord"], info["span"], info["le_x"]
    q = 0.5 * u * u * chord * span
    ar = span / chord
    pts = []
    for j, a in enumerate(alphas):
        n = max(acc[j, 3], 1)
        fx, fz = acc[j, 0] / n, acc[j, 1] / n
        xcp = acc[j, 2] / acc[j, 1] if abs(acc[j, 1]) > 1e-30 else le_x + 0.25 * chord
        cl, cd = fz / q, fx / q
        cdi = cl * cl / (math.pi * ar * OSWALD)
        # pitching moment about the quarter chord from the centre of pressure
        cm = -cl * (xcp - (le_x + 0.25 * chord)) / chord
        pts.append(PolarPoint(alphaDeg=float(a), cl=float(cl), cd=float(cd), cdi=float(cdi), cd0=float(cd - cdi),
                              cm=float(cm), ld=float(cl / cd) if cd != 0 else 0.0, liftN=float(fz), dragN=float(fx),
                              cpX_mm=float(xcp - le_x)))
    res = PolarSweepResult(points=pts, refArea=chord * span, refChord=chord, refSpan=span, aspectRatio=ar)
    lin = [(p.alphaDeg, p.cl) for p in pts if -4.0 <= p.alphaDeg <= 8.0]
    if len(lin) >= 2:
        A = np.array(lin)
        slope, icpt = np.polyfit(A[:, 0], A[:, 1], 1)
        res.clAlphaPerDeg = float(slope)
        res.clAlphaPerRad = float(slope * 180.0 / math.pi)
        res.alphaZeroLiftDeg = float(-icpt / slope) if slope != 0 else 0.0
    best = max(pts, key=lambda p: p.ld)
    res.maxLD, res.alphaAtMaxLD = best.ld, best.alphaDeg
    res.minCD0 = float(min(p.cd0 for p in pts))
    res.valid = not any(diverged)
    res.meta = {"lattice": [nx, nx // 2, nx // 2], "re": re, "u": u, "tau": info["tau"], "steps": steps,
                "storage": storage, "averaged_over_steps": [avg_from, steps], "tuned": tuned,
                "diverged": diverged}
    return res


def main(argv=None):
    import argparse
    import json
    ap = argparse.ArgumentParser(description="angle-of-attack polar of a NACA 2412 wing from a batched LBM run")
    ap.add_argument("--nx", type=int, default=128)
    ap.add_argument("--re", type=float, default=5e3)
    ap.add_argument("--u", type=float, default=0.06)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    r = polar_sweep(a.nx, re=a.re, u=a.u, steps=a.steps)
    if a.out:
        with open(a.out, "w") as f:
            json.dump(r.to_dict(), f, indent=1)
    print(r.markdown())
    print(json.dumps({k: v for k, v in r.to_dict().items() if k != "points"}))


if __name__ == "__main__":
    main()
