"""Parity cases shared by the golden-fixture generator (make_golden.py) and the
tests. Each case is a geometry spec + parameters + a step schedule; fixtures
record what FlowCraft's own LbmReference (compiled from its sources) produced
for it.

The first cases restate the reference's only LBM tests
(tests/gpu_vs_cpu_test.cpp:27-80 — the 48x24x24 sphere, tau 0.6, U 0.05,
Cs 0.12, mid-speed seed, 60 steps, both lattices — and :149-172, the +10 deg
inclined ellipsoid wing, 80 steps). The rest cover the boundary branches the
reference implements: no-slip and mixed side walls, reverse flow, a missing
SDF, solid cells beside the outlet, odd sizes, Smagorinsky off, the warm-start
ResetFromField path, and the 128x64x64 Re=100 sphere of the plain-FP32
parity configuration.
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

sys.path.insert(0, os.path.abspath(os.path.join(os.path.dirname(__file__), "..", "..")))

from flowcraft_b200.geometry import inclined_ellipsoid_wing_grid, sphere_grid  # noqa: E402

GOLDEN_DIR = os.path.dirname(os.path.abspath(__file__))


def geometry(spec: dict):
    """(solid u8 (nz,ny,nx), sdf f32 (nz,ny,nx) or None) for a geometry spec."""
    kind = spec["kind"]
    nx, ny, nz = spec["dims"]
    if kind == "sphere":
        solid, sdf = sphere_grid(nx, ny, nz, *spec["center"], spec["r"])
    elif kind == "wing":
        solid, sdf = inclined_ellipsoid_wing_grid(nx, ny, nz, reverse=spec.get("reverse", False))
    elif kind == "outlet_block":
        # a sphere plus a solid slab touching the x = nx-2 and x = 1 columns,
        # so the outlet (either direction) extrapolates from solid neighbours
        solid, sdf = sphere_grid(nx, ny, nz, *spec["center"], spec["r"])
        solid = solid.copy()
        sdf = sdf.copy()
        solid[:, 2:5, nx - 3:nx - 1] = 1
        sdf[:, 2:5, nx - 3:nx - 1] = -0.5
        solid[:, ny - 4:ny - 2, 1:3] = 1
        sdf[:, ny - 4:ny - 2, 1:3] = -0.5
    else:
        raise ValueError(kind)
    if not spec.get("sdf", True):
        sdf = None
    return solid, sdf


def input_digest(solid, sdf) -> str:
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(solid, dtype=np.uint8).tobytes())
    if sdf is not None:
        h.update(np.ascontiguousarray(sdf, dtype=np.float32).tobytes())
    return h.hexdigest()


def field_digest(field: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(field, dtype=np.float32).tobytes()).hexdigest()


REF_TEST = dict(tau=0.6, inlet_velocity=0.05, smagorinsky_cs=0.12)
SPHERE48 = {"kind": "sphere", "dims": [48, 24, 24], "center": [20, 12, 12], "r": 5}

CASES = {
    # tests/gpu_vs_cpu_test.cpp:27-80
    "sphere48_q19": dict(geom=SPHERE48, q=19, params=REF_TEST, seed_mid=True, steps=[60]),
    "sphere48_q15": dict(geom=SPHERE48, q=15, params=REF_TEST, seed_mid=True, steps=[60]),
    # tests/gpu_vs_cpu_test.cpp:149-172
    "wing_q19": dict(geom={"kind": "wing", "dims": [48, 32, 24]}, q=19, params=REF_TEST, seed_mid=True, steps=[80]),
    "wing_q15": dict(geom={"kind": "wing", "dims": [48, 32, 24]}, q=15, params=REF_TEST, seed_mid=True, steps=[80]),
    # boundary branches
    "noslip_reverse_q19": dict(geom={"kind": "sphere", "dims": [23, 13, 11], "center": [12, 6.3, 5.2], "r": 3.1},
                               q=19, params=dict(tau=0.55, inlet_velocity=0.07, smagorinsky_cs=0.15,
                                                 reverse_flow=1, free_slip_y=0, free_slip_z=0),
                               seed_mid=True, steps=[40]),
    "ground_q15": dict(geom={"kind": "sphere", "dims": [29, 15, 12], "center": [10, 7, 3], "r": 3.6},
                       q=15, params=dict(tau=0.7, inlet_velocity=0.04, smagorinsky_cs=0.1,
                                         free_slip_y=1, free_slip_z=0),
                       seed_mid=False, steps=[50]),
    "ywall_q19": dict(geom={"kind": "sphere", "dims": [17, 9, 14], "center": [7, 4.5, 7], "r": 2.4},
                      q=19, params=dict(tau=0.62, inlet_velocity=0.06, smagorinsky_cs=0.0,
                                        free_slip_y=0, free_slip_z=1),
                      seed_mid=True, steps=[35]),
    "nosdf_q19": dict(geom=dict(SPHERE48, sdf=False), q=19, params=REF_TEST, seed_mid=True, steps=[30]),
    "outlet_block_q19": dict(geom={"kind": "outlet_block", "dims": [21, 12, 9], "center": [8, 6, 4.5], "r": 2.5},
                             q=19, params=dict(tau=0.6, inlet_velocity=0.05, smagorinsky_cs=0.12),
                             seed_mid=True, steps=[1, 25], reverse_after=12),
    "tiny_q15": dict(geom={"kind": "sphere", "dims": [5, 3, 4], "center": [2.5, 1.5, 2], "r": 0.9},
                     q=15, params=dict(tau=0.58, inlet_velocity=0.05, smagorinsky_cs=0.12),
                     seed_mid=True, steps=[9]),
    "warmstart_q19": dict(geom=SPHERE48, q=19, params=REF_TEST, seed_mid=True, steps=[20, 20],
                          reset_from_field_after=20),
    # four 64-cell chunks per row with the sphere in the second: pairs cut by
    # the wall inside a row (the one-cell path of warps off the row ends)
    "interior_q19": dict(geom={"kind": "sphere", "dims": [256, 22, 20], "center": [101.5, 11, 10], "r": 5.3},
                         q=19, params=dict(tau=0.57, inlet_velocity=0.06, smagorinsky_cs=0.1), seed_mid=True,
                         steps=[60]),
    "interior_q15": dict(geom={"kind": "sphere", "dims": [256, 22, 20], "center": [101.5, 11, 10], "r": 5.3},
                         q=15, params=dict(tau=0.6, inlet_velocity=0.05, smagorinsky_cs=0.12), seed_mid=True,
                         steps=[60]),
    # plain-FP32 parity configuration: 128x64x64, sphere r=10 at (40,32,32),
    # U=0.05, Re=100 on the diameter -> nu = 0.05*20/100, tau = 3nu + 1/2
    "c1_q19": dict(geom={"kind": "sphere", "dims": [128, 64, 64], "center": [40, 32, 32], "r": 10}, q=19,
                   params=dict(tau=0.53, inlet_velocity=0.05, smagorinsky_cs=0.1), seed_mid=False,
                   steps=[200, 800]),
}


def params_for(case: dict):
    from oracle.oracle import Params
    p = dict(case["params"])
    return Params(tau=p["tau"], inlet_velocity=p["inlet_velocity"], reverse_flow=bool(p.get("reverse_flow", 0)),
                  free_slip_y=bool(p.get("free_slip_y", 1)), free_slip_z=bool(p.get("free_slip_z", 1)),
                  smagorinsky_cs=p["smagorinsky_cs"])


def sample_indices(n_cells: int, count: int = 384, seed: int = 7) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.unique(rng.integers(0, n_cells, size=count))


def run_schedule(sim, case: dict, on_checkpoint):
    """Drives any solver adapter through a case's step schedule.

    ``sim`` provides step(n), readback_field(), reset_from_field(field) and
    set_params(params_dict). ``on_checkpoint(step, field)`` is called after
    each segment of ``case["steps"]``. ``reverse_after`` flips the flow
    direction live (LbmSolver::SetParams) at that step count;
    ``reset_from_field_after`` re-seeds from the solver's own field at that
    checkpoint (the warm-start path, FlowCraft/main.cpp:1496-1565)."""
    done = 0
    rev_at = case.get("reverse_after")
    for seg in case["steps"]:
        target = done + seg
        while done < target:
            stop = target
            if rev_at is not None and done < rev_at < target:
                stop = rev_at
            sim.step(stop - done)
            done = stop
            if rev_at is not None and done == rev_at:
                p = dict(case["params"])
                p["reverse_flow"] = 1 - int(p.get("reverse_flow", 0))
                sim.set_params(p)
        field = sim.readback_field()
        on_checkpoint(done, field)
        if case.get("reset_from_field_after") == done:
            sim.reset_from_field(field)


class OracleAdapter:
    """Adapter over oracle.oracle.Oracle for run_schedule."""

    def __init__(self, case: dict, precision: str = "f32", threads: int = 0):
        from oracle.oracle import Oracle
        solid, sdf = geometry(case["geom"])
        self.o = Oracle(solid, sdf, case["q"], params_for(case), case["seed_mid"], precision, threads)
        self.case = case

    def step(self, n):
        self.o.step(n)

    def readback_field(self):
        return self.o.readback_field()

    def reset_from_field(self, field):
        self.o.reset_from_field(field)

    def set_params(self, p):
        c = dict(self.case)
        c["params"] = p
        self.o.set_params(params_for(c))

    def stats(self):
        return self.o.stats()


def load_fixture(name: str) -> dict:
    import json
    with open(os.path.join(GOLDEN_DIR, f"{name}.json")) as f:
        return json.load(f)
