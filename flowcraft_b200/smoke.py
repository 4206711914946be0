"""SmokeTrailSystem (FlowCraft/SmokeTrail.h:26-184) on the device.

The reference keeps its particles on the host and samples the velocity from
a full 4-float field readback every frame (SmokeTrail.cpp:278-343). Here the
particles and their trails live in device memory next to the solver's
populations and every Step samples the velocity there; only the trails come
back to the host, on request (Trails()), for whatever draws them. BuildMesh
(the camera-facing trail quads) is rendering and stays with the caller.

Method names and argument meanings follow the reference. Step takes the
solver instead of the (grid, field) pair: the field is the solver's own
current state.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from .lbm import LbmSolver

X, Y, Z = 0, 1, 2  # SliceAxis (FieldOverlay.h:24)


@dataclass
class PlaneConfinement:
    """SmokeTrailSystem::PlaneConfinement (SmokeTrail.h:44-47): a grid axis
    (X, Y, Z) and the index of the plane along it."""
    axis: int
    index: int


def _conf(c: PlaneConfinement | None):
    return (-1, 0) if c is None else (int(c.axis), int(c.index))


class SmokeTrailSystem:
    def __init__(self, solver: LbmSolver):
        self.s = solver
        self._lib = solver._lib
        self._count = 0
        self._length = 0

    def _check(self, rc, what):
        self.s._check(rc, what)

    def Reset(self, reverseFlow: bool, particleCount: int, trailLength: int,
              confine: PlaneConfinement | None = None, seed: int = 12345) -> None:
        """Every particle to a random point of the domain (or plane), trails
        of max(trailLength, 2) points (SmokeTrail.cpp:257-276). reverseFlow is
        accepted and unused, as in the reference."""
        del reverseFlow
        a, i = _conf(confine)
        self._check(self._lib.fc_lbm_particles_reset(self.s._h, int(particleCount), int(trailLength), int(seed), a, i),
                    "particles Reset")
        self._count = max(int(particleCount), 0)
        self._length = max(int(trailLength), 2)

    def Step(self, reverseFlow: bool, mmPerSecPerLatticeUnit: float, dtSeconds: float,
             suspendRespawn: bool = False, confine: PlaneConfinement | None = None) -> None:
        a, i = _conf(confine)
        self._check(self._lib.fc_lbm_particles_step(self.s._h, int(bool(reverseFlow)), float(mmPerSecPerLatticeUnit),
                                                    float(dtSeconds), int(bool(suspendRespawn)), a, i),
                    "particles Step")

    def ScatterRandom(self, confine: PlaneConfinement | None = None) -> None:
        a, i = _conf(confine)
        self._check(self._lib.fc_lbm_particles_scatter(self.s._h, a, i), "particles ScatterRandom")

    def ShiftPlane(self, confine: PlaneConfinement) -> None:
        self._check(self._lib.fc_lbm_particles_shift_plane(self.s._h, int(confine.axis), int(confine.index)),
                    "particles ShiftPlane")

    def SetPositions(self, points) -> None:
        """Every particle to one given point (count x 3, world units)."""
        pts = np.ascontiguousarray(np.asarray(points, dtype=np.float32).reshape(-1))
        self._check(self._lib.fc_lbm_particles_set(self.s._h, pts.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                                    pts.size), "particles SetPositions")

    def Trails(self):
        """(points[count, length, 3] oldest first, lens[count])."""
        out = np.zeros((self._count, self._length, 3), dtype=np.float32)
        lens = np.zeros(self._count, dtype=np.int32)
        self._check(self._lib.fc_lbm_particles_read(self.s._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                                    out.size, lens.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                                    lens.size), "particles Trails")
        return out, lens

    def Heads(self) -> np.ndarray:
        """The newest point of every active particle (NaN rows for inactive)."""
        pts, lens = self.Trails()
        head = np.full((self._count, 3), np.nan, dtype=np.float32)
        act = lens > 0
        head[act] = pts[np.nonzero(act)[0], lens[act] - 1]
        return head
