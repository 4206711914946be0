"""ORACLE — test infrastructure only, never the product path.

A numpy restatement of FlowCraft's smoke-trail advection
(FlowCraft/SmokeTrail.cpp) for particles that stay in the fluid: CellAt
(:36-61), SampleVelocityInterpolated (:69-116) and the position update of
SmokeTrailSystem::Step (:278-343), in float32 with one rounding per
operation (the reference is built without contraction). Respawns are random
in the reference; this restatement only reports which particles would
respawn. `step_reference` runs the reference's own class through
oracle/_ref (the pin for the restatement).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
f32 = np.float32


def _cell_at(p, origin, cs, dims):
    """Grid cell of world point p (grid x from world y, grid y from world x)."""
    nx, ny, nz = dims
    lx, ly, lz = f32(p[0]) - f32(origin[0]), f32(p[1]) - f32(origin[1]), f32(p[2]) - f32(origin[2])
    x, y, z = int(np.floor(ly / f32(cs))), int(np.floor(lx / f32(cs))), int(np.floor(lz / f32(cs)))
    return (x, y, z), (0 <= x < nx and 0 <= y < ny and 0 <= z < nz)


def sample_velocity(field, solid, dims, cs, origin, p):
    """SampleVelocityInterpolated: world velocity at world point p."""
    nx, ny, nz = dims
    fl = field.reshape(-1, 4)
    sd = solid.reshape(-1)
    lx, ly, lz = f32(p[0]) - f32(origin[0]), f32(p[1]) - f32(origin[1]), f32(p[2]) - f32(origin[2])
    gxf = ly / f32(cs) - f32(0.5)
    gyf = lx / f32(cs) - f32(0.5)
    gzf = lz / f32(cs) - f32(0.5)
    gx0, gy0, gz0 = int(np.floor(gxf)), int(np.floor(gyf)), int(np.floor(gzf))
    tx, ty, tz = gxf - f32(gx0), gyf - f32(gy0), gzf - f32(gz0)

    def s(x, y, z):
        x, y, z = min(max(x, 0), nx - 1), min(max(y, 0), ny - 1), min(max(z, 0), nz - 1)
        c = (z * ny + y) * nx + x
        if sd[c]:
            return np.zeros(3, dtype=f32)
        return np.array([fl[c, 2], fl[c, 1], fl[c, 3]], dtype=f32)

    def lerp(a, b, t):
        return a + (b - a) * f32(t)

    c00 = lerp(s(gx0, gy0, gz0), s(gx0 + 1, gy0, gz0), tx)
    c10 = lerp(s(gx0, gy0 + 1, gz0), s(gx0 + 1, gy0 + 1, gz0), tx)
    c01 = lerp(s(gx0, gy0, gz0 + 1), s(gx0 + 1, gy0, gz0 + 1), tx)
    c11 = lerp(s(gx0, gy0 + 1, gz0 + 1), s(gx0 + 1, gy0 + 1, gz0 + 1), tx)
    c0 = lerp(c00, c10, ty)
    c1 = lerp(c01, c11, ty)
    return lerp(c0, c1, tz)


def advect(field, solid, dims, cs, origin, positions, steps, mm_per_sec, dt, confine_axis=-1):
    """Trails (count, steps + 1, 3) of particles starting at `positions`, and
    a mask of the particles that stayed in the fluid all along (the others
    would have respawned in the reference)."""
    sd = solid.reshape(-1)
    nx, ny, nz = dims
    dt = min(f32(dt), f32(0.1))
    scale = f32(mm_per_sec) * f32(dt)
    pos = np.array(positions, dtype=f32).reshape(-1, 3)
    out = np.zeros((pos.shape[0], steps + 1, 3), dtype=f32)
    ok = np.ones(pos.shape[0], dtype=bool)
    for p in range(pos.shape[0]):
        cur = pos[p].copy()
        out[p, 0] = cur
        for k in range(steps):
            (x, y, z), inb = _cell_at(cur, origin, cs, dims)
            if not inb or sd[(z * ny + y) * nx + x]:
                ok[p] = False
                break
            v = sample_velocity(field, solid, dims, cs, origin, cur)
            if confine_axis == 0:
                v[1] = f32(0)
            elif confine_axis == 1:
                v[0] = f32(0)
            elif confine_axis == 2:
                v[2] = f32(0)
            cur = cur + v * scale
            out[p, k + 1] = cur
    return out, ok


def step_reference(solid, field, dims, cs, origin, positions, trail_length, steps, mm_per_sec, dt, reverse=False,
                   confine_axis=-1, confine_index=0):
    """The reference's SmokeTrailSystem::Step, `steps` times, from the given
    positions: (trails (count, trail_length, 3) oldest first, lens)."""
    lib = ctypes.CDLL(os.path.join(HERE, "_ref", "libfcref.so"))
    fn = lib.ref_smoke_step
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_int] * 3 + [ctypes.c_float] + [ctypes.c_void_p] * 3 + [ctypes.c_int, ctypes.c_int,
                   ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_int,
                   ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    nx, ny, nz = dims
    sd = np.ascontiguousarray(solid, dtype=np.uint8).reshape(-1)
    fl = np.ascontiguousarray(field, dtype=np.float32).reshape(-1)
    org = np.ascontiguousarray(origin, dtype=np.float32)
    pos = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1)
    count = pos.size // 3
    out = np.zeros((count, trail_length, 3), dtype=np.float32)
    lens = np.zeros(count, dtype=np.int32)
    fn(nx, ny, nz, float(cs), org.ctypes.data, sd.ctypes.data, fl.ctypes.data, count, int(trail_length),
       pos.ctypes.data, int(steps), int(reverse), float(mm_per_sec), float(dt), int(confine_axis), int(confine_index),
       out.ctypes.data, lens.ctypes.data)
    return out, lens


def reference_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libfcref.so"))
