"""Analytic solver geometry: the (solid, signedDistance) pair of FlowCraft's
VoxelGrid (FlowCraft/VoxelGrid.h:13-61) built from closed-form signed distance
functions instead of a triangle-mesh voxelization.

Conventions follow the reference exactly:
  * index (z*ny + y)*nx + x, arrays shaped (nz, ny, nx);
  * signedDistance > 0 in fluid, < 0 in solid (VoxelGrid.h:18-33);
  * solid = 1 where the distance at the cell centre (x+0.5, y+0.5, z+0.5) is
    negative, as in the reference's analytic test grids
    (tests/gpu_vs_cpu_test.cpp:28-41, :84-105).

Every builder works on numpy (CPU) arrays; ``aircraft_grid_torch`` builds the
large procedural aircraft directly on a CUDA device with torch, because a
268M-cell grid is far too slow to build cell-by-cell on the host.
"""
from __future__ import annotations

import math

import numpy as np


def _centres(nx: int, ny: int, nz: int):
    f32 = np.float32
    x = np.arange(nx, dtype=f32)[None, None, :] + f32(0.5)
    y = np.arange(ny, dtype=f32)[None, :, None] + f32(0.5)
    z = np.arange(nz, dtype=f32)[:, None, None] + f32(0.5)
    return x, y, z


def sphere_grid(nx: int, ny: int, nz: int, cx: float, cy: float, cz: float, r: float):
    """Sphere SDF d = |c_cell - c| - r in float32 (gpu_vs_cpu_test.cpp:32-41)."""
    f32 = np.float32
    x, y, z = _centres(nx, ny, nz)
    dx = x - f32(cx)
    dy = y - f32(cy)
    dz = z - f32(cz)
    d = np.sqrt(dx * dx + dy * dy + dz * dz) - f32(r)
    d = np.ascontiguousarray(d.astype(np.float32))
    return (d < 0).astype(np.uint8), d


def inclined_ellipsoid_wing_grid(nx=48, ny=32, nz=24, cx=20.0, cy=16.0, cz=12.0, angle=0.1745,
                                 semi=(7.0, 9.0, 2.2), scale=3.0, reverse=False):
    """The inclined ellipsoid 'wing' of tests/gpu_vs_cpu_test.cpp:84-105
    (+10 deg angle of attack, nose up toward the inlet); ``reverse`` gives the
    mirror pitch used for -X flow (:174-189)."""
    f32 = np.float32
    x, y, z = _centres(nx, ny, nz)
    ca, sa = f32(math.cos(angle)), f32(math.sin(angle))
    dx = x - f32(cx)
    dy = y - f32(cy)
    dz = z - f32(cz)
    if not reverse:
        rx = dx * ca - dz * sa
        rz = dx * sa + dz * ca
    else:
        rx = dx * ca + dz * sa
        rz = -dx * sa + dz * ca
    a, b, c = (f32(v) for v in semi)
    d = (np.sqrt((rx / a) * (rx / a) + (dy / b) * (dy / b) + (rz / c) * (rz / c)) - f32(1.0)) * f32(scale)
    d = np.ascontiguousarray(np.broadcast_to(d, (nz, ny, nx)).astype(np.float32))
    return (d < 0).astype(np.uint8), d


def naca4_half_thickness(xc, t, xp=np):
    """NACA 4-digit half thickness y_t(x/c) (closed trailing edge variant)."""
    return 5.0 * t * (0.2969 * xp.sqrt(xp.clip(xc, 0.0, 1.0)) - 0.1260 * xc - 0.3516 * xc ** 2
                      + 0.2843 * xc ** 3 - 0.1036 * xc ** 4)


def naca4_camber(xc, m, p, xp=np):
    """NACA 4-digit mean camber line y_c(x/c)."""
    if m == 0.0:
        return xc * 0.0
    xc = xp.clip(xc, 0.0, 1.0)
    front = m / (p * p) * (2 * p * xc - xc * xc)
    back = m / ((1 - p) ** 2) * ((1 - 2 * p) + 2 * p * xc - xc * xc)
    return xp.where(xc < p, front, back)


def _wing_sdf(px, py, pz, le_x, root_y, tip_y, z0, chord_root, taper, aoa_deg, m, p, t, xp):
    """Approximate signed distance to a straight tapered NACA wing with its
    span along +y from root_y to tip_y (|y| symmetric about root when
    tip_y < root_y is not used), flow along +x, angle of attack about y."""
    span = abs(tip_y - root_y)
    s = xp.clip((py - root_y) / (tip_y - root_y), 0.0, 1.0)
    chord = chord_root * (1.0 - (1.0 - taper) * s)
    a = math.radians(aoa_deg)
    ca, sa = math.cos(a), math.sin(a)
    # rotate about the quarter chord so positive AoA lifts the nose (toward -x)
    qx = le_x + 0.25 * chord
    rx = (px - qx) * ca - (pz - z0) * sa
    rz = (px - qx) * sa + (pz - z0) * ca
    xc = (rx + 0.25 * chord) / chord
    yt = naca4_half_thickness(xc, t, xp) * chord
    yc = naca4_camber(xc, m, p, xp) * chord
    inside_chord = (xc >= 0.0) & (xc <= 1.0)
    d_thick = xp.abs(rz - yc) - yt
    d_chord = xp.maximum(-xc, xc - 1.0) * chord
    d_section = xp.where(inside_chord, d_thick, xp.maximum(d_chord, xp.abs(rz - yc)))
    lo, hi = min(root_y, tip_y), max(root_y, tip_y)
    d_span = xp.maximum(lo - py, py - hi)
    # exterior combination (exact for box-like unions, approximate here)
    out_sec = xp.clip(d_section, 0.0, None)
    out_span = xp.clip(d_span, 0.0, None)
    outside = xp.sqrt(out_sec * out_sec + out_span * out_span)
    inside = xp.clip(xp.maximum(d_section, d_span), None, 0.0)
    del span
    return outside + inside


def naca_wing_grid(nx, ny, nz, chord, span, aoa_deg, digits="0012", le_x=None, xp=np, device=None):
    """Extruded NACA 4-digit wing (span along grid y, centred), an analytic
    stand-in for a triangulated, voxelized wing. Works with numpy or torch."""
    m = int(digits[0]) / 100.0
    p = int(digits[1]) / 10.0
    t = int(digits[2:]) / 100.0
    if le_x is None:
        le_x = 0.25 * nx
    if xp is np:
        x, y, z = _centres(nx, ny, nz)
    else:
        x = (xp.arange(nx, device=device, dtype=xp.float32) + 0.5)[None, None, :]
        y = (xp.arange(ny, device=device, dtype=xp.float32) + 0.5)[None, :, None]
        z = (xp.arange(nz, device=device, dtype=xp.float32) + 0.5)[:, None, None]
    y0 = 0.5 * ny - 0.5 * span
    d = _wing_sdf(x, y, z, le_x, y0, y0 + span, 0.5 * nz, chord, 1.0, aoa_deg, m, p, t, xp)
    if xp is np:
        d = np.ascontiguousarray(np.broadcast_to(d, (nz, ny, nx)).astype(np.float32))
        return (d < 0).astype(np.uint8), d
    d = d.expand(nz, ny, nx).contiguous().float()
    return (d < 0).to(xp.uint8), d


def _ellipsoid_sdf(px, py, pz, c, semi, xp):
    # scaled-distance approximation (exact on the surface, monotone off it)
    rx, ry, rz = semi
    k = xp.sqrt(((px - c[0]) / rx) ** 2 + ((py - c[1]) / ry) ** 2 + ((pz - c[2]) / rz) ** 2)
    return (k - 1.0) * min(semi)


def aircraft_grid_torch(nx=1024, ny=512, nz=512, device="cuda", z_chunk=32, z_lo=0, z_hi=None):
    """Procedural high-wing aircraft on a 1024x512x512 lattice: ellipsoidal
    fuselage (length 0.39*nx = 400 cells at nx=1024), a tapered NACA 2412 wing
    (span 360, root chord 60, taper 0.6) mounted on top, a NACA 0012
    horizontal tail and vertical fin. Returns (solid u8, sdf f32) torch tensors
    shaped (nz, ny, nx) on ``device`` — or only layers [z_lo, z_hi) of it.
    Built in z-chunks to bound temporaries."""
    import torch

    sx = nx / 1024.0
    fus_len = 400.0 * sx
    fus_r = 0.06 * fus_len * 1.6
    x0 = 0.30 * nx
    cy = 0.5 * ny
    cz = 0.5 * nz
    z_hi = nz if z_hi is None else min(z_hi, nz)
    solid = torch.empty((z_hi - z_lo, ny, nx), dtype=torch.uint8, device=device)
    sdf = torch.empty((z_hi - z_lo, ny, nx), dtype=torch.float32, device=device)
    x = (torch.arange(nx, device=device, dtype=torch.float32) + 0.5)[None, None, :]
    y = (torch.arange(ny, device=device, dtype=torch.float32) + 0.5)[None, :, None]
    half_span = 180.0 * sx
    root_c = 60.0 * sx
    wing_le = x0 + 0.30 * fus_len
    wing_z = cz + 0.8 * fus_r
    tail_le = x0 + 0.86 * fus_len
    for z0 in range(z_lo, z_hi, z_chunk):
        z1 = min(z_hi, z0 + z_chunk)
        z = (torch.arange(z0, z1, device=device, dtype=torch.float32) + 0.5)[:, None, None]
        d = _ellipsoid_sdf(x, y, z, (x0 + 0.5 * fus_len, cy, cz), (0.5 * fus_len, fus_r, fus_r), torch)
        for side in (+1.0, -1.0):
            w = _wing_sdf(x, y, z, wing_le, cy, cy + side * half_span, wing_z, root_c, 0.6, 2.0,
                          0.02, 0.4, 0.12, torch)
            d = torch.minimum(d, w)
            ht = _wing_sdf(x, y, z, tail_le, cy, cy + side * 0.35 * half_span, cz, 0.5 * root_c, 0.7, 0.0,
                           0.0, 0.0, 0.12, torch)
            d = torch.minimum(d, ht)
        # vertical fin: the same section rotated to span along +z
        fin = _wing_sdf(x, z, y, tail_le, cz, cz + 0.5 * half_span, cy, 0.6 * root_c, 0.6, 0.0,
                        0.0, 0.0, 0.12, torch)
        d = torch.minimum(d, fin)
        d = d.expand(z1 - z0, ny, nx)
        sdf[z0 - z_lo:z1 - z_lo] = d
        solid[z0 - z_lo:z1 - z_lo] = (d < 0).to(torch.uint8)
    return solid, sdf
