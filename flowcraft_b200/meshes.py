"""Procedural triangle meshes for the voxelizer: the shapes the benchmark
configurations describe (there are no mesh files for them).

All meshes are returned as (positions float32 (V, 3), indices uint32 (T*3,))
in world coordinates with outward (counter-clockwise) winding, like the
output of FlowCraft's STL loader (FlowCraft/Mesh.h). The flow axis is
world y, which the voxel grid maps to grid x (FlowCraft/VoxelGrid.h:43-56).

* ``icosphere(level)``: a subdivided icosahedron; level 3 has 1280
  triangles.
* ``naca_wing(...)``: an extruded or tapered NACA 4-digit wing with flat end
  caps, chord along world y, span along world x, at an angle of attack about
  the span axis.
* ``aircraft(...)``: an ellipsoidal fuselage, a tapered NACA 2412 high wing and
  NACA 0012 horizontal and vertical tails.
"""
from __future__ import annotations

import math

import numpy as np


def icosphere(level: int = 3, radius: float = 1.0, center=(0.0, 0.0, 0.0)):
    t = (1.0 + math.sqrt(5.0)) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [np.array(v, dtype=np.float64) / np.linalg.norm(v) for v in verts]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
             (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(level):
        cache = {}

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    pos = np.array(verts) * radius + np.asarray(center, dtype=np.float64)
    return pos.astype(np.float32), np.array(faces, dtype=np.uint32).ravel()


def naca4_section(digits: str, n: int = 64):
    """Closed NACA 4-digit section as (x/c, y/c) points, counter-clockwise
    from the trailing edge over the upper surface (cosine spacing)."""
    m = int(digits[0]) / 100.0
    p = int(digits[1]) / 10.0
    t = int(digits[2:]) / 100.0
    beta = np.linspace(0.0, math.pi, n)
    x = 0.5 * (1.0 - np.cos(beta))
    yt = 5 * t * (0.2969 * np.sqrt(x) - 0.1260 * x - 0.3516 * x ** 2 + 0.2843 * x ** 3 - 0.1036 * x ** 4)
    if m > 0:
        yc = np.where(x < p, m / p ** 2 * (2 * p * x - x ** 2), m / (1 - p) ** 2 * ((1 - 2 * p) + 2 * p * x - x ** 2))
        dyc = np.where(x < p, 2 * m / p ** 2 * (p - x), 2 * m / (1 - p) ** 2 * (p - x))
    else:
        yc = np.zeros_like(x)
        dyc = np.zeros_like(x)
    th = np.arctan(dyc)
    xu, yu = x - yt * np.sin(th), yc + yt * np.cos(th)
    xl, yl = x + yt * np.sin(th), yc - yt * np.cos(th)
    # upper surface trailing edge -> leading edge, then lower leading -> trailing
    xs = np.concatenate([xu[::-1], xl[1:-1]])
    ys = np.concatenate([yu[::-1], yl[1:-1]])
    return np.stack([xs, ys], axis=1)


def _loft(sections, caps=True):
    """Triangulates a list of closed rings (K, P, 3) into a closed surface."""
    sections = np.asarray(sections)
    k, pcount, _ = sections.shape
    pos = sections.reshape(-1, 3)
    tris = []
    for s in range(k - 1):
        for j in range(pcount):
            a = s * pcount + j
            b = s * pcount + (j + 1) % pcount
            c = (s + 1) * pcount + (j + 1) % pcount
            d = (s + 1) * pcount + j
            tris += [(a, b, c), (a, c, d)]
    extra = [pos]
    if caps:
        base = len(pos)
        for s, flip in ((0, True), (k - 1, False)):
            centre = sections[s].mean(axis=0)
            extra.append(centre[None, :])
            ci = base
            base += 1
            for j in range(pcount):
                a = s * pcount + j
                b = s * pcount + (j + 1) % pcount
                tris.append((ci, b, a) if flip else (ci, a, b))
    pos = np.concatenate(extra, axis=0)
    tri = np.asarray(tris, dtype=np.uint32)
    # orient outward: flip all if the signed volume is negative
    v0, v1, v2 = pos[tri[:, 0]], pos[tri[:, 1]], pos[tri[:, 2]]
    vol = np.einsum("ij,ij->i", v0, np.cross(v1, v2)).sum()
    if vol < 0:
        tri = tri[:, [0, 2, 1]]
    return pos, tri


def naca_wing(digits="0012", chord=96.0, span=128.0, aoa_deg=4.0, n_chord=64, n_span=16, root=(0.0, 0.0, 0.0),
              taper=1.0, half=False):
    """Wing with chord along +y (the flow axis), span along x, nose at
    root.y, pitched nose-up by aoa_deg about the quarter chord."""
    sec = naca4_section(digits, n_chord)
    a = math.radians(aoa_deg)
    rings = []
    xs = np.linspace(0.0, span, n_span + 1) if half else np.linspace(-0.5 * span, 0.5 * span, n_span + 1)
    for xspan in xs:
        frac = abs(xspan) / (span if half else 0.5 * span)
        c = chord * (1.0 - (1.0 - taper) * frac)
        yy = (sec[:, 0] - 0.25) * c
        zz = sec[:, 1] * c
        # nose-up pitch: the leading edge (y < 0 relative to the quarter chord) moves up
        yr = yy * math.cos(a) + zz * math.sin(a)
        zr = -yy * math.sin(a) + zz * math.cos(a)
        ring = np.stack([np.full_like(yr, xspan), yr + 0.25 * c, zr], axis=1) + np.asarray(root)
        rings.append(ring)
    pos, tri = _loft(rings)
    return pos.astype(np.float32), tri.ravel().astype(np.uint32)


def _ellipsoid(center, semi, n_u=96, n_v=48):
    """UV ellipsoid with its long axis along y."""
    tris, pos = [], []
    cy, cx, cz = center[1], center[0], center[2]
    ry, rx, rz = semi[1], semi[0], semi[2]
    pos.append((cx, cy - ry, cz))
    for i in range(1, n_v):
        th = math.pi * i / n_v
        for j in range(n_u):
            ph = 2 * math.pi * j / n_u
            pos.append((cx + rx * math.sin(th) * math.cos(ph), cy - ry * math.cos(th), cz + rz * math.sin(th) * math.sin(ph)))
    pos.append((cx, cy + ry, cz))
    last = len(pos) - 1
    for j in range(n_u):
        tris.append((0, 1 + (j + 1) % n_u, 1 + j))
    for i in range(n_v - 2):
        for j in range(n_u):
            a = 1 + i * n_u + j
            b = 1 + i * n_u + (j + 1) % n_u
            c = 1 + (i + 1) * n_u + (j + 1) % n_u
            d = 1 + (i + 1) * n_u + j
            tris += [(a, b, c), (a, c, d)]
    base = 1 + (n_v - 2) * n_u
    for j in range(n_u):
        tris.append((last, base + j, base + (j + 1) % n_u))
    pos = np.asarray(pos, dtype=np.float64)
    tri = np.asarray(tris, dtype=np.uint32)
    v0, v1, v2 = pos[tri[:, 0]], pos[tri[:, 1]], pos[tri[:, 2]]
    if np.einsum("ij,ij->i", v0 - pos.mean(0), np.cross(v1 - v0, v2 - v0)).sum() < 0:
        tri = tri[:, [0, 2, 1]]
    return pos, tri


def merge(*parts):
    pos, tri, base = [], [], 0
    for p, t in parts:
        pos.append(np.asarray(p, dtype=np.float64))
        tri.append(np.asarray(t, dtype=np.int64).reshape(-1, 3) + base)
        base += len(p)
    return np.concatenate(pos).astype(np.float32), np.concatenate(tri).astype(np.uint32).ravel()


def aircraft(fuselage_length=400.0, span=360.0, root_chord=60.0, taper=0.6, center=(0.0, 0.0, 0.0),
             n_chord=96, n_span=96, fuselage_res=(192, 96)):
    """Procedural high-wing aircraft, nose toward -y (facing the inflow)."""
    cx, cy, cz = center
    fr = 0.096 * fuselage_length
    fus = _ellipsoid((cx, cy, cz), (fr, 0.5 * fuselage_length, fr), *fuselage_res)
    wing_y = cy - 0.5 * fuselage_length + 0.30 * fuselage_length
    wing_z = cz + 0.8 * fr
    wing = naca_wing("2412", root_chord, span, 2.0, n_chord, n_span, root=(cx, wing_y, wing_z), taper=taper)
    tail_y = cy - 0.5 * fuselage_length + 0.86 * fuselage_length
    htail = naca_wing("0012", 0.5 * root_chord, 0.35 * span, 0.0, n_chord // 2, n_span // 3, root=(cx, tail_y, cz),
                      taper=0.7)
    # vertical fin: the same construction rotated so the span runs along +z
    fpos, ftri = naca_wing("0012", 0.6 * root_chord, 0.25 * span, 0.0, n_chord // 2, n_span // 4,
                           root=(0.0, 0.0, 0.0), taper=0.6, half=True)
    fpos = fpos.astype(np.float64)
    fin = np.stack([fpos[:, 2] + cx, fpos[:, 1] + tail_y, fpos[:, 0] + cz + 0.5 * fr], axis=1)
    ftri = ftri.reshape(-1, 3)[:, [0, 2, 1]]  # the axis swap mirrors the winding
    return merge(fus, (wing[0], wing[1]), (htail[0], htail[1]), (fin, ftri))


# The large configuration's aircraft: fuselage 400 cells long, wing span 360,
# root chord 60 (taper 0.6), tessellated to 57,516 triangles, placed on a
# 1024x512x512 lattice (scaled with nx) with the nose at 0.30 nx and the
# fuselage axis on the lattice's y and z centre lines.
C5_TESSELLATION = dict(n_chord=72, n_span=72, fuselage_res=(176, 88))


def aircraft_c5(nx: int = 1024):
    """(positions, indices) of the large configuration's aircraft mesh in
    lattice units for an nx-long lattice (world y is the flow axis)."""
    s = nx / 1024.0
    return aircraft(fuselage_length=400.0 * s, span=360.0 * s, root_chord=60.0 * s, **C5_TESSELLATION)


def aircraft_c5_origin(nx: int = 1024, ny: int = 512, nz: int = 512, z_lo: int = 0):
    """World origin of the grid (cell size 1) that puts aircraft_c5(nx) where
    the configuration places it. Cell (x, y, z) has its centre at world
    (ox + y + 0.5, oy + x + 0.5, oz + z + 0.5) (grid x spans world y); the
    fuselage centre sits at lattice coordinate (0.30 nx + 200 s, ny / 2,
    nz / 2), s = nx / 1024, rounded to whole cells so that every cell centre
    is exact in float (a grid over any sub-box then computes the same
    centres). `z_lo`: origin of a slab whose first layer is lattice layer
    z_lo."""
    s = nx / 1024.0
    return (-float(ny // 2), -float(round(0.30 * nx + 200.0 * s)), -float(nz // 2) + z_lo)
