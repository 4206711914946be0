"""Voxelizer test cases: procedural meshes (flowcraft_b200/meshes.py) and the
grids they are voxelized on.

``GOLDEN`` cases run Voxelizer::Voxelize's own grid derivation (target
resolution and padding, Voxelizer.cpp:146-166) and have fixtures made by the
reference voxelizer itself (make_voxel_golden.py). ``EXPLICIT`` cases put a
mesh on a chosen grid (cell size, origin, dims) to reach the edge cases the
derived grid never produces: a seed cell inside the model, a seed cell on the
surface shell, a triangle soup with degenerate and out-of-grid triangles,
inward winding, and no triangles at all. Those are checked against the
oracle, which the golden cases pin to the reference.
"""
from __future__ import annotations

import hashlib

import numpy as np

from flowcraft_b200 import meshes


def _cavity():
    op, oi = meshes.icosphere(3, 10.0)
    ip, ii = meshes.icosphere(2, 6.0)
    return meshes.merge((op, oi), (ip, ii.reshape(-1, 3)[:, [0, 2, 1]].ravel()))


def _soup(seed=7, count=300):
    rng = np.random.default_rng(seed)
    centres = rng.uniform(-8.0, 8.0, size=(count, 1, 3))
    tri = centres + rng.normal(0.0, 1.5, size=(count, 3, 3))
    tri[::17, 2] = tri[::17, 1]          # zero-area triangles (two equal corners)
    tri[5::23] += 1.0e4                  # triangles far outside the grid
    pos = tri.reshape(-1, 3).astype(np.float32)
    return pos, np.arange(len(pos), dtype=np.uint32)


def _inward():
    p, i = meshes.icosphere(3, 9.0)
    return p, i.reshape(-1, 3)[:, [0, 2, 1]].ravel()


MESHES = {
    "icosphere": lambda: meshes.icosphere(3, 10.0, (5.0, 7.0, -3.0)),
    "naca0012": lambda: meshes.naca_wing("0012", 40.0, 50.0, 4.0, 32, 8),
    "naca2412_taper": lambda: meshes.naca_wing("2412", 30.0, 60.0, 6.0, 32, 10, taper=0.6),
    "aircraft_small": lambda: meshes.aircraft(100.0, 90.0, 15.0, 0.6, n_chord=24, n_span=24, fuselage_res=(48, 24)),
    "aircraft": lambda: meshes.aircraft(),
    "cavity": _cavity,
    "c1_sphere": lambda: meshes.icosphere(3, 10.0, (32.0, 40.0, 32.0)),
    "soup": _soup,
    "inward": _inward,
}

GOLDEN = {
    "icosphere_r48": dict(mesh="icosphere", res=48),
    "icosphere_r96": dict(mesh="icosphere", res=96),
    "naca0012_r96": dict(mesh="naca0012", res=96),
    "naca2412_taper_r96": dict(mesh="naca2412_taper", res=96),
    "aircraft_small_r96": dict(mesh="aircraft_small", res=96),
    "cavity_r80": dict(mesh="cavity", res=80),
    "aircraft_r256": dict(mesh="aircraft", res=256),
    "icosphere_r64_nopad": dict(mesh="icosphere", res=64, padding=(0.0, 0.0, 0.0)),
}

# (mesh, dims (nx, ny, nz), cell size, origin)
EXPLICIT = {
    # the c1 benchmark obstacle: radius 10 at grid (40, 32, 32) of 128x64x64
    "c1_sphere_128x64x64": dict(mesh="c1_sphere", dims=(128, 64, 64), cell=1.0, origin=(0.0, 0.0, 0.0)),
    # seed cell (0,0,0) inside the sphere: the interior is the reached component
    "seed_inside": dict(mesh="icosphere", dims=(24, 20, 22), cell=0.75, origin=(5.0, 7.0, -3.0)),
    # seed cell on the surface shell: nothing is reached, every cell ends solid
    "seed_on_shell": dict(mesh="icosphere", dims=(20, 20, 20), cell=1.0, origin=(-1.27, 0.73, -9.27)),
    "soup": dict(mesh="soup", dims=(40, 36, 34), cell=0.5, origin=(-10.0, -9.0, -8.5)),
    "inward": dict(mesh="inward", dims=(30, 30, 30), cell=0.7, origin=(-10.5, -10.5, -10.5)),
    "ragged_tiles": dict(mesh="naca2412_taper", dims=(37, 75, 13), cell=0.9, origin=(-31.0, -4.0, -6.0)),
}


def mesh(name):
    pos, idx = MESHES[name]()
    return np.ascontiguousarray(pos, dtype=np.float32), np.ascontiguousarray(idx, dtype=np.uint32)


def digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def mesh_digest(pos, idx) -> str:
    return hashlib.sha256(pos.tobytes() + idx.tobytes()).hexdigest()
