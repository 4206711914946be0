"""Analytic geometry builders follow VoxelGrid's conventions
(FlowCraft/VoxelGrid.h): index (z*ny+y)*nx+x, SDF positive in fluid."""
import numpy as np

from flowcraft_b200.geometry import inclined_ellipsoid_wing_grid, naca_wing_grid, sphere_grid


def test_sphere_sign_and_layout():
    solid, sdf = sphere_grid(48, 24, 24, 20, 12, 12, 5)
    assert solid.shape == (24, 24, 48) and sdf.dtype == np.float32
    assert ((sdf < 0) == solid.astype(bool)).all()
    # centre cell (x=19..20, y=11..12, z=11..12) is solid; corners are fluid
    assert solid[11, 11, 19] == 1 and solid[0, 0, 0] == 0
    vol = solid.sum()
    assert abs(vol - 4 / 3 * np.pi * 125) / (4 / 3 * np.pi * 125) < 0.1


def test_wing_is_inclined_nose_up():
    solid, sdf = inclined_ellipsoid_wing_grid()
    assert solid.shape == (24, 32, 48) and solid.sum() > 100
    zs, ys, xs = np.nonzero(solid)
    # leading edge (small x) sits higher than the trailing edge: nose up
    lead = zs[xs <= xs.min() + 2].mean()
    trail = zs[xs >= xs.max() - 2].mean()
    assert lead > trail


def test_naca_wing_numpy():
    solid, sdf = naca_wing_grid(96, 48, 48, chord=40, span=30, aoa_deg=4, digits="0012")
    assert solid.shape == (48, 48, 96) and solid.sum() > 0
    assert ((sdf < 0) == solid.astype(bool)).all()
    t = solid.sum(axis=(0, 1))
    assert t[:20].sum() == 0 and t[-20:].sum() == 0  # wing sits inside the box
