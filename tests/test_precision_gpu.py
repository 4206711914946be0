"""The precision study's error bounds at reduced size: the NACA 0012 wing of
the 384x192x192 precision configuration at quarter size (96x48x48, chord 24,
span 32, 4 deg), U 0.06, Cs 0.1, 600 steps from the mid-speed seed, on
D3Q19 at the full-size case's viscosity (tau 0.50173) and on D3Q15 at the
study's tau for D3Q15 (0.6: D3Q15 does not hold the lower viscosity). FP32,
FP16-offset and BF16-offset storage on the GPU against
the FP64 oracle: maximum density and speed errors over the fluid cells, and
the drag and lift coefficients of the last step, whose errors are measured
in units of the drag coefficient (the D3Q19 wing carries almost no lift
600 steps after the start, so a lift error relative to the lift would
measure nothing). The bounds hold the measured errors with a margin of
about 3. BF16 storage does not hold the D3Q19 lift at this viscosity
(8 mantissa bits of (f - w) 2^8 at tau - 1/2 = 0.0017; the full-size study
shows the same), so its lift is not bounded there."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

sys.path.insert(0, os.path.dirname(__file__))

NX, NY, NZ, CHORD, SPAN, AOA, U, STEPS = 96, 48, 48, 24.0, 32.0, 4.0, 0.06, 600
TAU = 0.5 + 3.0 * U * 96.0 / 1e4

# (max |drho|, max | |u| error |, |dCd| / Cd, |dCl| / Cd) against FP64
BOUNDS = {
    "FP32": (2e-5, 2e-5, 5e-4, 5e-4),
    "FP16_OFFSET": (1e-3, 1.5e-3, 1e-2, 2e-2),
    "BF16_OFFSET": (1e-2, 1e-2, 1e-1, 1e-1),
}


def _geometry():
    from flowcraft_b200 import geometry as geo
    solid, sdf = geo.naca_wing_grid(NX, NY, NZ, chord=CHORD, span=SPAN, aoa_deg=AOA, digits="0012")
    return np.ascontiguousarray(solid, np.uint8), np.ascontiguousarray(sdf, np.float32)


def _coeffs(force):
    q = 0.5 * U * U * CHORD * SPAN
    return force[0] / q, force[2] / q


@pytest.fixture(scope="module")
def fp64_runs(oracle_built):
    from precision_study import D3Q15_CS, D3Q15_TAU, D3Q19_CS
    solid, sdf = _geometry()
    out = {}
    for q, cs, tau in ((19, D3Q19_CS, TAU), (15, D3Q15_CS, D3Q15_TAU)):
        p = oracle_built.Params(tau, U, False, True, True, cs)
        o = oracle_built.Oracle(solid, sdf, q, p, seed_mid=True, precision="f64")
        o.step(STEPS)
        f = o.readback_field_f64().reshape(-1, 4)
        assert not o.has_diverged()
        o.close()
        out[q] = (f, cs, tau)
    return solid, sdf, out


@pytest.mark.parametrize("q", [19, 15])
@pytest.mark.parametrize("storage", ["FP32", "FP16_OFFSET", "BF16_OFFSET"])
def test_storage_error_vs_fp64_on_the_precision_wing(gpu, fp64_runs, q, storage):
    from flowcraft_b200.lbm import LatticeModel, LbmSolver, Params, Storage, VoxelGrid
    solid, sdf, ref = fp64_runs
    r, cs, tau = ref[q]
    s = LbmSolver()
    assert s.Init(0, VoxelGrid(NX, NY, NZ, solid=solid.ravel(), signedDistance=sdf.ravel()),
                  LatticeModel.D3Q19 if q == 19 else LatticeModel.D3Q15, Storage[storage]), s.LastError()
    s.Reset(Params(tau=tau, inletVelocity=U, smagorinskyCs=cs), True)
    s.Step(None, STEPS)
    g = s.ReadbackField().reshape(-1, 4).astype(np.float64)
    assert not s.HasDiverged()
    s.close()
    sol = solid.ravel().astype(bool)
    fl = ~sol
    drho = np.abs(g[fl, 0] - r[fl, 0]).max()
    du = np.abs(np.linalg.norm(g[fl, 1:], axis=1) - np.linalg.norm(r[fl, 1:], axis=1)).max()
    cd, cl = _coeffs(g[sol][:, 1:4].sum(axis=0))
    rcd, rcl = _coeffs(r[sol][:, 1:4].sum(axis=0))
    dcd, dcl = abs(cd - rcd) / rcd, abs(cl - rcl) / rcd
    print(f"D3Q{q} {storage}: max|drho| {drho:.2e} max|du| {du:.2e} dCd {dcd:.2e} dCl {dcl:.2e} "
          f"(Cd {rcd:.4f} Cl {rcl:.4f})")
    b = BOUNDS[storage]
    assert drho < b[0] and du < b[1]
    assert dcd < b[2]
    if not (storage == "BF16_OFFSET" and q == 19):
        assert dcl < b[3]
