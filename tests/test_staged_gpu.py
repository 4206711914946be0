"""The interior rows staged in shared memory by TMA tensor copies
(k_bulk_tiles, fc_options.flags = FC_OPTION_TMA_STAGING) against the direct
pair kernel (the default) and against the FP64 oracle.

The staged kernel (16-bit formats) reads the same stored values and runs the
same pair and one-cell collisions, so it must give bit-identical populations;
FP32 lattices keep the unstaged path, which the same comparison covers."""
import numpy as np
import pytest

from cases import OracleAdapter, geometry

pytestmark = pytest.mark.gpu

# (nx, ny, nz), sphere (cx, cy, cz, r), params: several interior chunks per
# row, a single one (nx = 136), walls cutting interior rows, both flow
# directions, every slip setting; the last sphere's rows end on both sides of
# the chunk edge x = 128, so one-cell updates read the halo columns
LATTICES = [
    ((320, 36, 30), (90.0, 18.0, 15.0, 7.0), dict(tau=0.56, inlet_velocity=0.06, smagorinsky_cs=0.1)),
    ((136, 24, 20), (60.0, 12.0, 10.0, 5.0),
     dict(tau=0.6, inlet_velocity=0.05, smagorinsky_cs=0.12, reverse_flow=1, free_slip_y=0)),
    ((200, 18, 26), (70.0, 9.0, 13.0, 4.5), dict(tau=0.58, inlet_velocity=0.05, smagorinsky_cs=0.0, free_slip_z=0)),
    ((256, 22, 24), (131.5, 11.0, 12.0, 6.5), dict(tau=0.57, inlet_velocity=0.06, smagorinsky_cs=0.1)),
]


def _params(p):
    from flowcraft_b200.lbm import Params
    return Params(tau=p["tau"], inletVelocity=p["inlet_velocity"], reverseFlow=bool(p.get("reverse_flow", 0)),
                  freeSlipY=bool(p.get("free_slip_y", 1)), freeSlipZ=bool(p.get("free_slip_z", 1)),
                  smagorinskyCs=p["smagorinsky_cs"])


def _solver(shape, sphere, params, storage, q, flags):
    from flowcraft_b200.lbm import LatticeModel, LbmSolver, Storage, Streaming, VoxelGrid
    nx, ny, nz = shape
    solid, sdf = geometry({"kind": "sphere", "dims": [nx, ny, nz], "center": list(sphere[:3]), "r": sphere[3]})
    s = LbmSolver()
    assert s.Init(0, VoxelGrid(nx, ny, nz, solid=solid, signedDistance=sdf),
                  LatticeModel.D3Q19 if q == 19 else LatticeModel.D3Q15, Storage[storage], Streaming.PINGPONG,
                  flags), s.LastError()
    s.Reset(_params(params), True)
    return s


@pytest.mark.parametrize("q", [19, 15])
@pytest.mark.parametrize("storage", ["FP32", "FP16_OFFSET", "BF16_OFFSET"])
@pytest.mark.parametrize("k", range(len(LATTICES)))
def test_staged_bit_identical_to_unstaged(gpu, k, storage, q):
    from flowcraft_b200.lbm import OPTION_TMA_STAGING
    shape, sphere, params = LATTICES[k]
    a = _solver(shape, sphere, params, storage, q, OPTION_TMA_STAGING)
    b = _solver(shape, sphere, params, storage, q, 0)
    l0a, l0b = a.LaunchCount(), b.LaunchCount()
    a.Step(None, 25)
    b.Step(None, 25)
    # the staged path (16-bit formats) adds its own launch per step
    assert a.LaunchCount() - l0a == b.LaunchCount() - l0b + (0 if storage == "FP32" else 25)
    pa, pb = a.SavePopulations(), b.SavePopulations()
    assert np.array_equal(pa.view(np.uint32), pb.view(np.uint32)), f"{shape} {storage} D3Q{q}"
    assert not a.HasDiverged()
    a.close()
    b.close()


@pytest.mark.parametrize("storage,tol", [("FP16_OFFSET", 2e-4), ("BF16_OFFSET", 2e-3)])
def test_staged_16bit_error_vs_fp64_oracle(gpu, oracle_built, storage, tol):
    """The staged 16-bit path against the FP64 oracle, with the tolerances of
    the unstaged 16-bit tests."""
    shape, sphere, params = LATTICES[0]
    case = dict(geom={"kind": "sphere", "dims": list(shape), "center": list(sphere[:3]), "r": sphere[3]}, q=19,
                params=params, seed_mid=True)
    from flowcraft_b200.lbm import OPTION_TMA_STAGING
    s = _solver(shape, sphere, params, storage, 19, OPTION_TMA_STAGING)
    ora = OracleAdapter(case, precision="f64")
    s.Step(None, 30)
    ora.step(30)
    g = s.ReadbackField().reshape(-1, 4).astype(np.float64)
    r = ora.o.readback_field_f64().reshape(-1, 4)
    fl = ~geometry(case["geom"])[0].ravel().astype(bool)
    assert np.abs(g - r)[fl].max() < tol
    s.close()


def test_staged_step_range_chunks(gpu):
    """StepRange over z chunks that start and end inside the interior."""
    shape, sphere, params = LATTICES[0]
    from flowcraft_b200.lbm import OPTION_TMA_STAGING
    full = _solver(shape, sphere, params, "FP16_OFFSET", 19, OPTION_TMA_STAGING)
    part = _solver(shape, sphere, params, "FP16_OFFSET", 19, OPTION_TMA_STAGING)
    for _ in range(4):
        full.Step(None, 1)
        for z0 in (0, 1, 7, 19, 29):
            part.StepRange(None, z0, {0: 1, 1: 6, 7: 12, 19: 10, 29: 1}[z0])
        part.AdvanceSubstep()
    assert np.array_equal(full.SavePopulations().view(np.uint32), part.SavePopulations().view(np.uint32))
