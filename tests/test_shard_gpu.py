"""One lattice split into z-slabs (flowcraft_b200.shard), ranks emulated in
one process on one GPU: every rank steps its slab through the solver's
StepRange / LayerCopy / AdvanceSubstep with halo layers exchanged as device
copies, and the owned layers must carry the unsplit lattice's bits: the
populations, and the field readback (moments on fluid cells, the
momentum-exchange force on solid cells) after the outer halos' refresh."""
import numpy as np
import pytest

from cases import geometry

pytestmark = pytest.mark.gpu

# (nx, ny, nz), sphere (cx, cy, cz, r) centred on the 2-rank cut z = nz / 2
CASES = [
    ((64, 32, 40), (20.0, 16.0, 20.0, 6.0), dict(tau=0.56, inletVelocity=0.06, smagorinskyCs=0.1)),
    ((96, 24, 27), (30.0, 12.0, 13.5, 5.0), dict(tau=0.6, inletVelocity=0.05, smagorinskyCs=0.12, freeSlipZ=False)),
]


def _run(storage, q, world, case, steps):
    import torch

    from flowcraft_b200 import shard
    from flowcraft_b200.lbm import LatticeModel, LbmSolver, Params, Storage, VoxelGrid
    (nx, ny, nz), sph, prm = case
    solid, sdf = geometry({"kind": "sphere", "dims": [nx, ny, nz], "center": list(sph[:3]), "r": sph[3]})
    model = LatticeModel.D3Q19 if q == 19 else LatticeModel.D3Q15
    full = LbmSolver()
    assert full.Init(0, VoxelGrid(nx, ny, nz, solid=solid.ravel(), signedDistance=sdf.ravel()), model,
                     Storage[storage]), full.LastError()
    full.Reset(Params(**prm), True)
    full.Step(None, steps)
    ref = full.ReadbackField().reshape(nz, ny * nx, 4)
    ranks = shard.emulated_ranks(solid, sdf, world, 0, model, Storage[storage], Params(**prm))
    shard.step_emulated([st for _, _, st in ranks], steps)
    shard.refresh_emulated([st for _, _, st in ranks])  # the solid-cell forces read two layers out
    torch.cuda.synchronize()
    out = []
    for s, lay, _ in ranks:
        out.append((shard.owned_field(s, lay), ref[lay.z0:lay.z1].reshape(-1, 4), lay))
        assert not s.HasDiverged()
        s.close()
    full.close()
    return out


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("storage,q", [("FP32", 19), ("FP16_OFFSET", 19), ("FP32", 15)])
def test_slabs_are_bit_identical_to_the_unsplit_lattice(gpu, storage, q, world):
    for case in CASES:
        for got, want, lay in _run(storage, q, world, case, 24):
            assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), (case[0], lay)


def test_slab_population_sets_match(gpu):
    """The populations themselves, not only the moments, on the 3-rank split."""
    import torch

    from flowcraft_b200 import shard
    from flowcraft_b200.lbm import LatticeModel, LbmSolver, Params, Storage, VoxelGrid
    (nx, ny, nz), sph, prm = CASES[0]
    solid, sdf = geometry({"kind": "sphere", "dims": [nx, ny, nz], "center": list(sph[:3]), "r": sph[3]})
    full = LbmSolver()
    assert full.Init(0, VoxelGrid(nx, ny, nz, solid=solid.ravel(), signedDistance=sdf.ravel()), LatticeModel.D3Q19,
                     Storage.FP32)
    full.Reset(Params(**prm), True)
    full.Step(None, 11)  # odd: the slabs end on the other population set
    ref = full.SavePopulations().reshape(19, nz, ny * nx)
    ranks = shard.emulated_ranks(solid, sdf, 3, 0, LatticeModel.D3Q19, Storage.FP32, Params(**prm))
    shard.step_emulated([st for _, _, st in ranks], 11)
    torch.cuda.synchronize()
    for s, lay, _ in ranks:
        got = s.SavePopulations().reshape(19, lay.local_nz, ny * nx)[:, lay.own0:lay.own1]
        assert np.array_equal(got.view(np.uint32), ref[:, lay.z0:lay.z1].view(np.uint32)), lay
        s.close()
    full.close()
