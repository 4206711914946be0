"""Batches (fc_lbm_batch_*): many lattices of uneven sizes stepped by one
bulk launch per step (persistent, or one block per tile) or by the members'
own bulk kernels side by side, with CUDA-graph replay and the autotuner,
must give the same bits as stepping every lattice on its own."""
import numpy as np
import pytest

from cases import geometry

pytestmark = pytest.mark.gpu

SHAPES = [  # (nx, ny, nz), sphere (cx, cy, cz, r), params
    ((96, 48, 40), (30.0, 24.0, 20.0, 6.0), dict(tau=0.56, inletVelocity=0.06, smagorinskyCs=0.1)),
    ((128, 32, 36), (40.0, 16.0, 18.0, 5.0), dict(tau=0.6, inletVelocity=0.05, smagorinskyCs=0.12, freeSlipY=False)),
    ((64, 40, 24), (20.0, 20.0, 12.0, 4.5), dict(tau=0.58, inletVelocity=0.05, smagorinskyCs=0.1, reverseFlow=True)),
    ((200, 24, 20), (60.0, 12.0, 10.0, 4.0), dict(tau=0.55, inletVelocity=0.04, smagorinskyCs=0.08, freeSlipZ=False)),
]


def _make(storage, q=19):
    from flowcraft_b200.lbm import LatticeModel, LbmSolver, Params, Storage, VoxelGrid
    out = []
    for (nx, ny, nz), sph, prm in SHAPES:
        solid, sdf = geometry({"kind": "sphere", "dims": [nx, ny, nz], "center": list(sph[:3]), "r": sph[3]})
        s = LbmSolver()
        assert s.Init(0, VoxelGrid(nx, ny, nz, solid=solid.ravel(), signedDistance=sdf.ravel()),
                      LatticeModel.D3Q19 if q == 19 else LatticeModel.D3Q15, Storage[storage])
        s.Reset(Params(**prm), True)
        out.append(s)
    return out


def _same(a, b):
    for x, y in zip(a, b):
        fx, fy = x.SavePopulations(), y.SavePopulations()
        assert np.array_equal(fx.view(np.uint32), fy.view(np.uint32))


@pytest.mark.parametrize("storage,q", [("FP32", 19), ("FP16_OFFSET", 19), ("FP32", 15)])
def test_batch_is_bit_identical_to_single_steps(gpu, storage, q):
    from flowcraft_b200.batch import LbmBatch
    batched, single = _make(storage, q), _make(storage, q)
    b = LbmBatch(batched)
    b.Step(11)   # five graph replays and one direct step
    b.Step(6)    # a rebuilt graph after the odd count
    for s in single:
        s.Step(None, 17)
    _same(batched, single)
    for rows, mult in ((4, 2), (16, 1), (8, 0), (0, 1)):
        b.Config(rows, mult)
        b.Step(4)
        for s in single:
            s.Step(None, 4)
    _same(batched, single)
    # the members remain ordinary solvers: readbacks and stepping on their own
    for x, y in zip(batched, single):
        assert np.array_equal(x.ReadbackField().view(np.uint32), y.ReadbackField().view(np.uint32))
        x.Step(None, 1)
        y.Step(None, 1)
    _same(batched, single)
    b.close()


def test_blocks_that_take_many_chunks(gpu):
    """About 6M cells: with one wave of resident blocks every block takes
    several chunks of tiles in turn, within a lattice and across lattice
    ends (tile counts that are no multiple of the chunk), and the batch
    still gives the bits of single stepping."""
    from flowcraft_b200.batch import LbmBatch
    from flowcraft_b200.lbm import LatticeModel, LbmSolver, Params, Storage, VoxelGrid
    # tiles at 16 / 4 rows: 3668 / 13100, 612 / 2448, 3232 / 12120 (chunks of 8)
    shapes = [((250, 100, 131), (80.0, 50.0, 65.0, 12.0)), ((130, 62, 51), (40.0, 31.0, 25.0, 6.0)),
              ((200, 120, 101), (60.0, 60.0, 50.0, 10.0))]

    def make():
        out = []
        for (nx, ny, nz), sph in shapes:
            solid, sdf = geometry({"kind": "sphere", "dims": [nx, ny, nz], "center": list(sph[:3]), "r": sph[3]})
            s = LbmSolver()
            assert s.Init(0, VoxelGrid(nx, ny, nz, solid=solid.ravel(), signedDistance=sdf.ravel()),
                          LatticeModel.D3Q19, Storage.FP16_OFFSET)
            s.Reset(Params(tau=0.56, inletVelocity=0.06, smagorinskyCs=0.1), True)
            out.append(s)
        return out

    batched, single = make(), make()
    assert sum(s.CellCount() for s in batched) > 6_000_000
    b = LbmBatch(batched)
    for rows, mult in ((16, 1), (4, 1), (8, 0)):
        b.Config(rows, mult)
        b.Step(4)
        for s in single:
            s.Step(None, 4)
    _same(batched, single)
    assert not any(s.HasDiverged() for s in batched)
    b.close()
    for s in batched + single:
        s.close()


def test_one_block_per_tile_over_many_lattices(gpu):
    """40 small lattices of varied sizes and parameters: the one-block-per-tile
    form carries at most 32 lattices in one launch's parameters, so a step
    takes two launches; every lattice keeps the bits of single stepping."""
    from flowcraft_b200.batch import LbmBatch
    from flowcraft_b200.lbm import LatticeModel, LbmSolver, Params, Storage, VoxelGrid

    def make():
        out = []
        r = np.random.default_rng(7)
        for k in range(40):
            nx = int(r.integers(8, 33)) * 2
            ny, nz = int(r.integers(8, 25)), int(r.integers(8, 25))
            solid, sdf = geometry({"kind": "sphere", "dims": [nx, ny, nz],
                                   "center": [nx / 3.0, ny / 2.0, nz / 2.0], "r": min(ny, nz) / 5.0})
            s = LbmSolver()
            assert s.Init(0, VoxelGrid(nx, ny, nz, solid=solid.ravel(), signedDistance=sdf.ravel()),
                          LatticeModel.D3Q19, Storage.FP16_OFFSET)
            s.Reset(Params(tau=float(r.uniform(0.52, 0.6)), inletVelocity=float(r.uniform(0.03, 0.07)),
                           smagorinskyCs=0.1, reverseFlow=bool(k % 5 == 3)), True)
            out.append(s)
        return out

    batched, single = make(), make()
    b = LbmBatch(batched)
    b.Config(8, 0)
    b.Step(7)  # three graph replays of two launches per step, then one direct step
    for s in single:
        s.Step(None, 7)
    _same(batched, single)
    assert not any(s.HasDiverged() for s in batched)
    b.close()
    for s in batched + single:
        s.close()


def test_tuner_picks_a_shape_and_keeps_results(gpu):
    from flowcraft_b200.batch import CANDIDATES, LbmBatch
    batched, single = _make("FP16_OFFSET"), _make("FP16_OFFSET")
    b = LbmBatch(batched)
    r = b.Tune(steps=4)
    assert (r["rows"], r["grid_mult"]) in CANDIDATES
    assert len(r["ms_per_step"]) == len(CANDIDATES) == 8 and all(v > 0 for v in r["ms_per_step"].values())
    for s in single:
        s.Step(None, len(CANDIDATES) * (4 + 2))
    b.Step(8)
    for s in single:
        s.Step(None, 8)
    _same(batched, single)
    assert not any(s.HasDiverged() for s in batched)
    b.close()


def test_batch_refuses_mismatched_members(gpu):
    from flowcraft_b200.batch import LbmBatch
    from flowcraft_b200.closure import ClosureWeights
    from flowcraft_b200.lbm import LatticeModel, LbmError, LbmSolver, Storage, VoxelGrid
    a = _make("FP32")
    b16 = _make("FP16_OFFSET")
    with pytest.raises(LbmError):
        LbmBatch([a[0], b16[1]])
    odd = LbmSolver()
    assert odd.Init(0, VoxelGrid(33, 8, 8, solid=np.zeros(33 * 64, np.uint8)), LatticeModel.D3Q19, Storage.FP32)
    with pytest.raises(LbmError):
        LbmBatch([a[0], odd])
    b16[0].SetClosure(ClosureWeights.random(0))
    with pytest.raises(LbmError):
        LbmBatch([b16[0], b16[1]])
    with pytest.raises(LbmError):
        LbmBatch([a[0], a[0]])


def test_batch_refuses_member_given_a_closure_after_create(gpu):
    """A learned closure set on a member after the batch was created is
    refused at the next batch step instead of being stepped with Smagorinsky."""
    from flowcraft_b200.batch import LbmBatch
    from flowcraft_b200.closure import ClosureWeights
    from flowcraft_b200.lbm import FC_LBM_ERR_UNSUPPORTED, LbmError
    m = _make("FP16_OFFSET")
    b = LbmBatch(m)
    b.Step(2)
    m[1].SetClosure(ClosureWeights.random(0))
    with pytest.raises(LbmError) as ei:
        b.Step(2)
    assert ei.value.code == FC_LBM_ERR_UNSUPPORTED
    with pytest.raises(LbmError):
        b.Tune(1)
    m[1].SetClosure(None)
    b.Step(2)
    b.close()


def test_polar_sweep_small(gpu):
    """A 3-angle polar on 64x32x32 wings: finite forces, lift rising with
    angle, drag positive, the reference's polar fields filled in."""
    from flowcraft_b200.sweep import polar_sweep
    r = polar_sweep(nx=64, alphas=[-2.0, 4.0, 10.0], re=2e3, u=0.06, steps=400, tune=False, chunk=40)
    assert r.valid and len(r.points) == 3
    cl = [p.cl for p in r.points]
    assert cl[0] < cl[1] < cl[2]
    assert all(p.cd > 0 for p in r.points)
    assert r.clAlphaPerDeg > 0 and r.refChord == 24.0 and abs(r.aspectRatio - 0.75 * 32 / 24.0) < 1e-9
