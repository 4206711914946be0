"""fc_lbm_stats_noalloc: solver statistics computed without allocating any
device memory, for callers that cannot allocate — applications whose own
pool allocator owns all of the GPU's memory, runs under a fixed memory budget,
and latency-critical loops where a cudaMalloc/cudaFree could synchronize the
device. The test calls the entry point through the C ABI on device buffers the
test owns, twice in a row, and checks each result against
fc_lbm_readback_stats on the same state with the tolerance the other stats
tests use. It lives in its own file, collected last, and passes alone in a
fresh process as well as after the other tests."""
import numpy as np
import pytest

from cases import geometry

pytestmark = pytest.mark.gpu

SLOTS = 12  # FC_LBM_STATS_SLOTS in include/fc_lbm.h


def _case():
    # 160x40x40 = 256,000 cells: two partial-sum blocks of the reduction
    return dict(geom={"kind": "sphere", "dims": [160, 40, 40], "center": [52.0, 20.0, 20.0], "r": 7.0}, q=19,
                params=dict(tau=0.56, inlet_velocity=0.06, smagorinsky_cs=0.1), seed_mid=True)


def test_stats_noalloc_matches_readback_stats(gpu):
    import torch

    from flowcraft_b200 import lbm

    lib = gpu
    case = _case()
    solid, sdf = geometry(case["geom"])
    nz, ny, nx = solid.shape
    s = lbm.LbmSolver()
    assert s.Init(0, lbm.VoxelGrid(nx, ny, nz, solid=solid, signedDistance=sdf), lbm.LatticeModel.D3Q19,
                  lbm.Storage.FP32), s.LastError()
    p = case["params"]
    s.Reset(lbm.Params(tau=p["tau"], inletVelocity=p["inlet_velocity"], smagorinskyCs=p["smagorinsky_cs"]), True)
    s.Step(None, 50)
    ref = s.ReadbackStats()

    # the caller's own device buffers: inputs and the output slots
    pops = torch.from_numpy(s.SavePopulations()).to("cuda").contiguous()
    d_solid = torch.from_numpy(solid.ravel().copy()).to("cuda")
    d_sdf = torch.from_numpy(sdf.ravel().copy()).to("cuda")
    out = torch.empty(SLOTS, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()

    for call in range(2):
        out.fill_(float("nan"))
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        rc = lib.fc_lbm_stats_noalloc(pops.data_ptr(), d_solid.data_ptr(), d_sdf.data_ptr(), nx, ny, nz,
                                      lbm.LatticeModel.D3Q19, lbm.Storage.FP32, out.data_ptr(), stream)
        assert rc == lbm.FC_LBM_OK
        torch.cuda.synchronize()
        if call == 1:  # the first call on a device looks the scratch address up; later calls touch nothing else
            assert torch.cuda.mem_get_info()[0] == free_before
        v = out.cpu().numpy()
        fluid = v[6]
        assert fluid == ref.fluidCells > 0
        assert float(np.float32(v[0] / fluid)) == pytest.approx(ref.avgDensity, rel=2e-6)
        assert float(np.float32(v[1] / fluid)) == pytest.approx(ref.avgSpeed, rel=2e-6)
        assert v[2] == pytest.approx(ref.totalMass, rel=1e-9)
        for k, f in zip((3, 4, 5), ref.forceSum):
            assert v[k] == pytest.approx(f, rel=1e-9, abs=1e-12)
        assert float(np.float32(v[3])) == pytest.approx(ref.forceX, rel=2e-6, abs=1e-9)
        assert np.float32(v[7]) == np.float32(ref.minDensity)
        assert np.float32(v[8]) == np.float32(ref.maxDensity)
        assert np.float32(v[9]) == np.float32(ref.maxSpeed)
        assert np.float32(v[10]) == np.float32(ref.maxStress)
        assert (v[11] != 0) == ref.hasNaN
    s.close()


def test_stats_noalloc_rejects_lattices_beyond_its_scratch(gpu):
    import torch

    from flowcraft_b200 import lbm

    lib = gpu
    tiny = torch.zeros(16, dtype=torch.float32, device="cuda")
    out = torch.zeros(SLOTS, dtype=torch.float64, device="cuda")
    # 1024^3 cells exceed the 2^29-cell limit: refused before any work is queued
    rc = lib.fc_lbm_stats_noalloc(tiny.data_ptr(), tiny.data_ptr(), None, 1024, 1024, 1024,
                                  lbm.LatticeModel.D3Q19, lbm.Storage.FP32, out.data_ptr(), None)
    assert rc == lbm.FC_LBM_ERR_TOO_LARGE
    assert lib.fc_lbm_stats_noalloc(None, None, None, 8, 8, 8, 1, 0, out.data_ptr(), None) == lbm.FC_LBM_ERR_INVALID_ARG
