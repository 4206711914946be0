"""fc_lbm_stats_noalloc: solver statistics computed without allocating any
device memory, for callers that cannot allocate — applications whose own
pool allocator owns all of the GPU's memory, runs under a fixed memory budget,
and latency-critical loops where a cudaMalloc/cudaFree could synchronize the
device. The test calls the entry point through the C ABI on device buffers the
test owns, twice in a row, and checks each result against
fc_lbm_readback_stats on the same state with the tolerance the other stats
tests use, for both lattices, the three storage formats and a grid without a
signed-distance field. It lives in its own file, collected last, and passes
alone in a fresh process as well as after the other tests."""
import numpy as np
import pytest

from cases import geometry

pytestmark = pytest.mark.gpu

SLOTS = 12  # FC_LBM_STATS_SLOTS in include/fc_lbm.h

# (lattice, storage, with signed distance)
CASES = [
    pytest.param(19, 0, True, id="q19-fp32"),
    pytest.param(15, 1, True, id="q15-fp16-offset"),
    pytest.param(19, 2, True, id="q19-bf16-offset"),
    pytest.param(19, 0, False, id="q19-fp32-no-sdf"),
]


def _geom():
    # 160x40x40 = 256,000 cells: 125 partial-sum blocks of the reduction
    return {"kind": "sphere", "dims": [160, 40, 40], "center": [52.0, 20.0, 20.0], "r": 7.0}


def _weights(lbm, model, nx, ny, nz, solid):
    """w_i of the lattice: the populations of a state at rest (rho 1, u 0)."""
    s = lbm.LbmSolver()
    assert s.Init(0, lbm.VoxelGrid(nx, ny, nz, solid=solid), model, lbm.Storage.FP32), s.LastError()
    s.Reset(lbm.Params(tau=0.6, inletVelocity=0.0, smagorinskyCs=0.0), False)
    w = s.SavePopulations()[:, 0].astype(np.float32)
    s.close()
    return w


def _device_set(lbm, storage, pops, w):
    """The caller's own device copy of a population set in `storage`'s format,
    checked to decode to exactly the solver's values (so both entry points see
    the same populations)."""
    import torch

    if storage == lbm.Storage.FP32:
        return torch.from_numpy(pops.copy()).to("cuda").contiguous()
    off = (pops.astype(np.float64) - w[:, None].astype(np.float64)) * 256.0
    if storage == lbm.Storage.FP16_OFFSET:
        h = torch.from_numpy(off).to(torch.float16)
    else:
        h = torch.from_numpy(off).to(torch.bfloat16)
    back = (h.to(torch.float64).numpy() / 256.0 + w[:, None].astype(np.float64)).astype(np.float32)
    # the exact decode: fmaf(h, 2^-8, w) rounds once, as float32(h * 2^-8 + w) in float64 does
    assert np.array_equal(back, pops), "re-encoded offsets do not decode to the solver's populations"
    return h.to("cuda").contiguous()


@pytest.mark.parametrize("q,storage,with_sdf", CASES)
def test_stats_noalloc_matches_readback_stats(gpu, q, storage, with_sdf):
    import torch

    from flowcraft_b200 import lbm

    lib = gpu
    model = lbm.LatticeModel.D3Q19 if q == 19 else lbm.LatticeModel.D3Q15
    storage = lbm.Storage(storage)
    solid, sdf = geometry(_geom())
    if not with_sdf:
        sdf = None
    nz, ny, nx = solid.shape
    s = lbm.LbmSolver()
    assert s.Init(0, lbm.VoxelGrid(nx, ny, nz, solid=solid, signedDistance=sdf), model, storage), s.LastError()
    s.Reset(lbm.Params(tau=0.56, inletVelocity=0.06, smagorinskyCs=0.1), True)
    s.Step(None, 50)
    ref = s.ReadbackStats()
    pops = s.SavePopulations()
    s.close()
    w = _weights(lbm, model, nx, ny, nz, solid) if storage != lbm.Storage.FP32 else None

    # the caller's own device buffers: inputs and the output slots
    d_pops = _device_set(lbm, storage, pops, w)
    d_solid = torch.from_numpy(solid.ravel().copy()).to("cuda")
    d_sdf = torch.from_numpy(sdf.ravel().copy()).to("cuda") if with_sdf else None
    out = torch.empty(SLOTS, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()

    for call in range(2):
        out.fill_(float("nan"))
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        rc = lib.fc_lbm_stats_noalloc(d_pops.data_ptr(), d_solid.data_ptr(),
                                      d_sdf.data_ptr() if d_sdf is not None else None, nx, ny, nz, model, storage,
                                      out.data_ptr(), stream)
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
