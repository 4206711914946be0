"""Asynchronous field readback (fc_lbm_readback_field_async): the snapshot is
the state every step queued before the call leaves, even while later steps
run and overwrite both population sets, and those steps compute exactly what
they compute without a readback in flight."""
import time

import numpy as np
import pytest

from cases import geometry

pytestmark = pytest.mark.gpu

CASE = dict(geom={"kind": "sphere", "dims": [96, 40, 36], "center": [30.0, 20.0, 18.0], "r": 6.0}, q=19,
            params=dict(tau=0.56, inlet_velocity=0.06, smagorinsky_cs=0.1), seed_mid=True)


def _solver(storage, streaming, case=CASE):
    from flowcraft_b200.lbm import LatticeModel, LbmSolver, Params, Storage, Streaming, VoxelGrid
    solid, sdf = geometry(case["geom"])
    nz, ny, nx = solid.shape
    s = LbmSolver()
    assert s.Init(0, VoxelGrid(nx, ny, nz, solid=solid, signedDistance=sdf), LatticeModel.D3Q19, Storage[storage],
                  Streaming[streaming]), s.LastError()
    p = case["params"]
    s.Reset(Params(tau=p["tau"], inletVelocity=p["inlet_velocity"], smagorinskyCs=p["smagorinsky_cs"]), True)
    return s


def _same(a, b):
    return np.array_equal(np.asarray(a).view(np.uint32), np.asarray(b).view(np.uint32))


@pytest.mark.parametrize("storage,streaming", [("FP32", "PINGPONG"), ("FP16_OFFSET", "PINGPONG"),
                                               ("FP16_OFFSET", "AA"), ("FP32", "AA")])
def test_async_snapshot_and_overlapped_steps(gpu, storage, streaming):
    from flowcraft_b200.lbm import PinnedBuffer
    a, b = _solver(storage, streaming), _solver(storage, streaming)
    buf = PinnedBuffer(a.CellCount() * 4)
    a.Step(None, 5)
    b.Step(None, 5)
    a.ReadbackFieldAsync(buf.array)
    a.Step(None, 4)  # overwrites both population sets while the copy is in flight
    a.ReadbackWait(60000)
    assert _same(buf.array, b.ReadbackField())
    b.Step(None, 4)
    assert _same(a.SavePopulations(), b.SavePopulations())
    # a second readback right after, and a reset that overwrites the snapshot's set
    a.ReadbackFieldAsync(buf.array)
    a.Reset(a.GetParams(), True)
    a.ReadbackWait(60000)
    assert _same(buf.array, b.ReadbackField())
    buf.free()
    a.close()
    b.close()


def test_async_readback_overlaps_steps(gpu):
    """The copy of a 256x128x128 field (134 MB) runs beside the steps: the
    steps plus an overlapped readback take less than the steps plus a
    blocking one."""
    from flowcraft_b200.lbm import PinnedBuffer
    case = dict(CASE, geom={"kind": "sphere", "dims": [256, 128, 128], "center": [80.0, 64.0, 64.0], "r": 12.0})
    s = _solver("FP16_OFFSET", "PINGPONG", case)
    buf = PinnedBuffer(s.CellCount() * 4)
    host = np.empty(s.CellCount() * 4, np.float32)
    s.Step(None, 4)
    s.Sync()
    s.ReadbackFieldAsync(buf.array)
    s.ReadbackWait()
    t0 = time.perf_counter()
    s.ReadbackField()
    s.Step(None, 30)
    s.Sync()
    blocking = time.perf_counter() - t0
    t0 = time.perf_counter()
    s.ReadbackFieldAsync(buf.array)
    s.Step(None, 30)
    s.Sync()
    s.ReadbackWait()
    overlapped = time.perf_counter() - t0
    print(f"steps + blocking readback {blocking * 1e3:.1f} ms, steps + overlapped readback {overlapped * 1e3:.1f} ms")
    assert overlapped < blocking
    del host
    buf.free()
    s.close()
