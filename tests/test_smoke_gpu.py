"""Smoke-trail particles on the device (flowcraft_b200.smoke, particles.cu).

Advection must match the reference's SmokeTrailSystem::Step bit for bit on
the FP32 path (fixture made by the reference: tests/golden/smoke_golden.json),
under either streaming scheme; the respawn, vanish, scatter and plane rules
are checked against the reference's stated behaviour."""
import json
import os

import numpy as np
import pytest

from cases import CASES, GOLDEN_DIR, field_digest, geometry

pytestmark = pytest.mark.gpu


def _params(p):
    from flowcraft_b200.lbm import Params
    return Params(tau=p["tau"], inletVelocity=p["inlet_velocity"], reverseFlow=bool(p.get("reverse_flow", 0)),
                  freeSlipY=bool(p.get("free_slip_y", 1)), freeSlipZ=bool(p.get("free_slip_z", 1)),
                  smagorinskyCs=p["smagorinsky_cs"])


def _solver(case, storage="FP32", streaming="PINGPONG"):
    from flowcraft_b200.lbm import LatticeModel, LbmSolver, Storage, Streaming, VoxelGrid
    solid, sdf = geometry(case["geom"])
    nz, ny, nx = solid.shape
    s = LbmSolver()
    assert s.Init(0, VoxelGrid(nx, ny, nz, solid=solid, signedDistance=sdf),
                  LatticeModel.D3Q19 if case["q"] == 19 else LatticeModel.D3Q15, Storage[storage],
                  Streaming[streaming]), s.LastError()
    s.Reset(_params(case["params"]), case["seed_mid"])
    return s, solid


@pytest.mark.parametrize("streaming", ["PINGPONG", "AA"])
def test_device_trails_match_reference(gpu, streaming):
    from flowcraft_b200.smoke import PlaneConfinement, SmokeTrailSystem
    fx = json.load(open(os.path.join(GOLDEN_DIR, "smoke_golden.json")))
    s, solid = _solver(CASES[fx["case"]], "FP32", streaming)
    s.Step(None, fx["case_steps"])
    assert field_digest(s.ReadbackField()) == fx["field_sha256"]
    sm = SmokeTrailSystem(s)
    for run in fx["runs"]:
        pos = np.array(run["positions"], dtype=np.float32)
        conf = PlaneConfinement(run["confine_axis"], run["confine_index"]) if run["confine_axis"] >= 0 else None
        sm.Reset(False, len(pos), fx["trail_length"], conf)
        sm.SetPositions(pos)
        for _ in range(fx["steps"]):
            sm.Step(False, run["mm_per_sec"], run["dt"], False, conf)
        got, lens = sm.Trails()
        want = np.array(run["trail_bits"], dtype=np.uint32)
        for p in np.nonzero(np.array(run["keep"]))[0]:
            n = run["lens"][p]
            assert lens[p] == n
            assert np.array_equal(got[p, :n].view(np.uint32), want[p, :n]), (run["name"], p)
    s.close()


def test_respawn_vanish_scatter_and_plane_rules(gpu):
    from flowcraft_b200.smoke import X, Z, PlaneConfinement, SmokeTrailSystem
    case = CASES["sphere48_q19"]
    s, solid = _solver(case)
    s.Step(None, 20)
    nz, ny, nx = solid.shape
    sd = solid.astype(bool)
    sm = SmokeTrailSystem(s)

    def cell(p):  # world -> grid (x from world y, y from world x)
        return int(np.floor(p[1])), int(np.floor(p[0])), int(np.floor(p[2]))

    # Reset scatters over the whole domain, every head in a fluid cell
    sm.Reset(False, 2000, 6, seed=7)
    heads = sm.Heads()
    xs = [cell(h)[0] for h in heads]
    assert min(xs) < nx // 4 and max(xs) > 3 * nx // 4
    assert all(not sd[z, y, x] for x, y, z in map(cell, heads))
    # particles outside the grid respawn at the inlet face (x = 0; x = nx-1 reversed), in fluid
    for reverse in (False, True):
        sm.SetPositions(np.tile(np.array([[-5.0, -5.0, -5.0]], np.float32), (2000, 1)))
        sm.Step(reverse, 10.0, 0.05)
        got, lens = sm.Trails()
        assert (lens == 1).all()
        for h in got[:, 0]:
            x, y, z = cell(h)
            assert x == (nx - 1 if reverse else 0) and not sd[z, y, x]
    # with respawning suspended they vanish instead, and come back after
    sm.SetPositions(np.tile(np.array([[-5.0, -5.0, -5.0]], np.float32), (2000, 1)))
    sm.Step(False, 10.0, 0.05, True)
    assert (sm.Trails()[1] == 0).all()
    sm.Step(False, 10.0, 0.05, True)
    assert (sm.Trails()[1] == 0).all()
    sm.Step(False, 10.0, 0.05)
    assert (sm.Trails()[1] == 1).all()
    # confined to the plane z = 5: seeded on it, advected within it
    c = PlaneConfinement(Z, 5)
    sm.ScatterRandom(c)
    for _ in range(4):
        sm.Step(False, 10.0, 0.05, False, c)
    got, lens = sm.Trails()
    stayed = np.nonzero(lens == 5)[0]  # a respawn jitters along the confined axis (the reference's rule)
    assert len(stayed) > 1900
    pts = np.concatenate([got[p, :5] for p in stayed])
    assert np.all(pts[:, 2] == np.float32(5.5))
    # ShiftPlane moves every kept point onto the new plane (grid x = 30 is world y = 30.5)
    cx = PlaneConfinement(X, 30)
    sm.ScatterRandom(cx)
    for _ in range(3):
        sm.Step(False, 10.0, 0.05, False, cx)
    sm.ShiftPlane(PlaneConfinement(X, 30 + 4))
    got, lens = sm.Trails()
    pts = np.concatenate([got[p, :lens[p]] for p in range(len(lens))])
    assert np.all(pts[:, 1] == np.float32(34.5))
    s.close()


def test_fp16_trails_follow_fp32(gpu):
    """The 16-bit formats advect through their own (rounded) velocity field."""
    from flowcraft_b200.smoke import SmokeTrailSystem
    fx = json.load(open(os.path.join(GOLDEN_DIR, "smoke_golden.json")))
    run = fx["runs"][0]
    pos = np.array(run["positions"], dtype=np.float32)
    res = {}
    for st in ("FP32", "FP16_OFFSET"):
        s, _ = _solver(CASES[fx["case"]], st)
        s.Step(None, fx["case_steps"])
        sm = SmokeTrailSystem(s)
        sm.Reset(False, len(pos), 8)
        sm.SetPositions(pos)
        for _ in range(7):
            sm.Step(False, run["mm_per_sec"], run["dt"])
        res[st] = sm.Trails()[0]
        s.close()
    assert np.abs(res["FP32"] - res["FP16_OFFSET"]).max() < 2e-3
