"""In-place (AA-pattern) streaming: one population set instead of two.

The AA step stores every value the ping-pong step stores, only in other
slots, so the FP32 path must still reproduce LbmReference bit-for-bit on the
golden cases, and every format must give bit-identical fields, statistics,
forces and populations to ping-pong on lattices that route cells through
every branch: Bouzidi near and far links, plain bounce-back, free-slip and
no-slip faces, inlet and outlet in both flow directions (flipped live), solid
outlet neighbours, and a warm start from a field; with the learned closure
too.
"""
import numpy as np
import pytest

from cases import CASES, field_digest, geometry, load_fixture, run_schedule

pytestmark = pytest.mark.gpu


def _params(p: dict):
    from flowcraft_b200.lbm import Params
    return Params(tau=p["tau"], inletVelocity=p["inlet_velocity"], reverseFlow=bool(p.get("reverse_flow", 0)),
                  freeSlipY=bool(p.get("free_slip_y", 1)), freeSlipZ=bool(p.get("free_slip_z", 1)),
                  smagorinskyCs=p["smagorinsky_cs"])


class Sim:
    def __init__(self, case, storage="FP32", streaming="AA"):
        from flowcraft_b200.lbm import LatticeModel, LbmSolver, Storage, Streaming, VoxelGrid
        solid, sdf = geometry(case["geom"])
        nz, ny, nx = solid.shape
        self.solid = solid.ravel().astype(bool)
        self.s = LbmSolver()
        grid = VoxelGrid(nx, ny, nz, solid=solid, signedDistance=sdf)
        model = LatticeModel.D3Q19 if case["q"] == 19 else LatticeModel.D3Q15
        assert self.s.Init(0, grid, model, Storage[storage], Streaming[streaming]), self.s.LastError()
        self.s.Reset(_params(case["params"]), case["seed_mid"])

    def step(self, n):
        self.s.Step(None, n)

    def readback_field(self):
        return self.s.ReadbackField()

    def reset_from_field(self, field):
        self.s.ResetFromField(field)

    def set_params(self, p):
        self.s.SetParams(_params(p))


EVEN_GOLDEN = [n for n, c in CASES.items() if c["geom"]["dims"][0] % 2 == 0]


@pytest.mark.parametrize("name", EVEN_GOLDEN)
def test_aa_fp32_matches_reference_bit_for_bit(gpu, name):
    case = CASES[name]
    fx = load_fixture(name)
    sim = Sim(case)
    got = []
    run_schedule(sim, case, lambda step, field: got.append((step, field.copy())))
    idx = np.array(fx["sample_idx"])
    assert len(got) == len(fx["checkpoints"])
    for (step, field), cp in zip(got, fx["checkpoints"]):
        assert step == cp["step"]
        assert np.array_equal(field.view(np.uint32).reshape(-1, 4)[idx], np.array(cp["sample_bits"], np.uint32))
        assert field_digest(field) == cp["field_sha256"], f"{name}@{step}: AA differs from LbmReference"


def _sphere(dims, center, r, q, **params):
    p = dict(tau=0.6, inlet_velocity=0.05, smagorinsky_cs=0.12)
    p.update(params)
    return dict(geom={"kind": "sphere", "dims": list(dims), "center": list(center), "r": r}, q=q, params=p,
                seed_mid=True)


# even-nx lattices covering the boundary branches of the golden set
BRANCHES = {
    "noslip_reverse": _sphere((24, 13, 11), (12, 6.3, 5.2), 3.1, 19, tau=0.55, inlet_velocity=0.07,
                              smagorinsky_cs=0.15, reverse_flow=1, free_slip_y=0, free_slip_z=0),
    "ground_q15": dict(_sphere((30, 15, 12), (10, 7, 3), 3.6, 15, tau=0.7, inlet_velocity=0.04, smagorinsky_cs=0.1,
                               free_slip_y=1, free_slip_z=0), seed_mid=False),
    "ywall": _sphere((18, 9, 14), (7, 4.5, 7), 2.4, 19, tau=0.62, inlet_velocity=0.06, smagorinsky_cs=0.0,
                     free_slip_y=0, free_slip_z=1),
    "outlet_block": dict(geom={"kind": "outlet_block", "dims": [22, 12, 9], "center": [8, 6, 4.5], "r": 2.5}, q=19,
                         params=dict(tau=0.6, inlet_velocity=0.05, smagorinsky_cs=0.12), seed_mid=True),
    "wide_q15": _sphere((160, 40, 40), (52, 20, 20), 7, 15, tau=0.56, inlet_velocity=0.06, smagorinsky_cs=0.1),
    "wide_nosdf": dict(_sphere((128, 34, 30), (40, 17, 15), 6.5, 19, free_slip_z=0), geom={
        "kind": "sphere", "dims": [128, 34, 30], "center": [40, 17, 15], "r": 6.5, "sdf": False}),
    # four 64-cell chunks per row with the sphere in the second: warps off the
    # row ends hold pairs cut by the wall (one cell bulk, one wall-adjacent)
    "interior_chunks": _sphere((256, 22, 20), (101.5, 11, 10), 5.3, 19, tau=0.57, inlet_velocity=0.06,
                               smagorinsky_cs=0.1),
}


def _flip(case):
    p = dict(case["params"])
    p["reverse_flow"] = 0 if p.get("reverse_flow", 0) else 1
    return p


def _same(a, b):
    return np.array_equal(np.asarray(a).view(np.uint32), np.asarray(b).view(np.uint32))


def _compare(pp, aa, what):
    fa, fb = pp.s.ReadbackField(), aa.s.ReadbackField()
    assert _same(fa, fb), f"{what}: field differs"
    sa, sb = pp.s.ReadbackStats(), aa.s.ReadbackStats()
    for k in ("avgDensity", "avgSpeed", "maxSpeed", "totalMass", "maxStress"):
        assert getattr(sa, k) == getattr(sb, k), f"{what}: stats {k} differs"
    xa, xb = pp.s.AerodynamicForces(), aa.s.AerodynamicForces()
    assert list(xa.forceSum) == list(xb.forceSum), f"{what}: forces differ"
    qa, qb = pp.s.SavePopulations(), aa.s.SavePopulations()
    assert _same(qa, qb), f"{what}: populations differ"
    assert pp.s.HasDiverged() == aa.s.HasDiverged()


@pytest.mark.parametrize("storage", ["FP32", "FP16_OFFSET", "BF16_OFFSET"])
@pytest.mark.parametrize("name", list(BRANCHES))
def test_aa_bit_identical_to_pingpong(gpu, name, storage):
    case = BRANCHES[name]
    pp, aa = Sim(case, storage, "PINGPONG"), Sim(case, storage, "AA")
    _compare(pp, aa, f"{name} after reset")
    for sim in (pp, aa):
        sim.step(7)
    _compare(pp, aa, f"{name} after 7 steps")  # read before an odd step
    for sim in (pp, aa):
        sim.set_params(_flip(case))  # the outlet moves to the other end, live
        sim.step(9)
    _compare(pp, aa, f"{name} after 16 steps")  # read before an even step
    info = aa.s.BoundaryInfo()
    assert info["boundary_cells"] > 0 and info["bulk_cells"] > 0


def _closure_for(sim, seed):
    """Random weights normalized to the lattice's own inputs, with a training
    range that leaves the tails out, so both the MLP and the Smagorinsky
    fallback run."""
    from flowcraft_b200.closure import ClosureWeights
    cw = ClosureWeights.random(seed, 2e-3)
    sim.s.SetClosure(cw)
    x, _, _ = sim.s.ClosureProbe()
    fluid = ~sim.solid
    cw.mean[:4] = x[fluid].mean(axis=0)
    cw.std[:4] = np.maximum(x[fluid].std(axis=0), 1e-3)
    cw.mean[4], cw.std[4], cw.filter_width = 1.0, 1.0, 1.0
    cw.lo = np.percentile(x[fluid][:, :3], 3.0, axis=0).astype(np.float32)
    cw.hi = np.percentile(x[fluid][:, :3], 97.0, axis=0).astype(np.float32)
    return cw


@pytest.mark.parametrize("storage", ["FP16_OFFSET", "BF16_OFFSET"])
@pytest.mark.parametrize("name", ["noslip_reverse", "ground_q15", "outlet_block", "wide_q15", "wide_nosdf"])
def test_aa_learned_closure_bit_identical_to_pingpong(gpu, name, storage):
    """The learned closure in place: the same MLP inputs, fallbacks and stored
    values as the ping-pong learned step, so fields, populations and the
    coverage probe agree bit for bit, with a live flow reversal."""
    case = BRANCHES[name]
    pp, aa = Sim(case, storage, "PINGPONG"), Sim(case, storage, "AA")
    pp.step(3)
    aa.step(3)
    cw = _closure_for(pp, 11)
    for sim in (pp, aa):
        sim.s.SetClosure(cw)
    cov = pp.s.ClosureCoverage()
    assert cov == aa.s.ClosureCoverage()
    fluid = int((~pp.solid).sum())
    assert 0 < cov["cells_in_range"] < fluid, cov  # both the MLP and the fallback run
    for sim in (pp, aa):
        sim.step(7)
    _compare(pp, aa, f"{name} learned after 10 steps")
    xa, na, ra = pp.s.ClosureProbe()
    xb, nb, rb = aa.s.ClosureProbe()
    assert _same(xa, xb) and _same(na, nb) and np.array_equal(ra, rb)
    for sim in (pp, aa):
        sim.set_params(_flip(case))
        sim.step(8)
    _compare(pp, aa, f"{name} learned after 18 steps")


def test_aa_learned_ignores_the_tensor_core_option(gpu):
    """FC_OPTION_TC_CLOSURE applies to the ping-pong bulk step; in place the
    learned step keeps the warp-level MLP, so the flag changes nothing."""
    from flowcraft_b200.lbm import (LatticeModel, LbmSolver, OPTION_TC_CLOSURE, Params, Storage, Streaming,
                                    VoxelGrid)
    case = BRANCHES["wide_q15"]
    ref = Sim(case, "FP16_OFFSET")
    cw = _closure_for(ref, 7)
    ref.s.SetClosure(cw)
    solid, sdf = geometry(case["geom"])
    nz, ny, nx = solid.shape
    s = LbmSolver()
    assert s.Init(0, VoxelGrid(nx, ny, nz, solid=solid, signedDistance=sdf), LatticeModel.D3Q15,
                  Storage.FP16_OFFSET, Streaming.AA, OPTION_TC_CLOSURE), s.LastError()
    s.Reset(_params(case["params"]), case["seed_mid"])
    s.SetClosure(cw)
    ref.step(9)
    s.Step(None, 9)
    assert _same(ref.s.SavePopulations(), s.SavePopulations())
    s.close()


def test_aa_learned_step_range_chunks(gpu):
    """StepRange chunks in place with the closure equal whole steps."""
    case = BRANCHES["wide_q15"]
    full, chunks = Sim(case, "FP16_OFFSET"), Sim(case, "FP16_OFFSET")
    cw = _closure_for(full, 5)
    for sim in (full, chunks):
        sim.s.SetClosure(cw)
    for _ in range(5):
        full.step(1)
        for z0 in range(0, 40, 13):
            chunks.s.StepRange(None, z0, 13)
        chunks.s.AdvanceSubstep()
    assert _same(full.s.SavePopulations(), chunks.s.SavePopulations())


def test_aa_step_range_chunks_and_warm_start(gpu):
    case = BRANCHES["wide_q15"]
    full, chunks = Sim(case), Sim(case)
    for _ in range(5):
        full.step(1)
        for z0 in range(0, 40, 13):
            chunks.s.StepRange(None, z0, 13)
        chunks.s.AdvanceSubstep()
    assert _same(full.readback_field(), chunks.readback_field())
    # warm start from the field at an odd parity, on both schemes
    pp = Sim(case, streaming="PINGPONG")
    pp.step(5)
    f = pp.readback_field()
    for sim in (pp, full):
        sim.reset_from_field(f)
        sim.step(6)
    assert _same(pp.readback_field(), full.readback_field())


@pytest.mark.parametrize("odd", [0, 1])
def test_aa_population_load_at_either_parity(gpu, odd):
    """A checkpoint loaded into an in-place lattice before an even or an odd
    step continues exactly as the ping-pong lattice it came from."""
    case = BRANCHES["outlet_block"]
    src = Sim(case, "FP16_OFFSET", "PINGPONG")
    src.step(10)
    pops = src.s.SavePopulations()
    aa = Sim(case, "FP16_OFFSET", "AA")
    aa.step(odd)
    aa.s.LoadPopulations(pops)
    src.step(9)
    aa.step(9)
    assert _same(src.readback_field(), aa.readback_field())


def test_aa_unsupported_combinations(gpu):
    from flowcraft_b200.batch import LbmBatch
    from flowcraft_b200.lbm import LbmSolver, Storage, Streaming, VoxelGrid, LatticeModel
    s = LbmSolver()
    g = VoxelGrid(9, 4, 4, solid=np.zeros(144, np.uint8))
    assert s.Init(0, g, LatticeModel.D3Q19, Storage.FP32, Streaming.AA) is False
    assert "even nx" in s.LastError()
    aa = Sim(BRANCHES["ywall"], "FP16_OFFSET", "AA")
    with pytest.raises(RuntimeError):
        aa.s.LayerCopy(0, 1, True)
    with pytest.raises(RuntimeError):
        LbmBatch([aa.s])


def test_aa_holds_one_population_set(gpu):
    import torch
    case = _sphere((256, 128, 128), (80, 64, 64), 12, 19)
    set_bytes = 19 * 256 * 128 * 128 * 4
    used = {}
    for mode in ("PINGPONG", "AA"):
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        sim = Sim(case, "FP32", mode)
        free1 = torch.cuda.mem_get_info()[0]
        used[mode] = free0 - free1
        sim.s.close()
    assert used["PINGPONG"] - used["AA"] > 0.9 * set_bytes, used
