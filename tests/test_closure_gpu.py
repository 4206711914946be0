"""The learned closure fused into the collision (fc_lbm_set_closure):
its wall-distance input bit-exact against the oracle, its inputs and BF16
tensor-core inference against the oracle's restatement, whole steps with the
closure against the FP64 oracle running the same closure, and the per-cell
Smagorinsky fallback bit-identical to the plain kernels."""
import numpy as np
import pytest

from cases import CASES, OracleAdapter, geometry
from test_lbm_gpu import SHAPES, GpuAdapter, _shape_case

pytestmark = pytest.mark.gpu


def _weights(sim, seed=1, out_scale=2e-3):
    """Random weights normalized to the lattice's own input statistics."""
    from flowcraft_b200.closure import ClosureWeights
    cw = ClosureWeights.random(seed, out_scale)
    sim.s.SetClosure(cw)
    x, _, _ = sim.s.ClosureProbe()
    fluid = ~sim.solid.ravel().astype(bool)
    cw.mean[:4] = x[fluid].mean(axis=0)
    cw.std[:4] = np.maximum(x[fluid].std(axis=0), 1e-3)
    cw.mean[4], cw.std[4], cw.filter_width = 1.0, 1.0, 1.0
    lo, hi = np.percentile(x[fluid][:, :3], 0.5, axis=0), np.percentile(x[fluid][:, :3], 99.5, axis=0)
    cw.lo, cw.hi = lo.astype(np.float32), hi.astype(np.float32)
    return cw


def test_wall_distance_matches_oracle(gpu, oracle_built):
    from flowcraft_b200.lbm import Storage
    for case in (CASES["wing_q19"], _shape_case(*SHAPES[0][1:])):
        sim = GpuAdapter(case, storage=Storage.FP16_OFFSET)
        want = oracle_built.wall_distance(sim.solid)
        assert np.array_equal(sim.s.WallDistance(), want.ravel())
        sim.s.close()


def test_closure_refused_where_unsupported(gpu):
    from flowcraft_b200.closure import ClosureWeights
    from flowcraft_b200.lbm import LbmError, Storage
    sim = GpuAdapter(CASES["sphere48_q19"], storage=Storage.FP32)
    with pytest.raises(LbmError):
        sim.s.SetClosure(ClosureWeights.random(0))
    odd = _shape_case(*SHAPES[1][1:])
    sim = GpuAdapter(odd, storage=Storage.FP16_OFFSET)
    with pytest.raises(LbmError):
        sim.s.SetClosure(ClosureWeights.random(0))


LATTICE = {19: [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1), (1, 1, 0),
                (-1, -1, 0), (1, -1, 0), (-1, 1, 0), (1, 0, 1), (-1, 0, -1), (1, 0, -1), (-1, 0, 1), (0, 1, 1),
                (0, -1, -1), (0, 1, -1), (0, -1, 1)],
           15: [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1), (1, 1, 1),
                (-1, -1, -1), (1, 1, -1), (-1, -1, 1), (1, -1, 1), (-1, 1, -1), (-1, 1, 1), (1, -1, -1)]}


def _recompute_inputs(pops, q):
    """Inputs 0-2 from decoded populations in float64 (closure.cuh definitions)."""
    e = np.asarray(LATTICE[q], np.float64)
    f = pops.astype(np.float64)
    rho = f.sum(axis=0)
    u = (e.T @ f) / rho
    s = np.einsum("ia,ib,ic->abc", e, e, f)
    pi = s - rho * (np.eye(3)[:, :, None] / 3.0) - rho * np.einsum("ac,bc->abc", u, u)
    pp = np.einsum("abc,abc->c", pi, pi)
    mag = np.sqrt(pp)
    safe = np.where(mag > 0, mag, 1.0)
    x0 = np.log2(mag / rho + 1e-12)
    x1 = np.where(mag > 0, np.trace(pi) / safe, 0)
    x2 = np.where(mag > 0, np.linalg.det(np.moveaxis(pi, 2, 0)) / safe ** 3, 0)
    return np.stack([x0, x1, x2], axis=1), mag / rho


@pytest.mark.parametrize("q", [19, 15])
def test_probe_inputs_and_inference(gpu, oracle_built, q):
    from flowcraft_b200.lbm import Storage
    case = _shape_case(*SHAPES[0][1:], q=q)
    sim = GpuAdapter(case, storage=Storage.FP16_OFFSET)
    sim.step(30)
    cw = _weights(sim)
    sim.s.SetClosure(cw)
    x, nu, in_range = sim.s.ClosureProbe()
    fluid = ~sim.solid.ravel().astype(bool)
    # inputs 0-2 against a float64 recomputation from the stored populations
    want, q_mag = _recompute_inputs(sim.s.SavePopulations(), q)
    strong = fluid & (q_mag > 1e-5)
    assert strong.sum() > 1000
    assert np.abs(x[strong, 0] - want[strong, 0]).max() < 2e-3
    assert np.abs(x[strong, 1:3] - want[strong, 1:3]).max() < 2e-3
    # input 3 is the wall-distance byte / 16
    assert np.array_equal(x[:, 3], sim.s.WallDistance().astype(np.float32) * np.float32(0.0625))
    # nu_t against the oracle's BF16 restatement on the device's own inputs
    o = oracle_built.Oracle(sim.solid, None, q, oracle_built.Params(), precision="f32")
    o.set_closure(cw, wall=sim.s.WallDistance())
    ref = o.closure_eval(x)
    o.close()
    assert np.array_equal(ref >= 0, in_range)
    sel = fluid & in_range
    assert sel.sum() > 0.8 * fluid.sum()
    err = np.abs(nu[sel] - ref[sel]) / (np.abs(ref[sel]) + 1e-6)
    print(f"D3Q{q}: nu_t mean {ref[sel].mean():.3e}, rel err median {np.median(err):.2e} max {err.max():.2e}")
    assert np.median(err) < 1e-3 and np.quantile(err, 0.999) < 3e-2
    # the coverage counters agree with the probe
    cov = sim.s.ClosureCoverage()
    assert cov["cells_in_range"] == int(in_range.sum())
    n = len(in_range)
    groups = np.pad(in_range, (0, (-n) % 64)).reshape(-1, 64).any(axis=1)
    assert cov["warps_with_mlp"] == int(groups.sum())


@pytest.mark.parametrize("storage,tol,margin", [("FP16_OFFSET", 3e-4, 5.0), ("BF16_OFFSET", 2e-3, 2.0)])
@pytest.mark.parametrize("q", [19, 15])
def test_step_with_closure_vs_fp64_oracle(gpu, oracle_built, storage, tol, margin, q):
    """40 steps with the learned closure on the GPU (16-bit storage) against
    the FP64 oracle running the same closure; the closure must also change
    the flow by more than the storage error (`margin` times it) against plain
    Smagorinsky."""
    from flowcraft_b200.lbm import Storage
    case = _shape_case(*SHAPES[0][1:], q=q)
    probe = GpuAdapter(case, storage=Storage[storage])
    probe.step(30)
    cw = _weights(probe)
    probe.s.close()
    sim = GpuAdapter(case, storage=Storage[storage])
    sim.s.SetClosure(cw)
    ref = OracleAdapter(case, "f64")
    ref.o.set_closure(cw)
    plain = OracleAdapter(case, "f64")
    sim.step(40)
    ref.step(40)
    plain.step(40)
    g = sim.readback_field().reshape(-1, 4).astype(np.float64)
    r = ref.o.readback_field_f64().reshape(-1, 4)
    p = plain.o.readback_field_f64().reshape(-1, 4)
    solid = geometry(case["geom"])[0].ravel().astype(bool)
    d = np.abs(g - r)[~solid]
    effect = np.abs(p - r)[~solid]
    print(f"{storage} D3Q{q}: max|drho| {d[:, 0].max():.3e} max|du| {d[:, 1:].max():.3e}; "
          f"closure effect max|du| {effect[:, 1:].max():.3e}")
    assert np.isfinite(g).all()
    assert d[:, 0].max() < tol and d[:, 1:].max() < tol
    assert effect[:, 1:].max() > margin * d[:, 1:].max()


@pytest.mark.parametrize("shape_idx,q", [(0, 19), (2, 19), (0, 15)])
@pytest.mark.parametrize("storage,tol", [("FP16_OFFSET", 3e-4), ("BF16_OFFSET", 2e-3)])
def test_tensor_core_closure(gpu, oracle_built, shape_idx, q, storage, tol):
    """FC_OPTION_TC_CLOSURE: the bulk step's MLP once per block on the tcgen05
    tensor cores. The same BF16 operands and the same FP32 accumulation give
    the warp-level MMA path's results bit for bit, and against the FP64
    oracle running the same closure it keeps the tolerance of the warp-level
    path. The 96 x 20 x 24 lattice has a block row past the lattice and lanes
    past the row end."""
    from flowcraft_b200.lbm import (LatticeModel, LbmSolver, OPTION_TC_CLOSURE, Params, Storage, Streaming,
                                    VoxelGrid)
    case = _shape_case(*SHAPES[shape_idx][1:], q=q)
    probe = GpuAdapter(case, storage=Storage[storage])
    probe.step(30)
    cw = _weights(probe)
    probe.s.close()
    solid, sdf = geometry(case["geom"])
    nz, ny, nx = solid.shape
    p = case["params"]
    prm = Params(tau=p["tau"], inletVelocity=p["inlet_velocity"], reverseFlow=bool(p.get("reverse_flow", 0)),
                 freeSlipY=bool(p.get("free_slip_y", 1)), freeSlipZ=bool(p.get("free_slip_z", 1)),
                 smagorinskyCs=p["smagorinsky_cs"])
    sims = []
    for flags in (OPTION_TC_CLOSURE, 0):
        s = LbmSolver()
        assert s.Init(0, VoxelGrid(nx, ny, nz, solid=solid, signedDistance=sdf),
                      LatticeModel.D3Q19 if q == 19 else LatticeModel.D3Q15, Storage[storage], Streaming.PINGPONG,
                      flags), s.LastError()
        s.Reset(prm, case["seed_mid"])
        s.SetClosure(cw)
        sims.append(s)
    assert sims[0].ClosureCoverage()["cells_in_range"] > 0
    ref = OracleAdapter(case, "f64")
    ref.o.set_closure(cw)
    for s in sims:
        s.Step(None, 40)
    ref.step(40)
    fl = ~solid.ravel().astype(bool)
    g_tc, g_w = (s.ReadbackField().reshape(-1, 4).astype(np.float64) for s in sims)
    r = ref.o.readback_field_f64().reshape(-1, 4)
    d_w = np.abs(g_tc - g_w)[fl].max()
    d_r = np.abs(g_tc - r)[fl].max()
    print(f"{storage} D3Q{q} {SHAPES[shape_idx][0]}: tcgen05 vs warp MMA max |d| {d_w:.2e}, "
          f"vs FP64 oracle {d_r:.2e}")
    assert np.isfinite(g_tc).all() and not sims[0].HasDiverged()
    assert np.array_equal(g_tc.astype(np.float32).view(np.uint32), g_w.astype(np.float32).view(np.uint32))
    assert np.array_equal(sims[0].SavePopulations().view(np.uint32), sims[1].SavePopulations().view(np.uint32))
    assert d_r < tol
    for s in sims:
        s.close()


def test_fallback_reproduces_smagorinsky(gpu):
    """With a training range no cell falls into, every cell keeps the
    Smagorinsky tau_eff. The learned kernels collide every cell on the stored
    offsets, while the plain kernels collide single wall-adjacent cells on
    decoded populations: the FP32 results differ in the last bits, which now
    and then moves a stored 16-bit value by one step (about 4e-6 to 1.5e-5 in
    f here for FP16, 8x that for BF16), so the runs agree to a few storage
    steps, not bit for bit; the closure's own effect on this case is about
    1e-3."""
    from flowcraft_b200.closure import ClosureWeights
    from flowcraft_b200.lbm import Storage
    case = _shape_case(*SHAPES[0][1:])
    for storage, tol in ((Storage.FP16_OFFSET, 5e-5), (Storage.BF16_OFFSET, 4e-4)):
        a = GpuAdapter(case, storage=storage)
        b = GpuAdapter(case, storage=storage)
        cw = ClosureWeights.random(3)
        cw.lo[:] = 1e30
        cw.hi[:] = 1e30
        b.s.SetClosure(cw)
        _, _, in_range = b.s.ClosureProbe()
        assert not in_range.any()
        a.step(25)
        b.step(25)
        pa, pb = a.s.SavePopulations(), b.s.SavePopulations()
        diff = np.abs(pa.astype(np.float64) - pb)
        print(f"{storage.name}: fallback vs plain max |df| {diff.max():.2e}, equal {np.mean(pa == pb):.4f}")
        assert diff.max() < tol and np.mean(pa == pb) > 0.8
        b.s.SetClosure(None)
        a.step(5)
        b.step(5)
        assert np.abs(a.readback_field().astype(np.float64) - b.readback_field()).max() < 4 * tol


@pytest.mark.parametrize("wall_min,trust", [(2.0, 0.0), (0.0, 1.5), (1.5, 2.0)])
def test_near_wall_fallback_and_anchoring_vs_fp64_oracle(gpu, oracle_built, wall_min, trust):
    """The closure's near-wall Smagorinsky fallback (cells nearer a wall than
    wall_min cells) and its Smagorinsky trust band (3 nu_t within a factor
    `trust`): 40 FP16 steps against the FP64 oracle running the same rules;
    the probe leaves the near-wall cells out of the covered set; and the same
    rules under in-place AA streaming give the ping-pong result bit for bit."""
    from flowcraft_b200.lbm import LatticeModel, LbmSolver, Params, Storage, Streaming, VoxelGrid
    case = _shape_case(*SHAPES[0][1:], q=19)
    probe = GpuAdapter(case, storage=Storage.FP16_OFFSET)
    probe.step(30)
    cw = _weights(probe)
    cw.wall_min, cw.trust = wall_min, trust
    probe.s.SetClosure(cw)
    x, _, in_range = probe.s.ClosureProbe()
    near = x[:, 3] < wall_min
    assert not in_range[near].any()
    if wall_min > 0:
        assert near[~probe.solid.ravel().astype(bool)].sum() > 0
    probe.s.close()
    sim = GpuAdapter(case, storage=Storage.FP16_OFFSET)
    sim.s.SetClosure(cw)
    ref = OracleAdapter(case, "f64")
    ref.o.set_closure(cw)
    sim.step(40)
    ref.step(40)
    g = sim.readback_field().reshape(-1, 4).astype(np.float64)
    r = ref.o.readback_field_f64().reshape(-1, 4)
    solid = geometry(case["geom"])[0].ravel().astype(bool)
    d = np.abs(g - r)[~solid]
    print(f"wall_min {wall_min} trust {trust}: max|drho| {d[:, 0].max():.3e} max|du| {d[:, 1:].max():.3e}")
    assert np.isfinite(g).all()
    assert d[:, 0].max() < 3e-4 and d[:, 1:].max() < 3e-4
    # in place: bit-identical populations
    s, sdf_solid = geometry(case["geom"])
    nz, ny, nx = s.shape
    p = case["params"]
    prm = Params(tau=p["tau"], inletVelocity=p["inlet_velocity"], reverseFlow=bool(p.get("reverse_flow", 0)),
                 freeSlipY=bool(p.get("free_slip_y", 1)), freeSlipZ=bool(p.get("free_slip_z", 1)),
                 smagorinskyCs=p["smagorinsky_cs"])
    aa = LbmSolver()
    assert aa.Init(0, VoxelGrid(nx, ny, nz, solid=s, signedDistance=sdf_solid), LatticeModel.D3Q19,
                   Storage.FP16_OFFSET, Streaming.AA), aa.LastError()
    aa.Reset(prm, case["seed_mid"])
    aa.SetClosure(cw)
    aa.Step(None, 40)
    assert np.array_equal(aa.SavePopulations(), sim.s.SavePopulations())
    aa.close()
    sim.s.close()
