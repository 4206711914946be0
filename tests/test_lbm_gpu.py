"""GPU parity tests: the CUDA path, called through the C ABI, against
FlowCraft's own LbmReference (golden fixtures) and the CPU oracle.

The FP32 path must reproduce LbmReference bit-for-bit on every golden case,
including the 128x64x64 sphere after 1000 steps (the contract asks for 1e-5
relative; the test checks that bound first, then bit-equality). The 16-bit
offset formats are checked against the FP64 oracle with stated tolerances.
"""
import numpy as np
import pytest

from cases import CASES, OracleAdapter, field_digest, geometry, load_fixture, run_schedule

pytestmark = pytest.mark.gpu


def _params(p: dict):
    from flowcraft_b200.lbm import Params
    return Params(tau=p["tau"], inletVelocity=p["inlet_velocity"], reverseFlow=bool(p.get("reverse_flow", 0)),
                  freeSlipY=bool(p.get("free_slip_y", 1)), freeSlipZ=bool(p.get("free_slip_z", 1)),
                  smagorinskyCs=p["smagorinsky_cs"])


class GpuAdapter:
    def __init__(self, case, storage=None):
        from flowcraft_b200.lbm import LatticeModel, LbmSolver, Storage, VoxelGrid
        solid, sdf = geometry(case["geom"])
        nz, ny, nx = solid.shape
        self.solid = solid
        self.s = LbmSolver()
        grid = VoxelGrid(nx, ny, nz, solid=solid, signedDistance=sdf)
        model = LatticeModel.D3Q19 if case["q"] == 19 else LatticeModel.D3Q15
        assert self.s.Init(0, grid, model, storage if storage is not None else Storage.FP32), self.s.LastError()
        self.s.Reset(_params(case["params"]), case["seed_mid"])

    def step(self, n):
        self.s.Step(None, n)

    def readback_field(self):
        return self.s.ReadbackField()

    def reset_from_field(self, field):
        self.s.ResetFromField(field)

    def set_params(self, p):
        self.s.SetParams(_params(p))


def _rel_err(a, b, solid):
    a = a.reshape(-1, 4)[~solid].astype(np.float64)
    b = b.reshape(-1, 4)[~solid].astype(np.float64)
    drho = np.abs(a[:, 0] - b[:, 0]).max() / np.abs(b[:, 0]).max()
    ua = np.linalg.norm(a[:, 1:], axis=1)
    ub = np.linalg.norm(b[:, 1:], axis=1)
    du = np.abs(ua - ub).max() / max(ub.max(), 1e-30)
    return drho, du


@pytest.mark.parametrize("name", list(CASES))
def test_fp32_matches_reference_bit_for_bit(gpu, name):
    case = CASES[name]
    fx = load_fixture(name)
    sim = GpuAdapter(case)
    got = []
    run_schedule(sim, case, lambda step, field: got.append((step, field.copy())))
    solid = geometry(case["geom"])[0].ravel().astype(bool)
    idx = np.array(fx["sample_idx"])
    assert len(got) == len(fx["checkpoints"])
    for (step, field), cp in zip(got, fx["checkpoints"]):
        assert step == cp["step"]
        assert np.isfinite(field).all()
        ref_sample = np.array(cp["sample_bits"], dtype=np.uint32).view(np.float32)
        drho, du = _rel_err(field.reshape(-1, 4)[idx].ravel(), ref_sample.ravel(), solid[idx])
        assert drho <= 1e-5 and du <= 1e-5, f"{name}@{step}: rel err rho {drho:.3e} |u| {du:.3e}"
        assert np.array_equal(field.view(np.uint32).reshape(-1, 4)[idx], np.array(cp["sample_bits"], np.uint32))
        assert field_digest(field) == cp["field_sha256"], f"{name}@{step}: not bit-identical to LbmReference"


def test_step_range_chunks_equal_full_steps(gpu):
    case = CASES["sphere48_q19"]
    a = GpuAdapter(case)
    b = GpuAdapter(case)
    a.step(12)
    chunks = [(0, 5), (5, 1), (6, 11), (17, 7)]
    for _ in range(12):
        for z0, zc in chunks:
            b.s.StepRange(None, z0, zc)
        b.s.AdvanceSubstep()
    assert np.array_equal(a.readback_field(), b.readback_field())


def test_foreign_stream(gpu):
    import torch
    case = CASES["sphere48_q15"]
    a = GpuAdapter(case)
    b = GpuAdapter(case)
    a.step(20)
    st = torch.cuda.Stream()
    b.s.Step(st, 20)
    assert np.array_equal(a.readback_field(), b.readback_field())


def test_readback_field_range_and_probe(gpu):
    case = CASES["sphere48_q19"]
    sim = GpuAdapter(case)
    sim.step(30)
    full = sim.readback_field()
    part = np.full_like(full, np.nan)
    for z0 in range(0, 24, 7):
        sim.s.ReadbackFieldRange(z0, 7, part)
    assert np.array_equal(full, part)
    assert sim.s.ProbeSliceHealth(12) is False
    assert sim.s.ProbeSliceHealth(-5) is False and sim.s.ProbeSliceHealth(999) is False  # clamped


@pytest.mark.parametrize("name", ["sphere48_q19", "wing_q15", "outlet_block_q19"])
def test_stats_match_reference(gpu, name):
    case = CASES[name]
    fx = load_fixture(name)
    sim = GpuAdapter(case)
    run_schedule(sim, case, lambda step, field: None)
    st = sim.s.ReadbackStats()
    ref = fx["checkpoints"][-1]["stats"]
    assert st.valid and st.hasNaN == bool(ref["has_nan"])
    for mine, k in ((st.avgDensity, "avg_density"), (st.minDensity, "min_density"), (st.maxDensity, "max_density"),
                    (st.avgSpeed, "avg_speed"), (st.maxSpeed, "max_speed"), (st.forceX, "force_x"),
                    (st.forceY, "force_y"), (st.forceZ, "force_z"), (st.maxStress, "max_stress"),
                    (st.totalMass, "total_mass")):
        assert mine == pytest.approx(ref[k], rel=2e-6, abs=1e-9), k


def test_populations_match_oracle_state(gpu, oracle_built):
    """Exhaustive state check: every population of every cell after 37 steps
    equals the oracle's (fluid cells bit-for-bit, solid cells w_i)."""
    for name in ("sphere48_q19", "ground_q15"):
        case = CASES[name]
        sim = GpuAdapter(case)
        ora = OracleAdapter(case)
        sim.step(37)
        ora.step(37)
        assert np.array_equal(sim.s.SavePopulations().view(np.uint32), ora.o.populations().view(np.uint32))


def test_save_load_roundtrip_continues_identically(gpu):
    case = CASES["sphere48_q19"]
    a = GpuAdapter(case)
    a.step(15)
    pops = a.s.SavePopulations()
    a.step(15)
    b = GpuAdapter(case)
    b.s.LoadPopulations(pops)
    b.step(15)
    assert np.array_equal(a.readback_field(), b.readback_field())


def test_reset_from_field_mismatch_is_ignored(gpu):
    sim = GpuAdapter(CASES["tiny_q15"])
    sim.step(4)
    before = sim.readback_field()
    sim.s.ResetFromField(np.zeros(13, dtype=np.float32))  # LbmSolver.cpp:430 ignores it
    assert np.array_equal(sim.readback_field(), before)


@pytest.mark.parametrize("storage", ["FP32", "FP16_OFFSET"])
def test_probe_verdict_matches_host_check_of_the_field(gpu, storage):
    """ProbeSliceHealth evaluates the reference's checks (LbmSolver.cpp:699-716)
    on the device. Its verdict for every layer must equal those checks run on
    the host over the read-back field: any value not finite, or a fluid cell
    with rho <= 0 or |u|^2 > 4. The state is seeded with a NaN density, an
    excess speed and a negative density in three different layers."""
    from flowcraft_b200.lbm import Storage
    case = CASES["sphere48_q19"]
    sim = GpuAdapter(case, storage=Storage[storage])
    sim.step(5)
    nz, ny, nx = geometry(case["geom"])[0].shape
    solid = geometry(case["geom"])[0].reshape(nz, ny * nx).astype(bool)
    field = sim.readback_field().reshape(nz, ny * nx, 4).copy()
    fluid_y = np.nonzero(~solid[10])[0]
    field[10, fluid_y[5], 0] = np.nan
    field[12, fluid_y[7], 1:4] = (1.5, 1.0, 0.5)  # |u|^2 = 3.5: inside the bound
    field[13, fluid_y[9], 1:4] = (1.6, 1.2, 0.6)  # |u|^2 = 4.36
    field[15, fluid_y[11], 0] = -0.5
    sim.reset_from_field(field.ravel())
    got = sim.readback_field().reshape(nz, ny * nx, 4)
    for z in range(nz):
        v = got[z]
        sp2 = (v[:, 1] * v[:, 1] + v[:, 2] * v[:, 2]) + v[:, 3] * v[:, 3]
        want = (not np.isfinite(v).all()) or bool(np.any(~solid[z] & ((v[:, 0] <= 0) | (sp2 > 4.0))))
        assert sim.s.ProbeSliceHealth(z) is want, z
    assert [sim.s.ProbeSliceHealth(z) for z in (10, 12, 13, 15)] == [True, False, True, True]


def test_divergence_detection_from_host_injected_state(gpu, oracle_built):
    """Failure detection without a GPU fault: host-prepared fields with a NaN
    cell, and with a 3x3x3 block at negative density, are seeded through
    ResetFromField; the step's device flag and the slice probe report them
    exactly when the reference's divergence test (LbmReference.cpp:397-400)
    does, and Reset clears the flag."""
    case = CASES["sphere48_q19"]
    sim = GpuAdapter(case)
    sim.step(5)
    assert sim.s.HasDiverged() is False
    base = sim.readback_field().reshape(-1, 4).copy()
    nx, ny = 48, 24
    cell = lambda x, y, z: (z * ny + y) * nx + x  # noqa: E731

    def inject(field):
        sim.reset_from_field(field.ravel())
        ora = OracleAdapter(case)
        ora.reset_from_field(field.ravel())
        return ora

    f1 = base.copy()
    f1[cell(30, 3, 10), 0] = np.nan
    ora = inject(f1)
    assert sim.s.HasDiverged() is False
    assert sim.s.ProbeSliceHealth(10) is True and sim.s.ProbeSliceHealth(2) is False
    sim.step(1)
    ora.step(1)
    assert sim.s.HasDiverged() is True and ora.o.has_diverged()

    sim.s.Reset(_params(case["params"]), True)
    assert sim.s.HasDiverged() is False
    f2 = base.copy()
    single = f2.copy()
    single[cell(30, 3, 10), 0] = -1.0  # one cell: its neighbours stay positive
    ora = inject(single)
    sim.step(1)
    ora.step(1)
    assert sim.s.HasDiverged() is bool(ora.o.has_diverged()) is False
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                f2[cell(30 + dx, 4 + dy, 10 + dz), 0] = -1.0
    ora = inject(f2)
    assert sim.s.ProbeSliceHealth(10) is True
    sim.step(1)
    ora.step(1)
    assert sim.s.HasDiverged() is bool(ora.o.has_diverged()) is True


def test_wing_cross_check(gpu):
    """gpu_vs_cpu_test.cpp:149-172 on the CUDA path (see the oracle test for
    why lift is read one step early / averaged)."""
    s = {}
    for q in (19, 15):
        sim = GpuAdapter(CASES[f"wing_q{q}"])
        sim.step(79)
        assert sim.s.ReadbackStats().forceZ > 0
        sim.step(1)
        s[q] = sim.s.ReadbackStats()
        assert s[q].forceX > 0 and not s[q].hasNaN
    assert abs(s[19].avgSpeed - s[15].avgSpeed) < 0.005


@pytest.mark.parametrize("storage,tol_u,tol_rho", [("FP16_OFFSET", 2e-4, 2e-4), ("BF16_OFFSET", 2e-3, 2e-3)])
def test_offset_storage_error_vs_fp64(gpu, oracle_built, storage, tol_u, tol_rho):
    """16-bit (f_i - w_i)*2^8 storage, FP32 collision: error against the FP64
    oracle on the reference test case (60 steps). Per-step rounding of the
    stored offsets is ~5e-6 (FP16) / ~4e-5 (BF16) per population and adds up
    like a random walk over the steps. The reference's own GPU check allows
    1e-2 for its plain FP16 storage (gpu_vs_cpu_test.cpp:76)."""
    from flowcraft_b200.lbm import Storage
    for q in (19, 15):
        case = CASES[f"sphere48_q{q}"]
        sim = GpuAdapter(case, storage=Storage[storage])
        ref = OracleAdapter(case, "f64")
        sim.step(60)
        ref.step(60)
        g = sim.readback_field().reshape(-1, 4).astype(np.float64)
        r = ref.o.readback_field_f64().reshape(-1, 4)
        solid = geometry(case["geom"])[0].ravel().astype(bool)
        d = np.abs(g - r)[~solid]
        assert np.isfinite(g).all()
        print(f"{storage} D3Q{q}: max|drho| {d[:, 0].max():.3e}  max|du| {d[:, 1:].max():.3e}")
        assert d[:, 0].max() < tol_rho, d[:, 0].max()
        assert d[:, 1:].max() < tol_u, d[:, 1:].max()


def test_init_errors(gpu):
    from flowcraft_b200.lbm import LbmSolver, VoxelGrid
    s = LbmSolver()
    g = VoxelGrid(8, 4, 4, solid=np.zeros(128, np.uint8))
    assert s.Init(99, g) is False and "device" in s.LastError()
    # 4.2e9 cells fit the index type but not the device: clean refusal, no allocation
    big = VoxelGrid(2048, 2048, 1000, solid=np.zeros(1, np.uint8))
    assert s.Init(0, big) is False and "GiB" in s.LastError()
    assert s.Init(0, g) is True and s.IsValid() and s.Nx() == 8
    assert np.array_equal(s.SolidMask(), g.solid)
    s.Shutdown()
    assert not s.IsValid()


# Lattice shapes that route cells through every bulk-kernel variant: even nx
# with an odd number of interior 32-cell chunks (the two-cell interior kernel
# with a half-masked last group), odd nx (the one-cell interior kernel), a
# single interior chunk, and the shell (faces, inlet/outlet warps).
SHAPES = [
    ("even_masked", (160, 40, 40), (52.0, 20.0, 20.0, 7.0), dict(tau=0.56, inlet_velocity=0.06, smagorinsky_cs=0.1)),
    ("odd", (161, 41, 39), (50.3, 19.7, 20.2, 6.5),
     dict(tau=0.6, inlet_velocity=0.05, smagorinsky_cs=0.12, free_slip_y=0, reverse_flow=1)),
    ("one_chunk", (96, 20, 24), (30.0, 10.0, 12.0, 4.5),
     dict(tau=0.58, inlet_velocity=0.05, smagorinsky_cs=0.12, free_slip_z=0)),
]


def _shape_case(shape, sphere, params, q=19):
    nx, ny, nz = shape
    return dict(geom={"kind": "sphere", "dims": [nx, ny, nz], "center": list(sphere[:3]), "r": sphere[3]}, q=q,
                params=params, seed_mid=True, steps=[40])


@pytest.mark.parametrize("name,shape,sphere,params", SHAPES, ids=[s[0] for s in SHAPES])
@pytest.mark.parametrize("q", [19, 15])
def test_fp32_bit_exact_all_kernel_variants(gpu, oracle_built, name, shape, sphere, params, q):
    case = _shape_case(shape, sphere, params, q)
    sim = GpuAdapter(case)
    ora = OracleAdapter(case)
    sim.step(40)
    ora.step(40)
    g, r = sim.readback_field(), ora.readback_field()
    assert np.array_equal(g.view(np.uint32), r.view(np.uint32)), f"{name} D3Q{q}: differs from the oracle"
    info = sim.s.BoundaryInfo()
    assert info["bulk_cells"] > 0 and info["boundary_cells"] > 0


@pytest.mark.parametrize("storage,tol", [("FP16_OFFSET", 2e-4), ("BF16_OFFSET", 2e-3)])
def test_offset_storage_two_cell_kernel_vs_fp64(gpu, oracle_built, storage, tol):
    """The 16-bit formats through the two-cell interior kernel (even nx with
    interior chunks), against the FP64 oracle."""
    from flowcraft_b200.lbm import Storage
    name, shape, sphere, params = SHAPES[0]
    case = _shape_case(shape, sphere, params)
    sim = GpuAdapter(case, storage=Storage[storage])
    ref = OracleAdapter(case, "f64")
    sim.step(60)
    ref.step(60)
    g = sim.readback_field().reshape(-1, 4).astype(np.float64)
    r = ref.o.readback_field_f64().reshape(-1, 4)
    solid = geometry(case["geom"])[0].ravel().astype(bool)
    d = np.abs(g - r)[~solid]
    print(f"{storage} {shape}: max|drho| {d[:, 0].max():.3e}  max|du| {d[:, 1:].max():.3e}")
    assert np.isfinite(g).all() and d[:, 0].max() < tol and d[:, 1:].max() < tol
