"""Pins the restated CPU oracle (oracle/lbm_oracle.c) to FlowCraft's own
LbmReference: every checkpoint of every golden case must reproduce the
reference's full field bit-for-bit (SHA-256) and its statistics."""
import numpy as np
import pytest

from cases import CASES, OracleAdapter, field_digest, geometry, input_digest, load_fixture, run_schedule


def _cases_cpu():
    for name, case in CASES.items():
        if name == "c1_q19":  # 1000 steps; the CPU suite checks its first checkpoint only
            c = dict(case)
            c["steps"] = case["steps"][:1]
            yield name, c
        else:
            yield name, case


@pytest.mark.parametrize("name,case", list(_cases_cpu()), ids=[n for n, _ in _cases_cpu()])
def test_oracle_matches_reference_fixture(oracle_built, name, case):
    fx = load_fixture(name)
    solid, sdf = geometry(case["geom"])
    assert input_digest(solid, sdf) == fx["input_sha256"], "geometry builder drifted from the fixture"
    sim = OracleAdapter(case, precision="f32")
    got = []
    run_schedule(sim, case, lambda step, field: got.append((step, field_digest(field), sim.stats(),
                                                            field.view(np.uint32).reshape(-1, 4))))
    for (step, digest, stats, bits), cp in zip(got, fx["checkpoints"]):
        assert step == cp["step"]
        idx = np.array(fx["sample_idx"])
        assert np.array_equal(bits[idx], np.array(cp["sample_bits"], dtype=np.uint32)), f"{name}@{step} sample"
        assert digest == cp["field_sha256"], f"{name}@{step}: field differs from LbmReference"
        for k in ("avg_density", "min_density", "max_density", "avg_speed", "max_speed", "force_x", "force_y",
                  "force_z", "max_stress", "total_mass"):
            assert stats[k] == pytest.approx(cp["stats"][k], rel=1e-6, abs=1e-9), k
        assert stats["has_nan"] == cp["stats"]["has_nan"]
        assert bool(sim.o.has_diverged()) == cp["diverged"]


def test_reference_test_tolerances_and_f64(oracle_built):
    """The reference test's own pass criteria (gpu_vs_cpu_test.cpp:63-77),
    here between the FP32 oracle and the FP64 oracle, with much tighter
    bounds: FP32 LbmReference is within 1e-5 of the FP64 restatement."""
    case = CASES["sphere48_q19"]
    a = OracleAdapter(case, "f32")
    b = OracleAdapter(case, "f64")
    a.step(60)
    b.step(60)
    fa = a.o.readback_field().reshape(-1, 4).astype(np.float64)
    fb = b.o.readback_field_f64().reshape(-1, 4)
    solid = geometry(case["geom"])[0].ravel().astype(bool)
    d = np.abs(fa - fb)[~solid]
    assert np.isfinite(fa).all()
    assert d[:, 0].max() < 1e-5 and d[:, 1:].max() < 1e-5 and d[:, 1:].mean() < 1e-6


def test_reference_wing_force_signs(oracle_built):
    """gpu_vs_cpu_test.cpp:149-172 asks for drag > 0 and lift > 0 after 80
    steps and |avgSpeed19 - avgSpeed15| < 0.005. Lift still oscillates
    through zero at step 80 (start-up acoustics): the reference's GPU kernel
    computes the solid-cell force from the previous step's populations
    (shaders/lbm_step.comp.glsl:144), so its step-80 reading is the CPU
    solver's step-79 value, which is positive, while the CPU value at step 80
    is not. Restated on quantities that do not flip sign: drag at 80, the
    one-step-lagged lift, and lift averaged over steps 300-400."""
    s = {}
    for q in (19, 15):
        fx = load_fixture(f"wing_q{q}")
        s[q] = fx["checkpoints"][-1]["stats"]
        assert s[q]["force_x"] > 0 and not s[q]["has_nan"]
    assert abs(s[19]["avg_speed"] - s[15]["avg_speed"]) < 0.005
    for q in (19, 15):
        sim = OracleAdapter(CASES[f"wing_q{q}"], "f32")
        sim.step(79)
        assert sim.stats()["force_z"] > 0  # what the lagged GPU force reports at step 80
        sim.step(221)
        lift = []
        for _ in range(10):
            sim.step(10)
            st = sim.stats()
            lift.append(st["force_z"])
            assert st["force_x"] > 0
        assert np.mean(lift) > 0


def test_oracle_reset_from_field_size_mismatch_is_ignored(oracle_built):
    case = CASES["tiny_q15"]
    sim = OracleAdapter(case)
    sim.step(3)
    before = sim.readback_field()
    assert sim.o.reset_from_field(np.zeros(7, dtype=np.float32)) == -1
    assert np.array_equal(sim.readback_field(), before)
