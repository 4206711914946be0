"""The 16-bit formats and the learned closure over the plain-FP32 parity
configuration's full run: the 128x64x64 sphere (r 10, U 0.05, Re 100,
tau 0.53, Cs 0.1) for 1000 steps, FP16-offset storage with Smagorinsky and
with the learned closure, each against the FP64 oracle running the same
closure. The shorter checks in test_lbm_gpu.py and test_closure_gpu.py run
60 and 40 steps; this one shows the per-step storage rounding staying
bounded over the configuration's whole run instead of growing."""
import numpy as np
import pytest

from cases import CASES, OracleAdapter, geometry
from test_closure_gpu import _weights
from test_lbm_gpu import GpuAdapter

pytestmark = pytest.mark.gpu

STEPS = 1000


@pytest.mark.parametrize("learned", [False, True], ids=["smagorinsky", "learned"])
def test_fp16_offset_over_1000_steps_vs_fp64(gpu, oracle_built, learned):
    from flowcraft_b200.lbm import Storage
    case = CASES["c1_q19"]
    sim = GpuAdapter(case, storage=Storage.FP16_OFFSET)
    ref = OracleAdapter(case, "f64")
    if learned:
        probe = GpuAdapter(case, storage=Storage.FP16_OFFSET)
        probe.step(200)
        cw = _weights(probe)
        probe.s.close()
        sim.s.SetClosure(cw)
        ref.o.set_closure(cw)
    sim.step(STEPS)
    ref.step(STEPS)
    if learned:  # the closure covers most of the flow by the end of the run
        cov = sim.s.ClosureCoverage()
        assert cov["cell_fraction"] > 0.5
    g = sim.readback_field().reshape(-1, 4).astype(np.float64)
    r = ref.o.readback_field_f64().reshape(-1, 4)
    solid = geometry(case["geom"])[0].ravel().astype(bool)
    d = np.abs(g - r)[~solid]
    du = np.abs(np.linalg.norm(g[~solid, 1:], axis=1) - np.linalg.norm(r[~solid, 1:], axis=1))
    umax = np.linalg.norm(r[~solid, 1:], axis=1).max()
    print(f"{'learned' if learned else 'Smagorinsky'}: max|drho| {d[:, 0].max():.2e} max|du| {du.max():.2e} "
          f"rms|du| {np.sqrt((du ** 2).mean()):.2e} (|u| up to {umax:.3f})"
          + (f"; cells in the closure's range at the end {cov['cell_fraction']:.2f}" if learned else ""))
    assert np.isfinite(g).all() and not sim.s.HasDiverged()
    assert d[:, 0].max() < 1e-3 and du.max() < 1e-3
    assert np.sqrt((du ** 2).mean()) < 1e-4
    sim.s.close()
