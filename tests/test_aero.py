"""The aerodynamic force integral (FieldOverlay::ComputeAerodynamicForces,
FieldOverlay.cpp:469-621): the oracle's restatement against the values
FlowCraft's own code produced (tests/golden/aero_golden.json), and the
device FP64 integral (fc_lbm_aero_forces) against both."""
import json
import os

import numpy as np
import pytest

from cases import CASES, OracleAdapter, geometry
from conftest import ROOT

with open(os.path.join(ROOT, "tests", "golden", "aero_golden.json")) as _f:
    GOLDEN = json.load(_f)["cases"]


def _close(a, b, rel=2e-6, abs_=1e-9):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return np.all(np.abs(a - b) <= abs_ + rel * np.abs(b))


def _oracle_state(fx):
    case = CASES[fx["case"]]
    solid, _ = geometry(case["geom"])
    sim = OracleAdapter(case, precision="f32")
    sim.step(fx["steps"])
    return solid, sim.readback_field()


@pytest.mark.parametrize("i", range(len(GOLDEN)))
def test_oracle_aero_matches_reference(oracle_built, i):
    fx = GOLDEN[i]
    solid, field = _oracle_state(fx)
    a = oracle_built.aero_forces(solid, field, fx["cell_size"], fx["origin"])
    assert _close(a["force"], fx["force"])
    assert _close(a["center_of_pressure"], fx["center_of_pressure"])
    assert _close(a["lift_arrow_base"], fx["lift_arrow_base"])
    assert a["min_stress"] == fx["min_stress"] and a["max_stress"] == fx["max_stress"]
    assert a["has_nan"] == fx["has_nan"]


@pytest.mark.gpu
@pytest.mark.parametrize("i", range(len(GOLDEN)))
def test_device_aero_matches_reference_and_oracle(gpu, oracle_built, i):
    from flowcraft_b200.lbm import LatticeModel, LbmSolver, VoxelGrid
    from test_lbm_gpu import _params
    fx = GOLDEN[i]
    case = CASES[fx["case"]]
    solid, sdf = geometry(case["geom"])
    nz, ny, nx = solid.shape
    g = VoxelGrid(nx, ny, nz, fx["cell_size"], tuple(fx["origin"]), solid.ravel(), sdf.ravel())
    s = LbmSolver()
    model = LatticeModel.D3Q19 if case["q"] == 19 else LatticeModel.D3Q15
    assert s.Init(0, g, model), s.LastError()
    s.Reset(_params(case["params"]), case["seed_mid"])
    s.Step(None, fx["steps"])
    a = s.AerodynamicForces()
    s.close()
    assert _close((a.forceX, a.forceY, a.forceZ), fx["force"])
    assert _close(a.centerOfPressure, fx["center_of_pressure"])
    assert _close(a.liftArrowBase, fx["lift_arrow_base"])
    assert a.minStress == fx["min_stress"] and a.maxStress == fx["max_stress"]
    assert a.hasNaN == fx["has_nan"]
    osolid, ofield = _oracle_state(fx)
    o = oracle_built.aero_forces(osolid, ofield, fx["cell_size"], fx["origin"])
    # FP64 sums of identical float terms in a different order
    assert _close(a.forceSum, o["force_sum"], rel=1e-11, abs_=1e-12)
    assert _close(a.liftWeightSum, o["lift_weight_sum"], rel=1e-11)
    assert a.solidCells == o["solid_cells"]
