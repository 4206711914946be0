"""The CUDA voxelizer (fc_lbm_voxel_grid / fc_lbm_voxelize) against
FlowCraft's Voxelizer::Voxelize: bit-identical solid masks and signed
distances on the reference's own golden digests, and on the explicit-grid edge
cases against the oracle, in host and device memory; then the voxelized
c1 obstacle through the solver, bit-exact against the oracle solver."""
import json
import os

import numpy as np
import pytest

from conftest import ROOT
from voxel_cases import EXPLICIT, GOLDEN, digest, mesh

pytestmark = pytest.mark.gpu


def _golden():
    with open(os.path.join(ROOT, "tests", "golden", "voxel_golden.json")) as f:
        return json.load(f)["cases"]


def _host(a):
    return a.cpu().numpy() if hasattr(a, "cpu") else np.asarray(a)


@pytest.mark.parametrize("device", [None, 0], ids=["host", "device"])
@pytest.mark.parametrize("name", sorted(GOLDEN))
def test_voxelize_matches_reference_golden(gpu, name, device):
    from flowcraft_b200.voxelizer import Params, Voxelize
    case, fx = GOLDEN[name], _golden()[name]
    pos, idx = mesh(case["mesh"])
    g = Voxelize(pos, idx, Params(case["res"], case.get("padding", (0.3, 1.0, 0.5))), device=device)
    assert [g.nx, g.ny, g.nz] == fx["dims"]
    assert int(np.float32(g.cellSize).view(np.uint32)) == fx["cell_bits"]
    assert [int(v) for v in np.asarray(g.origin, np.float32).view(np.uint32)] == fx["origin_bits"]
    solid, sdf = _host(g.solid), _host(g.signedDistance)
    assert int(solid.sum()) == fx["solid_cells"]
    assert digest(solid) == fx["solid_sha256"]
    assert digest(sdf) == fx["sdf_sha256"]


@pytest.mark.parametrize("device", [None, 0], ids=["host", "device"])
@pytest.mark.parametrize("name", sorted(EXPLICIT))
def test_voxelize_explicit_grid_matches_oracle(gpu, oracle_built, name, device):
    from flowcraft_b200.voxelizer import VoxelizeOnGrid
    c = EXPLICIT[name]
    pos, idx = mesh(c["mesh"])
    origin = np.asarray(c["origin"], np.float32)
    want_s, want_d = oracle_built.voxelize(pos, idx, c["dims"], c["cell"], origin)
    g = VoxelizeOnGrid(pos, idx, c["dims"], c["cell"], origin, device=device)
    solid, sdf = _host(g.solid), _host(g.signedDistance)
    assert np.array_equal(solid, want_s.ravel())
    assert np.array_equal(sdf.view(np.uint32), want_d.ravel().view(np.uint32))


def test_grid_derivation_matches_oracle(gpu, oracle_built):
    from flowcraft_b200.voxelizer import GridForMesh, Params
    for name, res, pad in (("aircraft", 640, (0.3, 1.0, 0.5)), ("naca2412_taper", 100, (0.0, 0.25, 2.0)),
                           ("soup", 7, (0.5, 0.5, 0.5)), ("icosphere", 3, (0.3, 1.0, 0.5))):
        pos, _ = mesh(name)
        want = oracle_built.grid_for_mesh(pos, res, pad)
        for device in (None, 0):
            dims, cell, origin = GridForMesh(pos, Params(res, pad), device=device)
            assert dims == want[0] and np.float32(cell) == np.float32(want[1])
            assert np.array_equal(np.asarray(origin, np.float32).view(np.uint32), want[2].view(np.uint32))


def test_signed_zero_bounds_keep_the_first_vertex(gpu, oracle_built):
    """std::min/std::max keep the first of equal values: -0.0 then +0.0 gives -0.0."""
    from flowcraft_b200.voxelizer import GridForMesh, Params
    pos = np.array([[-0.0, 1.0, -0.0], [0.0, 2.0, 0.0], [1.0, -0.0, 3.0], [2.0, 0.0, 1.0]], np.float32)
    for order in (pos, pos[[1, 0, 3, 2]]):
        want = oracle_built.grid_for_mesh(order, 16, (0.0, 0.0, 0.0))
        dims, cell, origin = GridForMesh(order, Params(16, (0.0, 0.0, 0.0)))
        assert dims == want[0]
        assert np.array_equal(np.asarray(origin, np.float32).view(np.uint32), want[2].view(np.uint32))


def test_empty_and_invalid_meshes(gpu):
    from flowcraft_b200.voxelizer import Voxelize, VoxelizeOnGrid
    g = Voxelize(np.zeros((0, 3), np.float32), np.zeros(0, np.uint32))
    assert g.CellCount() == 0
    pos, idx = mesh("icosphere")
    g = VoxelizeOnGrid(pos, idx[:2], (9, 10, 11), 1.0, (0.0, 0.0, 0.0))
    assert not _host(g.solid).any() and np.isposinf(_host(g.signedDistance)).all()
    bad = idx.copy()
    bad[7] = len(pos)
    with pytest.raises(ValueError):
        VoxelizeOnGrid(pos, bad, (16, 16, 16), 1.5, (-12.0, -12.0, -12.0))


def test_voxelized_c1_obstacle_steps_bit_exact(gpu, oracle_built):
    """Mesh -> device voxel grid -> solver, against the oracle solver on the
    oracle's voxelization of the same mesh (the c1 obstacle, 128x64x64), for
    the configuration's 1000 steps."""
    import torch
    from flowcraft_b200.lbm import LatticeModel, LbmSolver, Params
    from flowcraft_b200.voxelizer import VoxelizeOnGrid
    c = EXPLICIT["c1_sphere_128x64x64"]
    pos, idx = mesh(c["mesh"])
    g = VoxelizeOnGrid(pos, idx, c["dims"], c["cell"], c["origin"], device=0)
    want_s, want_d = oracle_built.voxelize(pos, idx, c["dims"], c["cell"], np.asarray(c["origin"], np.float32))
    assert torch.equal(g.solid.cpu(), torch.from_numpy(want_s.ravel()))
    # tau from nu = u D / Re with u = 0.05, D = 20, Re = 100
    params = Params(tau=0.5 + 3.0 * 0.05 * 20.0 / 100.0, inletVelocity=0.05, smagorinskyCs=0.1)
    s = LbmSolver()
    assert s.Init(0, g, LatticeModel.D3Q19), s.LastError()
    s.Reset(params)
    s.Step(None, 1000)
    got = s.ReadbackField()
    s.close()
    o = oracle_built.Oracle(want_s, want_d, 19, oracle_built.Params(params.tau, 0.05, False, True, True, 0.1))
    o.step(1000)
    want = o.readback_field()
    o.close()
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
