"""The voxelizer oracle (oracle/voxel_oracle.c) against FlowCraft's own
Voxelizer::Voxelize: the committed golden digests (made by the reference, see
tests/golden/make_voxel_golden.py) and, where the reference build exists,
direct comparison on further meshes. Also the procedural meshes' topology."""
import json
import os

import numpy as np
import pytest

from conftest import ROOT
from voxel_cases import EXPLICIT, GOLDEN, digest, mesh, mesh_digest

GOLDEN_FILE = os.path.join(ROOT, "tests", "golden", "voxel_golden.json")


def _golden():
    with open(GOLDEN_FILE) as f:
        return json.load(f)["cases"]


@pytest.mark.parametrize("name", sorted(GOLDEN))
def test_oracle_reproduces_reference_golden(oracle_built, name):
    orc = oracle_built
    case, fx = GOLDEN[name], _golden()[name]
    pos, idx = mesh(case["mesh"])
    assert mesh_digest(pos, idx) == fx["mesh_sha256"], "procedural mesh changed"
    dims, cell, origin = orc.grid_for_mesh(pos, case["res"], case.get("padding", (0.3, 1.0, 0.5)))
    assert list(dims) == fx["dims"]
    assert int(np.float32(cell).view(np.uint32)) == fx["cell_bits"]
    assert [int(v) for v in np.asarray(origin, np.float32).view(np.uint32)] == fx["origin_bits"]
    solid, sdf = orc.voxelize(pos, idx, dims, cell, origin)
    assert int(solid.sum()) == fx["solid_cells"]
    assert digest(solid) == fx["solid_sha256"]
    assert digest(sdf) == fx["sdf_sha256"]


def test_oracle_matches_reference_on_soup_and_wing(oracle_built):
    orc = oracle_built
    if not orc.available("ref"):
        pytest.skip("reference build (oracle/_ref) not present")
    for name, res, pad in (("soup", 40, (0.3, 1.0, 0.5)), ("naca0012", 64, (0.1, 0.2, 0.9)),
                           ("inward", 36, (0.3, 1.0, 0.5))):
        pos, idx = mesh(name)
        dims, cell, origin, rs, rd = orc.voxelize_reference(pos, idx, res, pad)
        d2, c2, o2 = orc.grid_for_mesh(pos, res, pad)
        assert d2 == dims and c2 == cell and np.array_equal(o2, origin)
        s, d = orc.voxelize(pos, idx, dims, cell, origin)
        assert np.array_equal(s, rs)
        assert np.array_equal(d.view(np.uint32), rd.view(np.uint32))


def test_explicit_cases_have_their_intended_shape(oracle_built):
    """The edge cases reach what they are for (checked on the oracle)."""
    orc = oracle_built
    out = {}
    for name in ("seed_inside", "seed_on_shell", "soup"):
        c = EXPLICIT[name]
        pos, idx = mesh(c["mesh"])
        out[name] = orc.voxelize(pos, idx, c["dims"], c["cell"], np.asarray(c["origin"], np.float32))
    s, _ = out["seed_inside"]
    assert s.ravel()[0] == 0 and s[-1, -1, -1] == 1  # interior reached, exterior enclosed
    s, d = out["seed_on_shell"]
    assert s.all() and (d[np.isfinite(d)] <= 0.7 * 1.0 + 1.0).all()
    s, d = out["soup"]
    assert np.isinf(d).any() and (d < 0).any() and (d > 0).any()


def _edges_closed(idx):
    t = idx.reshape(-1, 3).astype(np.int64)
    e = np.concatenate([t[:, [0, 1]], t[:, [1, 2]], t[:, [2, 0]]])
    fwd = {tuple(x) for x in e}
    return all((b, a) in fwd for a, b in fwd) and len(fwd) == len(e)


def _volume(pos, idx):
    p = pos.astype(np.float64)
    t = idx.reshape(-1, 3)
    return np.einsum("ij,ij->i", p[t[:, 0]], np.cross(p[t[:, 1]], p[t[:, 2]])).sum() / 6.0


def test_procedural_meshes_are_closed_and_outward():
    from flowcraft_b200 import meshes
    pos, idx = meshes.icosphere(3, 10.0)
    assert idx.size // 3 == 1280 and _edges_closed(idx)
    assert abs(_volume(pos, idx) - 4.0 / 3.0 * np.pi * 1000.0) < 0.03 * 4.0 / 3.0 * np.pi * 1000.0
    for digits in ("0012", "2412"):
        pos, idx = meshes.naca_wing(digits, 40.0, 50.0, 4.0, 32, 8)
        assert _edges_closed(idx) and _volume(pos, idx) > 0
    pos, idx = meshes.aircraft()
    assert 60000 <= idx.size // 3 <= 120000 and _volume(pos, idx) > 0
