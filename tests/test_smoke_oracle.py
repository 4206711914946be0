"""The smoke-trail restatement (oracle/smoke_oracle.py) against the
reference's own SmokeTrailSystem::Step: the committed fixture (made by the
reference, tests/golden/make_smoke_golden.py) and, where the reference build
exists, a fresh run with other particles."""
import json
import os

import numpy as np
import pytest

from cases import CASES, GOLDEN_DIR, OracleAdapter, field_digest, geometry
from oracle import smoke_oracle as so


def _field(oracle_built, fx):
    case = CASES[fx["case"]]
    o = OracleAdapter(case)
    o.step(fx["case_steps"])
    f = o.readback_field()
    assert field_digest(f) == fx["field_sha256"]  # the restated solver reproduces the reference's field
    return case, f


def test_restatement_reproduces_reference_trails(oracle_built):
    fx = json.load(open(os.path.join(GOLDEN_DIR, "smoke_golden.json")))
    case, field = _field(oracle_built, fx)
    solid = geometry(case["geom"])[0]
    nz, ny, nx = solid.shape
    for run in fx["runs"]:
        pos = np.array(run["positions"], dtype=np.float32)
        want = np.array(run["trail_bits"], dtype=np.uint32).view(np.float32)
        lens = np.array(run["lens"])
        got, ok = so.advect(field, solid, (nx, ny, nz), fx["cell_size"], fx["origin"], pos, fx["steps"],
                            run["mm_per_sec"], run["dt"], run["confine_axis"])
        for p in np.nonzero(np.array(run["keep"]))[0]:
            assert ok[p]
            n = lens[p]
            assert np.array_equal(got[p, fx["steps"] + 1 - n:].view(np.uint32), want[p, :n].view(np.uint32))


@pytest.mark.skipif(not so.reference_available(), reason="reference build absent")
def test_restatement_matches_live_reference(oracle_built):
    fx = json.load(open(os.path.join(GOLDEN_DIR, "smoke_golden.json")))
    case, field = _field(oracle_built, fx)
    solid = geometry(case["geom"])[0]
    nz, ny, nx = solid.shape
    rng = np.random.default_rng(5)
    pos = np.stack([rng.uniform(2, ny - 2, 40), rng.uniform(4, nx - 6, 40), rng.uniform(2, nz - 2, 40)], 1)
    pos = pos.astype(np.float32)
    want, lens = so.step_reference(solid, field, (nx, ny, nz), 1.0, (0, 0, 0), pos, 5, 9, 30.0, 0.07)
    got, ok = so.advect(field, solid, (nx, ny, nz), 1.0, (0, 0, 0), pos, 9, 30.0, 0.07)
    checked = 0
    for p in range(len(pos)):
        if ok[p] and lens[p] == 5:
            assert np.array_equal(got[p, 5:].view(np.uint32), want[p].view(np.uint32))
            checked += 1
    assert checked >= 20
