"""What the shipped learned closure does a posteriori, and how far it moves
the forces.

* Against the filtered fine run (flowcraft_b200.closure_eval), at reduced
  size (coarse 128x64x64, fine 256x128x128, 1000 coarse steps) on both of the
  closure's evaluation cases: the coarse run with the learned closure has a
  smaller time-averaged wake velocity error than the coarse run with
  Smagorinsky, and its drag error is no more than one percentage point
  worse.
* On the precision configuration's NACA 0012 wing at full size (384x192x192,
  Re 1e4, 5000 steps, forces averaged over the last fifth): FP16 storage with
  the learned closure keeps the drag and lift within 1 % of the FP32
  Smagorinsky run, the accuracy bound the benchmark's pairing states.
* On the large configuration's aircraft at half size (512x256x256, the mesh
  voxelized on the device, Re 1e5 on the 30-cell root chord, 1500 steps,
  forces averaged over the last fifth): FP16 storage with Smagorinsky stays
  within 2 % of FP32 Smagorinsky in drag and lift, and FP16 with the learned
  closure within 5 %. The 1 % bound for the learned closure is not met on
  this case; FP16 storage alone already moves drag by about 1 % here."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _shipped():
    import os

    from flowcraft_b200.closure import ClosureWeights
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    return ClosureWeights.load(os.path.join(root, "flowcraft_b200", "data", "closure_c4.json"))


@pytest.mark.parametrize("name", ["sphere_re2e4", "wing2412_re1e4"])
def test_learned_closure_closer_to_filtered_fine_run(gpu, name):
    from flowcraft_b200 import closure_eval as ce
    c = {k.name: k for k in ce.C4_EVAL_CASES}[name]
    case = ce.EvalCase(c.name, c.geom, c.re, 128, 64, 64, coarse_steps=1000, every=25)
    r = ce.evaluate(case, _shipped())
    s, l = r["smagorinsky"], r["learned"]
    print(name, "wake rms |du|/U: smagorinsky %.5f learned %.5f; drag vs fine: %.4f %.4f" % (
        s["wake_rms_du_over_u"], l["wake_rms_du_over_u"], s["drag_vs_fine"], l["drag_vs_fine"]))
    assert not (s["diverged"] or l["diverged"] or r["fine"]["diverged"])
    assert l["wake_rms_du_over_u"] < s["wake_rms_du_over_u"]
    assert abs(l["drag_vs_fine"]) < abs(s["drag_vs_fine"]) + 0.01


def _avg_forces(solid, sdf, storage, closure, tau, steps=1500, u=0.05):
    from flowcraft_b200.lbm import LatticeModel, LbmSolver, Params, Storage, VoxelGrid
    nz, ny, nx = solid.shape
    s = LbmSolver()
    assert s.Init(0, VoxelGrid(nx, ny, nz, solid=solid, signedDistance=sdf), LatticeModel.D3Q19, Storage[storage])
    s.Reset(Params(tau=tau, inletVelocity=u, smagorinskyCs=0.1), True)
    if closure is not None:
        s.SetClosure(closure)
    a0 = steps - steps // 5
    s.Step(None, a0)
    acc, n = np.zeros(3), 0
    for _ in range(a0, steps, 10):
        s.Step(None, 10)
        acc += np.asarray(s.AerodynamicForces().forceSum)
        n += 1
    assert not s.HasDiverged()
    s.close()
    return acc / n


def test_learned_closure_within_1pct_on_the_precision_wing(gpu):
    import sys

    sys.path.insert(0, __import__("os").path.dirname(__file__))
    import precision_study as ps
    c = ps.case(False)
    solid, sdf = ps.geometry(c)
    tau = ps.tau_of(c)
    ref = _avg_forces(solid, sdf, "FP32", None, tau, steps=c["steps"], u=ps.U)
    learned = _avg_forces(solid, sdf, "FP16_OFFSET", _shipped(), tau, steps=c["steps"], u=ps.U)
    dcd, dcl = learned[0] / ref[0] - 1.0, learned[2] / ref[2] - 1.0
    print("precision wing: FP16 learned dCd %+.4f dCl %+.4f against FP32 Smagorinsky" % (dcd, dcl))
    assert abs(dcd) < 0.01 and abs(dcl) < 0.01


def test_aircraft_forces_envelope(gpu):
    import bench
    cfg = dict(nx=512, ny=256, nz=256)
    solid, sdf = bench.aircraft_on_device(cfg, "cuda:0")
    solid, sdf = solid.cpu().numpy(), sdf.cpu().numpy()
    tau = 0.5 + 3.0 * 0.05 * 30.0 / 1e5
    ref = _avg_forces(solid, sdf, "FP32", None, tau)
    fp16 = _avg_forces(solid, sdf, "FP16_OFFSET", None, tau)
    learned = _avg_forces(solid, sdf, "FP16_OFFSET", _shipped(), tau)
    d16 = (fp16[0] / ref[0] - 1.0, fp16[2] / ref[2] - 1.0)
    dl = (learned[0] / ref[0] - 1.0, learned[2] / ref[2] - 1.0)
    print("FP16 Smagorinsky dCd %+.4f dCl %+.4f; FP16 learned dCd %+.4f dCl %+.4f" % (*d16, *dl))
    assert abs(d16[0]) < 0.02 and abs(d16[1]) < 0.02
    assert abs(dl[0]) < 0.05 and abs(dl[1]) < 0.05
