"""Training the learned closure with the library's CUDA kernels: the MLP
gradient, forward pass and Adam step against the CPU oracle
(oracle/mlp_oracle.py), the training samples against a numpy restatement of
the 2x box filter, and a small end-to-end training that must beat the
Smagorinsky closure on held-out samples."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.tensor(np.asarray(a, np.float32), device="cuda:0")


def test_mlp_grad_forward_adam_match_oracle(gpu):
    import torch

    from flowcraft_b200.closure_train import MlpTrainer, he_init
    from oracle import mlp_oracle as mo
    rng = np.random.default_rng(3)
    p = he_init(7)
    p[160:192] = rng.normal(0, 0.1, 32)
    p[1216:1248] = rng.normal(0, 0.1, 32)
    x = rng.normal(0, 1, (3000, 5)).astype(np.float32)
    y = rng.normal(0, 1, 3000).astype(np.float32)
    tr = MlpTrainer(p)
    xd, yd = _dev(x), _dev(y)
    out = tr.predict(xd).cpu().numpy()
    want, _ = mo.forward(p.astype(np.float64), x)
    assert np.abs(out - want).max() < 1e-4 * max(1.0, np.abs(want).max())
    idx = torch.tensor(rng.permutation(3000)[:2500], device="cuda:0")
    loss, g = tr.grad(xd, yd, idx)
    g1 = g.cpu().numpy().copy()
    l_ref, g_ref = mo.loss_grad(p.astype(np.float64), x[idx.cpu().numpy()], y[idx.cpu().numpy()])
    assert abs(loss.item() - l_ref) < 1e-6 * l_ref
    assert np.abs(g1 - g_ref).max() < 2e-5 * np.abs(g_ref).max()
    # deterministic: the same call gives the same bits
    _, g2 = tr.grad(xd, yd, idx)
    assert np.array_equal(g1.view(np.uint32), g2.cpu().numpy().view(np.uint32))
    # one Adam step
    tr.adam(lr=1e-3)
    m = 0.1 * g_ref
    v = 0.001 * g_ref * g_ref
    step = 1e-3 * (m / 0.1) / (np.sqrt(v / 0.001) + 1e-8)
    assert np.abs(tr.params() - (p - step)).max() < 2e-6


def _box_filter_samples(pops, solid, tau_c, filter_width, tau_f, cs_f):
    """Restatement of the sample extraction in float64 numpy (closure.cu):
    the target fits the filtered viscous stress (each fine cell's relaxation
    time recovered from its post-collision stress) minus the resolved
    sub-grid stress."""
    from test_closure_gpu import LATTICE
    e = np.asarray(LATTICE[pops.shape[0]], np.float64)
    nz, ny, nx = solid.shape
    f = pops.astype(np.float64).reshape(-1, nz, ny, nx)
    rho = f.sum(0)
    j = np.einsum("ia,izyx->azyx", e, f)
    u = j / rho
    cz, cy, cx = nz // 2, ny // 2, nx // 2

    def blk(a):
        a = a[..., :2 * cz, :2 * cy, :2 * cx]
        return a.reshape(a.shape[:-3] + (cz, 2, cy, 2, cx, 2)).sum(axis=(-5, -3, -1))
    sol = blk(solid[None].astype(np.float64))[0] > 0
    rs = blk(rho[None])[0]
    m = blk(j)
    ub = m / rs
    rb = rs / 8.0
    uu = blk(np.einsum("zyx,azyx,bzyx->abzyx", rho, u, u).reshape(9, nz, ny, nx)).reshape(3, 3, cz, cy, cx)
    tau = uu / 8.0 - rb * np.einsum("azyx,bzyx->abzyx", ub, ub)
    # each fine cell's viscous stress from its post-collision stress
    m2 = np.einsum("ia,ib,izyx->abzyx", e, e, f)
    pst = m2 - rho / 3.0 * np.eye(3)[:, :, None, None, None] - np.einsum("zyx,azyx,bzyx->abzyx", rho, u, u)
    pmag = np.sqrt((pst * pst).sum(axis=(0, 1)))
    kq = 18.0 * 1.41421356 * cs_f * cs_f
    disc = np.maximum((1.0 - tau_f) ** 2 - kq * pmag / np.maximum(rho, 1e-6), 0.0)
    te = 0.5 * ((1.0 + tau_f) - np.sqrt(disc))
    vf = (te - 0.5) / (1.0 - te) * pst
    vis = blk(vf.reshape(9, nz, ny, nx)).reshape(3, 3, cz, cy, cx) / 8.0
    rows = []
    for z in range(1, cz - 1):
        for y in range(1, cy - 1):
            for x in range(2, cx - 2):
                if sol[z, y, x] or sol[z, y, x - 1] or sol[z, y, x + 1] or sol[z, y - 1, x] or sol[z, y + 1, x] \
                        or sol[z - 1, y, x] or sol[z + 1, y, x]:
                    continue
                gx = 0.5 * (ub[:, z, y, x + 1] - ub[:, z, y, x - 1])
                gy = 0.5 * (ub[:, z, y + 1, x] - ub[:, z, y - 1, x])
                gz = 0.5 * (ub[:, z + 1, y, x] - ub[:, z - 1, y, x])
                g = np.stack([gx, gy, gz])
                s = 0.5 * (g + g.T)
                sd = s - np.trace(s) / 3 * np.eye(3)
                t = vis[:, :, z, y, x] - tau[:, :, z, y, x]
                td = t - np.trace(t) / 3 * np.eye(3)
                sds = (sd * sd).sum()
                if not sds > 1e-18:
                    continue
                nu = max(0.0, (td * sd).sum() / (2 * rb[z, y, x] * sds) - (tau_c - 0.5) / 3.0)
                p = -(2.0 / 3.0) * rb[z, y, x] * (tau_c + 3 * nu) * s
                mag = np.sqrt((p * p).sum())
                rows.append([np.log2(mag / rb[z, y, x] + 1e-12), np.trace(p) / mag, np.linalg.det(p) / mag ** 3,
                             np.nan, filter_width, nu])
    return np.asarray(rows)


def test_closure_samples_match_numpy(gpu, oracle_built):
    from flowcraft_b200 import geometry
    from flowcraft_b200.lbm import LatticeModel, LbmSolver, Params, Storage, VoxelGrid
    solid, sdf = geometry.sphere_grid(64, 32, 32, 20.0, 16.0, 16.0, 5.0)
    s = LbmSolver()
    assert s.Init(0, VoxelGrid(64, 32, 32, solid=solid.ravel(), signedDistance=sdf.ravel()), LatticeModel.D3Q19,
                  Storage.FP32)
    s.Reset(Params(tau=0.52, inletVelocity=0.08, smagorinskyCs=0.1), True)
    s.Step(None, 150)
    rows = s.ClosureSamples(2.0).cpu().numpy()
    want = _box_filter_samples(s.SavePopulations(), solid, 0.5 + 0.5 * (0.52 - 0.5), 2.0, 0.52, 0.1)
    assert len(rows) == len(want) > 200
    assert np.isfinite(rows).all() and (rows[:, 5] >= 0).all()
    for k in (0, 5):
        scale = np.abs(want[:, k]).max()
        assert np.abs(rows[:, k] - want[:, k]).max() < 2e-3 * scale, k
    assert np.abs(rows[:, 1:3] - want[:, 1:3]).max() < 1e-3
    # wall distance of the coarse solid mask: the oracle's chamfer transform
    cs = oracle_built.wall_distance(solid[:32, :32, :64].reshape(16, 2, 16, 2, 32, 2).max(axis=(1, 3, 5)))
    assert set(np.unique(rows[:, 3] * 16).astype(int)) <= set(np.unique(cs).astype(int))
    s.close()


def test_training_beats_smagorinsky_a_priori(gpu):
    """A small training run: the loss falls and the trained MLP predicts the
    held-out eddy viscosity better than Smagorinsky at its best Cs; the
    trained closure then runs a coarse lattice stably."""
    from flowcraft_b200 import geometry
    from flowcraft_b200.closure_train import collect_samples, train_closure
    from flowcraft_b200.lbm import LatticeModel, LbmSolver, Params, Storage, VoxelGrid
    solid, sdf = geometry.sphere_grid(192, 96, 96, 60.0, 48.0, 48.0, 12.0)
    nu_f = 0.08 * 24.0 / 2000.0
    case = dict(solid=solid, sdf=sdf.ravel(), params=Params(tau=0.5 + 3 * nu_f, inletVelocity=0.08,
                                                            smagorinskyCs=0.1), warmup=600, every=100, count=4)
    samples, tau_c = collect_samples([case])
    cw, rep = train_closure(samples, tau_c, epochs=8, batch=2048, lr=2e-3, seed=0)
    print(rep)
    assert rep.samples > 20000
    assert rep.train_loss[-1] < 0.95 * rep.train_loss[0]
    assert rep.holdout_mse["mlp"] < 0.85 * rep.holdout_mse["zero"]
    assert rep.gain_vs_best_smagorinsky > 1.15
    csol, csdf = geometry.sphere_grid(96, 48, 48, 30.0, 24.0, 24.0, 6.0)
    s = LbmSolver()
    assert s.Init(0, VoxelGrid(96, 48, 48, solid=csol.ravel(), signedDistance=csdf.ravel()), LatticeModel.D3Q19,
                  Storage.FP16_OFFSET)
    s.Reset(Params(tau=0.5 + 0.5 * 3 * nu_f, inletVelocity=0.08, smagorinskyCs=0.1), True)
    s.SetClosure(cw)
    s.Step(None, 300)
    st = s.ReadbackStats()
    assert not st.hasNaN and not s.HasDiverged()
    _, nu, rng = s.ClosureProbe()
    assert rng.mean() > 0.5
    s.close()
