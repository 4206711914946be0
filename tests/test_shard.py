"""The z-slab split of one lattice (flowcraft_b200.shard) on the CPU: slab
ranges, layouts, and the step sequence over a stand-in solver whose update
reads the +-1 layers like the LBM pull and whose readback reads +-2 layers
like the solid-cell force, unsplit versus split over emulated ranks and over
gloo processes."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch

from flowcraft_b200 import shard


class FakeSolver:
    """Three populations per cell on (nz, nxy) layers: a rest population and
    two moving in +z / -z, bounced back at the lattice's z faces, then mixed
    within the cell and along the layer. Every output depends on the input
    layers z-1, z, z+1 only, as the D3Q19 pull does."""

    def __init__(self, init):
        self.pop = [init.copy(), np.zeros_like(init)]
        self.cur = 0
        self.nz = init.shape[1]

    def StepRange(self, cmd, z0, zc):
        fin, fout = self.pop[self.cur], self.pop[1 - self.cur]
        for z in range(max(z0, 0), min(z0 + zc, self.nz)):
            g0 = fin[0, z]
            g1 = fin[1, z - 1] if z > 0 else fin[2, z]
            g2 = fin[2, z + 1] if z + 1 < self.nz else fin[1, z]
            m = (g0 + g1 + g2) / 3.0
            for k, g in enumerate((g0, g1, g2)):
                fout[k, z] = g + 0.1 * (m - g) + 0.01 * np.roll(g, 1) * m

    def AdvanceSubstep(self):
        self.cur = 1 - self.cur

    def Readback(self, z):
        """Depends on the current set's layers z-2 .. z+2, like the momentum
        exchange force of a solid cell."""
        f = self.pop[self.cur]
        acc = f[0, z].copy()
        for d in (-2, -1, 1, 2):
            if 0 <= z + d < self.nz:
                acc = acc * 0.5 + f[(d + 2) % 3, z + d]
        return acc

    def LayerCopy(self, z, buf, to_buffer, next_set=False, cmd=None, ez=0):
        """ez = +1 / -1: only the population moving in +z / -z, as the
        buffer's first row (the stand-in's one plane per direction)."""
        p = self.pop[1 - self.cur if next_set else self.cur]
        b = buf.tensor.numpy()
        planes = [1] if ez == 1 else ([2] if ez == -1 else [0, 1, 2])
        if to_buffer:
            b[:len(planes)] = p[planes, z]
        else:
            p[planes, z] = b[:len(planes)]


class HostBuffer:
    def __init__(self, q, nxy):
        self.tensor = torch.zeros((q, nxy), dtype=torch.float64)
        self.ptr = self


def initial(nz, nxy=12, seed=7):
    return np.random.default_rng(seed).uniform(0.5, 1.5, size=(3, nz, nxy))


def unsplit(init, steps, readback=False):
    s = FakeSolver(init)
    for _ in range(steps):
        s.StepRange(None, 0, s.nz)
        s.AdvanceSubstep()
    if readback:
        return np.stack([s.Readback(z) for z in range(s.nz)])
    return s.pop[s.cur]


def owned_readback(s, lay):
    return np.stack([s.Readback(z) for z in range(lay.own0, lay.own1)])


def slab_stepper(init, rank, world, exchange):
    lay = shard.layout(init.shape[1], rank, world)
    s = FakeSolver(init[:, lay.lo:lay.hi])
    bufs = tuple(HostBuffer(3, init.shape[2]) for _ in range(4))
    return s, lay, shard.SlabStepper(s, lay, bufs, exchange, rank, dir_rows=1)


def test_slab_ranges_cover_and_balance():
    for nz in (1, 2, 7, 64, 513):
        for world in range(1, min(nz // 2, 9) + 1):
            r = shard.slab_ranges(nz, world)
            assert r[0][0] == 0 and r[-1][1] == nz
            assert all(a[1] == b[0] for a, b in zip(r, r[1:]))
            sizes = [b - a for a, b in r]
            assert max(sizes) - min(sizes) <= 1 and min(sizes) >= 1
    assert shard.slab_ranges(1, 1) == [(0, 1)]
    with pytest.raises(ValueError):
        shard.slab_ranges(5, 3)  # a one-layer slab cannot feed a two-layer halo
    with pytest.raises(ValueError):
        shard.slab_ranges(3, 0)


def test_layout_halos():
    lays = [shard.layout(10, r, 3) for r in range(3)]
    assert [(l.z0, l.z1) for l in lays] == [(0, 4), (4, 7), (7, 10)]
    assert [(l.lo, l.hi) for l in lays] == [(0, 6), (2, 9), (5, 10)]
    assert [(l.has_below, l.has_above) for l in lays] == [(False, True), (True, True), (True, False)]
    assert [(l.own0, l.own1) for l in lays] == [(0, 4), (2, 5), (2, 5)]
    one = shard.layout(5, 0, 1)
    assert (one.lo, one.hi, one.has_below, one.has_above) == (0, 5, False, False)


@pytest.mark.parametrize("nz,world", [(8, 2), (9, 3), (6, 3), (10, 5), (4, 2), (7, 1), (5, 2)])
def test_split_matches_unsplit(nz, world):
    """step_emulated's order (every rank's edges, the copies, every rank's
    interior and halos) over the host stand-in."""
    init = initial(nz)
    ref = unsplit(init, 6)
    ranks = [slab_stepper(init, r, world, None) for r in range(world)]
    shard.step_emulated([st for _, _, st in ranks], 6)
    for s, lay, _ in ranks:
        np.testing.assert_array_equal(s.pop[s.cur][:, lay.own0:lay.own1], ref[:, lay.z0:lay.z1])
    # readbacks reaching two layers need the outer halos refreshed
    rb = unsplit(init, 6, readback=True)
    shard.refresh_emulated([st for _, _, st in ranks])
    for s, lay, _ in ranks:
        np.testing.assert_array_equal(owned_readback(s, lay), rb[lay.z0:lay.z1])


def test_step_exchange_moves_only_the_streaming_planes():
    """Per step a side sends the planes streaming across the cut (one of the
    stand-in's three, 5 of D3Q19's 19); refresh sends whole layers."""
    init = initial(8)
    _, _, st = slab_stepper(init, 0, 2, None)
    (peer, send, recv), = st.posts(st.dir_rows)
    assert peer == 1 and send.tensor.shape[0] == 1 and recv.tensor.shape[0] == 1
    (_, send, _), = st.posts()
    assert send.tensor.shape[0] == 3
    assert shard.DIR_PLANES == 5


def test_stale_outer_halo_is_detected():
    """The refresh has teeth: without it the edge-layer readbacks differ."""
    init = initial(8)
    rb = unsplit(init, 3, readback=True)
    ranks = [slab_stepper(init, r, 2, None) for r in range(2)]
    shard.step_emulated([st for _, _, st in ranks], 3)
    assert any(not np.array_equal(owned_readback(s, lay), rb[lay.z0:lay.z1]) for s, lay, _ in ranks)


def test_missing_exchange_is_detected():
    """The check has teeth: skipping the halo unpack changes the owned layers."""
    init = initial(8)
    ref = unsplit(init, 4)
    ranks = [slab_stepper(init, r, 2, None) for r in range(2)]
    for _ in range(4):
        for _, _, st in ranks:
            st.edges()
            st.interior()
            st.s.AdvanceSubstep()
    diff = any(not np.array_equal(s.pop[s.cur][:, lay.own0:lay.own1], ref[:, lay.z0:lay.z1]) for s, lay, _ in ranks)
    assert diff


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gloo_rank(rank, world, port, nz, steps, out_dir):
    import datetime

    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        init = initial(nz)
        s, lay, st = slab_stepper(init, rank, world, shard.GlooExchange())
        st.step(steps)
        st.refresh()
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), s.pop[s.cur][:, lay.own0:lay.own1])
        np.save(os.path.join(out_dir, f"rb{rank}.npy"), owned_readback(s, lay))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_match_unsplit(tmp_path, world):
    import torch.multiprocessing as mp
    nz, steps = 10, 5
    mp.start_processes(_gloo_rank, args=(world, _free_port(), nz, steps, str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    ref = unsplit(initial(nz), steps)
    rb = unsplit(initial(nz), steps, readback=True)
    for r in range(world):
        lay = shard.layout(nz, r, world)
        np.testing.assert_array_equal(np.load(tmp_path / f"rank{r}.npy"), ref[:, lay.z0:lay.z1])
        np.testing.assert_array_equal(np.load(tmp_path / f"rb{r}.npy"), rb[lay.z0:lay.z1])
