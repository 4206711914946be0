"""One lattice split into z-slabs across ranks (one GPU each), with a halo
exchange per step.

Every |e_z| <= 1, so stepping a slab [z0, z1) of the global lattice needs one
layer of its neighbours' populations per side (the reference's LbmSolver
already steps z-ranges through StepRange, LbmSolver.h:141-170). The
momentum-exchange force of a solid cell reads the Bouzidi partner of its
fluid neighbour, two layers away (LbmReference.cpp:100-122), so a rank keeps
two halo layers per side. A rank runs an ordinary solver on its slab plus
those halo layers, which carry the true geometry, so every owned cell is
classified as in the whole lattice. A step goes:

  1. step the slab's first and last owned layers (StepRange);
  2. pack those two layers of the step's output and post the exchange: the
     first owned layer goes to the rank below (its inner upper halo), the
     last to the rank above;
  3. step the owned layers between them while the exchange runs;
  4. unpack the received layers into the output's inner halo layers;
  5. AdvanceSubstep.

Only the planes that stream across the cut travel per step: the layer next
to a lower halo reads from it the populations with e_z = +1 (the pull and
the Bouzidi near-side partner alike), and the layer next to an upper halo
those with e_z = -1, so each side sends 5 of the Q planes (D3Q19 and D3Q15)
instead of all of them.

The halo layers are never stepped (their content is what the neighbours
send), so the owned layers are bit-identical to the unsplit lattice. The
halos' other planes, and the outer halo layers, only feed readbacks of
solid-cell forces: refresh() exchanges both halo layers, all planes, in the
current population set, before such a readback.

The exchange is pluggable: NcclExchange (torch.distributed point-to-point on
the device buffers, one process per GPU) and GlooExchange (CPU tensors, for
tests of this orchestration); step_emulated / refresh_emulated run several
ranks in one process with plain device copies as the exchange.

What a slab does not reproduce bit for bit: the learned closure's wall
distance is a chamfer transform of the slab's own solid mask, so a cell whose
nearest wall lies beyond the halo sees a larger distance. Slabs therefore run
without the learned closure (Smagorinsky is per cell).
"""
from __future__ import annotations

import contextlib
from dataclasses import dataclass

HALO = 2  # halo layers per side
DIR_PLANES = 5  # planes with e_z = +1 (or -1), FC_LBM_DIR_PLANES


def slab_ranges(nz: int, world: int):
    """Contiguous, balanced [z0, z1) per rank; with more than one rank every
    slab holds at least two layers (the neighbours' outer halos)."""
    if world < 1 or nz < world * (2 if world > 1 else 1):
        raise ValueError("need at least two z layers per rank")
    base, extra = divmod(nz, world)
    out, z = [], 0
    for r in range(world):
        t = base + (1 if r < extra else 0)
        out.append((z, z + t))
        z += t
    return out


@dataclass
class SlabLayout:
    """Where a rank's slab sits in its local lattice."""
    z0: int          # first owned global layer
    z1: int          # one past the last owned global layer
    lo: int          # first global layer of the local lattice (z0 - 2, or 0)
    hi: int          # one past its last (z1 + 2, or nz)
    has_below: bool
    has_above: bool

    @property
    def local_nz(self) -> int:
        return self.hi - self.lo

    @property
    def own0(self) -> int:    # first owned layer, local index
        return self.z0 - self.lo

    @property
    def own1(self) -> int:    # one past the last owned layer, local index
        return self.z1 - self.lo


def layout(nz: int, rank: int, world: int) -> SlabLayout:
    z0, z1 = slab_ranges(nz, world)[rank]
    lo, hi = max(z0 - HALO, 0), min(z1 + HALO, nz)
    return SlabLayout(z0, z1, lo, hi, z0 > 0, z1 < nz)


def slab_stream(device: int):
    """A torch stream for a rank's solver calls and exchange. It must not be
    the legacy default stream: its handle is 0, which the solver reads as
    "my own stream", and the exchange would then not be ordered after the
    layer packs."""
    import torch
    return torch.cuda.Stream(device)


class SlabStepper:
    """The step sequence of one rank over any solver exposing
    StepRange(cmd, z0, zc), AdvanceSubstep() and LayerCopy(z, ptr,
    to_buffer, next_set, cmd, ez), with buffers given as (send_below,
    recv_below, send_above, recv_above) objects whose ``ptr`` the solver
    understands and whose ``tensor`` holds one row per plane. With a torch
    stream ``cmd`` (from slab_stream), the solver calls and the exchange all
    go on it. ``dir_rows``: the rows LayerCopy packs for one e_z direction."""

    def __init__(self, solver, lay: SlabLayout, buffers, exchange, rank: int, cmd=None, dir_rows: int = DIR_PLANES):
        if cmd is not None and not getattr(cmd, "cuda_stream", 0):
            raise ValueError("the slab stream must be a non-default torch.cuda.Stream")
        self.s, self.lay, self.buf, self.ex, self.rank, self.cmd = solver, lay, buffers, exchange, rank, cmd
        self.dir_rows = dir_rows

    def on_stream(self):
        """Makes cmd torch's current stream (for the exchange's copies and
        collectives), or does nothing without one."""
        if self.cmd is None:
            return contextlib.nullcontext()
        import torch
        return torch.cuda.stream(self.cmd)

    # local layers sent to (below, above) and received from them, per exchange
    def _send_layers(self, outer: bool):
        k = 1 if outer else 0
        return self.lay.own0 + k, self.lay.own1 - 1 - k

    def _recv_layers(self, outer: bool):
        k = 1 if outer else 0
        return self.lay.own0 - 1 - k, self.lay.own1 + k

    def pack(self, outer: bool = False, full: bool = False):
        """The layers the neighbours need into the send buffers. Per step
        (neither flag): the step's output edges, only the planes streaming
        across the cut (e_z = -1 down, +1 up). `full`: all planes of the
        current set's edges (inner) or second layers (`outer`)."""
        lo, hi = self._send_layers(outer)
        send_lo, _, send_hi, _ = self.buf
        step = not (outer or full)
        if self.lay.has_below:
            self.s.LayerCopy(lo, send_lo.ptr, True, step, self.cmd, -1 if step else 0)
        if self.lay.has_above:
            self.s.LayerCopy(hi, send_hi.ptr, True, step, self.cmd, 1 if step else 0)

    def unpack(self, outer: bool = False, full: bool = False):
        lo, hi = self._recv_layers(outer)
        _, recv_lo, _, recv_hi = self.buf
        step = not (outer or full)
        if self.lay.has_below:
            self.s.LayerCopy(lo, recv_lo.ptr, False, step, self.cmd, 1 if step else 0)
        if self.lay.has_above:
            self.s.LayerCopy(hi, recv_hi.ptr, False, step, self.cmd, -1 if step else 0)

    def edges(self):
        """Steps 1-2: the first and last owned layers, packed for the neighbours."""
        a, b = self.lay.own0, self.lay.own1 - 1
        self.s.StepRange(self.cmd, a, 1)
        if b != a:
            self.s.StepRange(self.cmd, b, 1)
        self.pack()

    def interior(self):
        """Step 3: the owned layers between the edges."""
        n = self.lay.own1 - self.lay.own0 - 2
        if n > 0:
            self.s.StepRange(self.cmd, self.lay.own0 + 1, n)

    def finish(self):
        """Steps 4-5: the received layers into the output's halos, then advance."""
        self.unpack()
        self.s.AdvanceSubstep()

    def posts(self, rows=None):
        """(peer, send, receive) of this rank's exchange: views of the
        buffers' first `rows` rows (all rows when None)."""
        send_lo, recv_lo, send_hi, recv_hi = self.buf
        out = []
        if self.lay.has_below:
            out.append((self.rank - 1, _Rows(send_lo, rows), _Rows(recv_lo, rows)))
        if self.lay.has_above:
            out.append((self.rank + 1, _Rows(send_hi, rows), _Rows(recv_hi, rows)))
        return out

    def step(self, n: int = 1):
        """n steps of this rank (one process per rank)."""
        with self.on_stream():
            for _ in range(n):
                self.edges()
                h = self.ex.post(self.posts(self.dir_rows))
                self.interior()
                self.ex.wait(h)
                self.finish()

    def refresh(self):
        """Both halo layers of the current set, all planes (one process per
        rank), before a readback of solid-cell forces."""
        with self.on_stream():
            for outer in (False, True):
                self.pack(outer=outer, full=True)
                self.ex.wait(self.ex.post(self.posts()))
                self.unpack(outer=outer, full=True)


class _Rows:
    """The leading rows of an exchange buffer, as the exchange sends them."""

    def __init__(self, buf, rows=None):
        self.tensor = buf.tensor if rows is None else buf.tensor[:rows]


class NcclExchange:
    """Point-to-point over torch.distributed (NCCL) on device tensors. The
    operations are ordered after torch's current stream, which SlabStepper
    makes the solver's stream, and wait() orders that stream after them."""

    def post(self, pairs):
        import torch.distributed as dist
        ops = []
        for peer, send, recv in pairs:
            ops.append(dist.P2POp(dist.isend, send.tensor, peer))
            ops.append(dist.P2POp(dist.irecv, recv.tensor, peer))
        return dist.batch_isend_irecv(ops) if ops else []

    def wait(self, reqs):
        for r in reqs:
            r.wait()


class GlooExchange:
    """The same exchange between CPU processes (gloo), for tests."""

    def post(self, pairs):
        import torch.distributed as dist
        reqs = []
        for peer, send, recv in pairs:
            reqs.append(dist.isend(send.tensor, peer))
            reqs.append(dist.irecv(recv.tensor, peer))
        return reqs

    def wait(self, reqs):
        for r in reqs:
            r.wait()


class DeviceBuffer:
    """A device byte buffer for one packed layer: `rows` planes of
    `row_bytes` (nx * ny elements) each."""

    def __init__(self, rows: int, row_bytes: int, device: int):
        import torch
        self.tensor = torch.empty((rows, row_bytes), dtype=torch.uint8, device=f"cuda:{device}")
        self.ptr = self.tensor.data_ptr()


def _copy_emulated(steppers, rows=None):
    for st in steppers:
        for peer, _send, recv in st.posts(rows):
            other = steppers[peer]
            # the peer's send buffer facing this rank
            src = _Rows(other.buf[0] if peer > st.rank else other.buf[2], rows)
            recv.tensor.copy_(src.tensor)


def _shared_stream(steppers):
    if len({id(st.cmd) for st in steppers}) > 1:
        raise ValueError("emulated ranks must share one stream")
    return steppers[0].on_stream()


def step_emulated(steppers, n: int = 1):
    """n steps of ranks emulated in one process: every rank's edges, then the
    exchange as copies on the ranks' shared stream, then every rank's
    interior and halos. The steppers share one stream (emulated_ranks builds
    them so), or none for host stand-ins."""
    with _shared_stream(steppers):
        for _ in range(n):
            for st in steppers:
                st.edges()
            _copy_emulated(steppers, steppers[0].dir_rows)
            for st in steppers:
                st.interior()
                st.finish()


def refresh_emulated(steppers):
    """SlabStepper.refresh for ranks emulated in one process."""
    with _shared_stream(steppers):
        for outer in (False, True):
            for st in steppers:
                st.pack(outer=outer, full=True)
            _copy_emulated(steppers)
            for st in steppers:
                st.unpack(outer=outer, full=True)


def make_slab_solver(solid, sdf, rank: int, world: int, device: int, model, storage, params, seed_mid=True,
                     stream=None):
    """An LbmSolver for rank's slab of a global (nz, ny, nx) geometry, with
    its halo layers, plus its layout and exchange buffers (allocated on
    ``stream``, the slab stream that will use them)."""
    import numpy as np
    import torch

    from .lbm import LatticeModel, LbmSolver, Storage, VoxelGrid
    nz, ny, nx = solid.shape
    lay = layout(nz, rank, world)
    sl = slice(lay.lo, lay.hi)
    ls = solid[sl]
    lsd = None if sdf is None else sdf[sl]
    if isinstance(ls, torch.Tensor):
        ls = ls.contiguous()
        lsd = None if lsd is None else lsd.contiguous()
    else:
        ls = np.ascontiguousarray(ls)
        lsd = None if lsd is None else np.ascontiguousarray(lsd)
    s = LbmSolver()
    g = VoxelGrid(nx, ny, lay.local_nz, solid=ls.reshape(-1), signedDistance=None if lsd is None else lsd.reshape(-1))
    if not s.Init(device, g, model, storage):
        raise RuntimeError(s.LastError())
    s.Reset(params, seed_mid)
    q = 19 if model == LatticeModel.D3Q19 else 15
    elem = 4 if storage == Storage.FP32 else 2
    with torch.cuda.stream(stream) if stream is not None else contextlib.nullcontext():
        bufs = tuple(DeviceBuffer(q, nx * ny * elem, device) for _ in range(4))
    return s, lay, bufs


def owned_field(solver, lay: SlabLayout):
    """(rho, ux, uy, uz) of the rank's owned layers (force and stress on
    solid cells), shape ((z1-z0)*ny*nx, 4). The solid cells of the first
    and last owned layers read the outer halos: refresh them first."""
    import numpy as np
    f = np.empty(solver.CellCount() * 4, dtype=np.float32)
    solver.ReadbackFieldRange(lay.own0, lay.z1 - lay.z0, f)
    per = f.size // lay.local_nz
    return f[lay.own0 * per:lay.own1 * per].reshape(-1, 4)


def emulated_ranks(solid, sdf, world: int, device: int, model, storage, params, seed_mid=True):
    """``world`` slab solvers of one geometry on one device, their calls on
    one shared slab stream, for step_emulated: [(solver, layout, stepper)]."""
    cmd = slab_stream(device)
    out = []
    for r in range(world):
        s, lay, bufs = make_slab_solver(solid, sdf, r, world, device, model, storage, params, seed_mid, cmd)
        out.append((s, lay, SlabStepper(s, lay, bufs, None, r, cmd=cmd)))
    return out


def nccl_rank(solid, sdf, model, storage, params, seed_mid=True):
    """This process's slab (torch.distributed initialized with NCCL, one GPU
    per rank, the current device set): returns (solver, layout, stepper).
    The solver's work and the NCCL point-to-point operations share the
    rank's slab stream."""
    import torch
    import torch.distributed as dist
    rank, world = dist.get_rank(), dist.get_world_size()
    dev = torch.cuda.current_device()
    cmd = slab_stream(dev)
    s, lay, bufs = make_slab_solver(solid, sdf, rank, world, dev, model, storage, params, seed_mid, cmd)
    return s, lay, SlabStepper(s, lay, bufs, NcclExchange(), rank, cmd=cmd)
