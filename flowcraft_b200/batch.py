"""Many lattices stepped together (``fc_lbm_batch_*`` in include/fc_lbm.h):
one bulk launch over the tiles of every member per step (persistent, or one
block per tile; or each member's own bulk kernel, side by side, when the
autotuner finds that faster), pairs of steps replayed as a CUDA graph, block shape picked by an
autotuner. The
members stay ordinary ``LbmSolver`` objects (readbacks, forces, SetParams);
the batch only steps them, bit-identically to ``LbmSolver.Step``."""
from __future__ import annotations

import ctypes

import numpy as np

from .lbm import FC_LBM_OK, LbmError, load_library

# (rows, grid_mult): the persistent launch's block shapes (grid_mult 1, 2),
# the one-block-per-tile launch (8, 0), then rows 0: every member's
# own bulk kernel, run side by side on forked streams
CANDIDATES = [(r, m) for r in (4, 8, 16) for m in (1, 2)] + [(8, 0), (0, 1)]


def candidate_name(c) -> str:
    if not c[0]:
        return "per_member"
    return "per_tile" if c[1] == 0 else f"rows{c[0]}_x{c[1]}"


class LbmBatch:
    def __init__(self, members):
        self._lib = load_library()
        self.members = list(members)
        arr = (ctypes.c_void_p * len(self.members))(*[m.handle for m in self.members])
        h = ctypes.c_void_p()
        rc = self._lib.fc_lbm_batch_create(arr, len(self.members), ctypes.byref(h))
        if rc != FC_LBM_OK:
            raise LbmError(rc, "fc_lbm_batch_create failed (members must share device, model and storage, have "
                               "an even nx and no learned closure)")
        self._h = h

    def _check(self, rc, what):
        if rc != FC_LBM_OK:
            raise LbmError(rc, f"{what}: {self._lib.fc_lbm_batch_last_error(self._h).decode()}")

    def Step(self, n: int) -> None:
        self._check(self._lib.fc_lbm_batch_step(self._h, int(n)), "batch step")

    def Config(self, rows: int = 8, grid_mult: int = 1) -> None:
        self._check(self._lib.fc_lbm_batch_config(self._h, int(rows), int(grid_mult)), "batch config")

    def Tune(self, steps: int = 10) -> dict:
        """Times the block shapes on real steps (each member advances by
        len(CANDIDATES) * (steps + 2) steps, even steps rounded up) and keeps
        the fastest."""
        r, m = ctypes.c_int32(), ctypes.c_int32()
        ms = (ctypes.c_float * len(CANDIDATES))()
        self._check(self._lib.fc_lbm_batch_tune(self._h, int(steps), ctypes.byref(r), ctypes.byref(m), ms),
                    "batch tune")
        return {"rows": r.value, "grid_mult": m.value,
                "ms_per_step": {candidate_name(c): float(ms[i])
                                for i, c in enumerate(CANDIDATES)}}

    def close(self):
        if getattr(self, "_h", None):
            self._lib.fc_lbm_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
