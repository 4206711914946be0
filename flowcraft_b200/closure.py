"""The learned sub-grid closure's weights and their file format.

``ClosureWeights`` holds the MLP that ``LbmSolver.SetClosure`` installs
(``fc_lbm_set_closure`` in include/fc_lbm.h): 5 inputs -> 32 -> 32 -> 1 with
ReLU, inputs normalized by ``mean`` / ``std``, output nu_t = relu(z) *
``out_scale``, and the training range [lo, hi] of inputs 0-2 outside which a
cell keeps the Smagorinsky closure. ``wall_min`` (cells) extends that
fallback to the cells nearer a wall, and ``trust`` > 0 anchors the network to
Smagorinsky: 3 nu_t stays within a factor ``trust`` of the Smagorinsky
value. The inputs are
  0 log2(|Pi_neq| / rho), 1 tr(Pi_neq) / |Pi_neq|, 2 det(Pi_neq) / |Pi_neq|^3,
  3 wall distance (cells), 4 filter width.
Weights are input-major (w1[k, j] feeds input k to hidden unit j).
"""
from __future__ import annotations

import json
from dataclasses import dataclass, field

import numpy as np

N_IN = 5
HIDDEN = 32


@dataclass
class ClosureWeights:
    w1: np.ndarray = field(default_factory=lambda: np.zeros((N_IN, HIDDEN), np.float32))
    b1: np.ndarray = field(default_factory=lambda: np.zeros(HIDDEN, np.float32))
    w2: np.ndarray = field(default_factory=lambda: np.zeros((HIDDEN, HIDDEN), np.float32))
    b2: np.ndarray = field(default_factory=lambda: np.zeros(HIDDEN, np.float32))
    w3: np.ndarray = field(default_factory=lambda: np.zeros(HIDDEN, np.float32))
    b3: float = 0.0
    out_scale: float = 1.0
    mean: np.ndarray = field(default_factory=lambda: np.zeros(N_IN, np.float32))
    std: np.ndarray = field(default_factory=lambda: np.ones(N_IN, np.float32))
    lo: np.ndarray = field(default_factory=lambda: np.full(3, -np.inf, np.float32))
    hi: np.ndarray = field(default_factory=lambda: np.full(3, np.inf, np.float32))
    filter_width: float = 1.0
    # cells nearer a wall than wall_min cells keep Smagorinsky; trust > 0 holds
    # 3 nu_t within [d / trust, d * trust] of Smagorinsky's d (0: off)
    wall_min: float = 0.0
    trust: float = 0.0
    meta: dict = field(default_factory=dict)

    @staticmethod
    def random(seed: int = 0, out_scale: float = 1e-3, mean=None, std=None) -> "ClosureWeights":
        """He-initialized weights (for tests and timing)."""
        rng = np.random.default_rng(seed)
        cw = ClosureWeights()
        cw.w1 = rng.normal(0, np.sqrt(2.0 / N_IN), (N_IN, HIDDEN)).astype(np.float32)
        cw.b1 = rng.normal(0, 0.1, HIDDEN).astype(np.float32)
        cw.w2 = rng.normal(0, np.sqrt(2.0 / HIDDEN), (HIDDEN, HIDDEN)).astype(np.float32)
        cw.b2 = rng.normal(0, 0.1, HIDDEN).astype(np.float32)
        cw.w3 = rng.normal(0, np.sqrt(2.0 / HIDDEN), HIDDEN).astype(np.float32)
        cw.b3 = float(rng.normal(0, 0.1))
        cw.out_scale = out_scale
        if mean is not None:
            cw.mean = np.asarray(mean, np.float32)
        if std is not None:
            cw.std = np.asarray(std, np.float32)
        return cw

    def to_dict(self) -> dict:
        d = {k: (np.asarray(v).tolist() if isinstance(v, np.ndarray) else v) for k, v in self.__dict__.items()}
        for k in ("lo", "hi"):
            d[k] = [float(v) if np.isfinite(v) else ("inf" if v > 0 else "-inf") for v in np.asarray(getattr(self, k))]
        return d

    @staticmethod
    def from_dict(d: dict) -> "ClosureWeights":
        cw = ClosureWeights()
        for k, v in d.items():
            if k in ("lo", "hi"):
                v = [float(x) for x in v]
            if k in ("w1", "b1", "w2", "b2", "w3", "mean", "std", "lo", "hi"):
                v = np.asarray(v, dtype=np.float32)
            setattr(cw, k, v)
        return cw

    def save(self, path: str) -> None:
        with open(path, "w") as f:
            json.dump(self.to_dict(), f)

    @staticmethod
    def load(path: str) -> "ClosureWeights":
        with open(path) as f:
            return ClosureWeights.from_dict(json.load(f))
