"""flowcraft_b200 — B200-native Lattice-Boltzmann time step for FlowCraft.

The product is the CUDA library ``libfc_lbm.so`` (C ABI in include/fc_lbm.h);
``lbm.LbmSolver`` is its Python host mirror of FlowCraft's ``LbmSolver``.
"""
from .lbm import (LatticeModel, LbmError, LbmSolver, Params, Stats, Storage, Streaming, VoxelGrid,  # noqa: F401
                  load_library)

__all__ = ["LatticeModel", "LbmError", "LbmSolver", "Params", "Stats", "Storage", "Streaming", "VoxelGrid",
           "load_library"]
