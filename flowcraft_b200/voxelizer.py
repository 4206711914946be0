"""Python mirror of FlowCraft's ``Voxelizer`` (FlowCraft/Voxelizer.h:12-53)
over the CUDA voxelizer of ``libfc_lbm.so`` (``fc_lbm_voxel_grid`` and
``fc_lbm_voxelize`` in include/fc_lbm.h).

``Voxelizer.Voxelize(positions, indices, params)`` returns the same
``VoxelGrid`` the reference's CPU voxelizer returns for the same mesh, bit for
bit, computed on the GPU. ``positions`` is a (V, 3) float array (or a list of
(x, y, z) triples), ``indices`` a flat uint32 array of triangle corners.
``device`` selects where the result lives: ``None`` gives host numpy arrays
like the reference; a CUDA ordinal gives torch tensors on that device that
``LbmSolver.Init`` consumes without a host round trip.

There is no CPU fallback: every call goes to the CUDA library.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from .lbm import (FC_LBM_ERR_INVALID_ARG, FC_LBM_ERR_TOO_LARGE, FC_LBM_OK, FC_MEMORY_DEVICE, FC_MEMORY_HOST,
                  LbmError, VoxelGrid, _VoxelParams, load_library)


@dataclass
class Params:
    """Voxelizer::Params (Voxelizer.h:14-31), same defaults."""
    targetResolution: int = 640
    paddingFactor: tuple = (0.3, 1.0, 0.5)

    def _c(self) -> _VoxelParams:
        p = _VoxelParams()
        p.target_resolution = int(self.targetResolution)
        p.padding[:] = [float(v) for v in self.paddingFactor]
        return p


def _check(rc: int, what: str):
    if rc != FC_LBM_OK:
        raise LbmError(rc, f"{what} failed")


def _mesh_arrays(positions, indices, device):
    """Host numpy or device torch copies of the mesh, contiguous, in the ABI's types."""
    if device is None:
        pos = np.ascontiguousarray(np.asarray(positions, dtype=np.float32).reshape(-1, 3))
        idx = np.ascontiguousarray(np.asarray(indices, dtype=np.uint32).ravel())
        return pos, idx, pos.ctypes.data, idx.ctypes.data, FC_MEMORY_HOST
    import torch
    dev = torch.device("cuda", int(device))
    pos = torch.as_tensor(np.asarray(positions, dtype=np.float32).reshape(-1, 3)) if not torch.is_tensor(
        positions) else positions.to(torch.float32).reshape(-1, 3)
    idx_np = None if torch.is_tensor(indices) else np.asarray(indices, dtype=np.uint32).ravel().view(np.int32)
    idx = torch.as_tensor(idx_np) if idx_np is not None else indices.reshape(-1).to(torch.int32)
    pos = pos.to(dev).contiguous()
    idx = idx.to(dev).contiguous()
    return pos, idx, pos.data_ptr(), idx.data_ptr(), FC_MEMORY_DEVICE


def _count(a) -> int:
    return int(a.numel()) if hasattr(a, "numel") else int(a.size)


class _on_device:
    """Makes `device` current for the call (the ABI works on the current
    device) and yields torch's current stream there, or None for host calls."""

    def __init__(self, device):
        self.device = device
        self._ctx = None

    def __enter__(self):
        if self.device is None:
            return None
        import torch
        self._ctx = torch.cuda.device(int(self.device))
        self._ctx.__enter__()
        return torch.cuda.current_stream(int(self.device)).cuda_stream

    def __exit__(self, *exc):
        if self._ctx is not None:
            self._ctx.__exit__(*exc)


def GridForMesh(positions, params: Params = Params(), device=None):
    """(nx, ny, nz), cellSize, origin of the padded domain (Voxelizer.cpp:146-166)."""
    lib = load_library()
    pos, idx, pp, _, mem = _mesh_arrays(positions, np.zeros(0, np.uint32), device)
    dims = (ctypes.c_int32 * 3)()
    cell = ctypes.c_float()
    origin = (ctypes.c_float * 3)()
    p = params._c()
    with _on_device(device) as stream:
        rc = lib.fc_lbm_voxel_grid(pp, _count(pos) // 3, ctypes.byref(p), mem, dims, ctypes.byref(cell), origin,
                                   stream)
    _check(rc, "fc_lbm_voxel_grid")
    return (dims[0], dims[1], dims[2]), cell.value, (origin[0], origin[1], origin[2])


def VoxelizeOnGrid(positions, indices, dims, cellSize: float, origin, device=None) -> VoxelGrid:
    """Rasterization, flood fill and sign reconciliation onto an explicit grid."""
    lib = load_library()
    nx, ny, nz = (int(d) for d in dims)
    pos, idx, pp, ip, mem = _mesh_arrays(positions, indices, device)
    n = nx * ny * nz
    d = (ctypes.c_int32 * 3)(nx, ny, nz)
    o = (ctypes.c_float * 3)(*[float(v) for v in origin])
    if device is None:
        solid = np.empty(n, dtype=np.uint8)
        sdf = np.empty(n, dtype=np.float32)
        sp, dp = solid.ctypes.data, sdf.ctypes.data
    else:
        import torch
        solid = torch.empty(n, dtype=torch.uint8, device=f"cuda:{int(device)}")
        sdf = torch.empty(n, dtype=torch.float32, device=f"cuda:{int(device)}")
        sp, dp = solid.data_ptr(), sdf.data_ptr()
    with _on_device(device) as stream:
        rc = lib.fc_lbm_voxelize(pp, _count(pos) // 3, ip, _count(idx), d, ctypes.c_float(cellSize), o, mem, sp, dp,
                                 stream)
    if rc == FC_LBM_ERR_INVALID_ARG:
        raise ValueError("fc_lbm_voxelize: invalid mesh or grid (an index outside the vertex array?)")
    if rc == FC_LBM_ERR_TOO_LARGE:
        raise ValueError("fc_lbm_voxelize: grid too large")
    _check(rc, "fc_lbm_voxelize")
    return VoxelGrid(nx, ny, nz, float(cellSize), tuple(float(v) for v in origin), solid, sdf)


def Voxelize(positions, indices, params: Params = Params(), device=None) -> VoxelGrid:
    """Voxelizer::Voxelize (Voxelizer.cpp:136-485): the padded grid of the mesh,
    voxelized. An empty mesh (no vertices, fewer than 3 indices) gives the
    reference's empty grid."""
    npos = np.asarray(positions).size if not hasattr(positions, "numel") else positions.numel()
    nidx = np.asarray(indices).size if not hasattr(indices, "numel") else indices.numel()
    if npos == 0 or nidx < 3:
        return VoxelGrid(0, 0, 0, 1.0, (0.0, 0.0, 0.0), np.zeros(0, np.uint8), np.zeros(0, np.float32))
    dims, cell, origin = GridForMesh(positions, params, device)
    return VoxelizeOnGrid(positions, indices, dims, cell, origin, device)


class Voxelizer:
    """Namespace mirror of the reference class: ``Voxelizer.Voxelize(...)``."""
    Params = Params
    Voxelize = staticmethod(Voxelize)
    VoxelizeOnGrid = staticmethod(VoxelizeOnGrid)
    GridForMesh = staticmethod(GridForMesh)
