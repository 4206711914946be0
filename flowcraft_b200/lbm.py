"""Python host mirror of FlowCraft's ``LbmSolver`` (FlowCraft/LbmSolver.h:59-230)
over the C ABI of ``libfc_lbm.so`` (include/fc_lbm.h).

Method names, argument meanings and error behaviour follow the reference:
``Init`` returns a bool and sets ``LastError()``; ``ResetFromField`` with a
mis-sized field is ignored; ``Step``/``StepRange`` only enqueue; readbacks
block. ``cmd`` arguments (an SDL_GPUCommandBuffer in the reference) are a
CUDA stream here: ``None`` means the solver's own stream, or pass an int
handle / ``torch.cuda.Stream``.

There is no CPU fallback: importing works without a GPU, but every solver
call goes to the CUDA library and fails loudly if it is missing.
"""
from __future__ import annotations

import ctypes
import enum
import os
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfc_lbm.so")

FC_LBM_OK = 0
FC_LBM_ERR_INVALID_ARG = -1
FC_LBM_ERR_OUT_OF_MEMORY = -2
FC_LBM_ERR_CUDA = -3
FC_LBM_ERR_TIMEOUT = -4
FC_LBM_ERR_NOT_INITIALIZED = -5
FC_LBM_ERR_UNSUPPORTED = -6
FC_LBM_ERR_TOO_LARGE = -7

FC_MEMORY_HOST = 0
FC_MEMORY_DEVICE = 1


class LatticeModel(enum.IntEnum):
    """FlowCraft/LatticeModel.h:12 — same enumerator order."""
    D3Q15 = 0
    D3Q19 = 1


class Storage(enum.IntEnum):
    FP32 = 0
    FP16_OFFSET = 1
    BF16_OFFSET = 2


class Streaming(enum.IntEnum):
    PINGPONG = 0
    AA = 1


class _GridDesc(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
        ("cell_size", ctypes.c_float), ("origin", ctypes.c_float * 3),
        ("solid", ctypes.c_void_p), ("signed_distance", ctypes.c_void_p),
        ("memory", ctypes.c_int32),
    ]


class _Params(ctypes.Structure):
    _fields_ = [
        ("tau", ctypes.c_float), ("inlet_velocity", ctypes.c_float),
        ("reverse_flow", ctypes.c_int32), ("free_slip_y", ctypes.c_int32),
        ("free_slip_z", ctypes.c_int32), ("smagorinsky_cs", ctypes.c_float),
    ]


# fc_options.flags: stage the interior rows in shared memory by TMA tensor
# copies (16-bit formats; identical results, off by default)
OPTION_TMA_STAGING = 1
# fc_options.flags: the learned closure's MLP on the tcgen05 tensor cores,
# once per block of the ping-pong bulk step (FC_OPTION_TC_CLOSURE)
OPTION_TC_CLOSURE = 2


class _Options(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("storage", ctypes.c_int32),
                ("streaming", ctypes.c_int32), ("flags", ctypes.c_int32)]


class _Stats(ctypes.Structure):
    _fields_ = [
        ("avg_density", ctypes.c_float), ("min_density", ctypes.c_float), ("max_density", ctypes.c_float),
        ("avg_speed", ctypes.c_float), ("max_speed", ctypes.c_float),
        ("force_x", ctypes.c_float), ("force_y", ctypes.c_float), ("force_z", ctypes.c_float),
        ("max_stress", ctypes.c_float), ("has_nan", ctypes.c_int32), ("valid", ctypes.c_int32),
        ("total_mass", ctypes.c_double), ("force_sum", ctypes.c_double * 3),
        ("density_sum", ctypes.c_double), ("speed_sum", ctypes.c_double),
        ("fluid_cells", ctypes.c_uint64),
    ]


_FPTR = ctypes.POINTER(ctypes.c_float)


class _AeroForces(ctypes.Structure):
    _fields_ = [("force", ctypes.c_float * 3), ("min_stress", ctypes.c_float), ("max_stress", ctypes.c_float),
                ("center_of_pressure", ctypes.c_float * 3), ("lift_arrow_base", ctypes.c_float * 3),
                ("has_nan", ctypes.c_int32), ("force_sum", ctypes.c_double * 3),
                ("lift_weight_sum", ctypes.c_double), ("force_weight_sum", ctypes.c_double),
                ("solid_cells", ctypes.c_uint64)]


class _Closure(ctypes.Structure):
    _fields_ = [("w1", _FPTR), ("b1", _FPTR), ("w2", _FPTR), ("b2", _FPTR), ("w3", _FPTR), ("b3", ctypes.c_float),
                ("out_scale", ctypes.c_float), ("mean", ctypes.c_float * 5), ("std", ctypes.c_float * 5),
                ("lo", ctypes.c_float * 3), ("hi", ctypes.c_float * 3), ("filter_width", ctypes.c_float),
                ("min_wall_distance", ctypes.c_float), ("trust_factor", ctypes.c_float)]


class _VoxelParams(ctypes.Structure):
    _fields_ = [("target_resolution", ctypes.c_int32), ("padding", ctypes.c_float * 3)]


# Every function the header declares, with its ctypes signature.
_P = ctypes.c_void_p
_I32 = ctypes.c_int32
_SZ = ctypes.c_size_t
_FP = ctypes.POINTER(ctypes.c_float)
_U64P = ctypes.POINTER(ctypes.c_uint64)
_I32P = ctypes.POINTER(ctypes.c_int32)
SIGNATURES = {
    "fc_lbm_create": (ctypes.c_int, [ctypes.POINTER(_P)]),
    "fc_lbm_destroy": (None, [_P]),
    "fc_lbm_init": (ctypes.c_int, [_P, ctypes.POINTER(_GridDesc), _I32, ctypes.POINTER(_Options)]),
    "fc_lbm_shutdown": (ctypes.c_int, [_P]),
    "fc_lbm_last_error": (ctypes.c_char_p, [_P]),
    "fc_lbm_reset": (ctypes.c_int, [_P, ctypes.POINTER(_Params), _I32]),
    "fc_lbm_reset_from_field": (ctypes.c_int, [_P, _FP, _SZ]),
    "fc_lbm_set_params": (ctypes.c_int, [_P, ctypes.POINTER(_Params)]),
    "fc_lbm_get_params": (ctypes.c_int, [_P, ctypes.POINTER(_Params)]),
    "fc_lbm_step": (ctypes.c_int, [_P, _P, _I32]),
    "fc_lbm_step_range": (ctypes.c_int, [_P, _P, _I32, _I32]),
    "fc_lbm_advance_substep": (ctypes.c_int, [_P]),
    "fc_lbm_readback_field": (ctypes.c_int, [_P, _FP, _SZ]),
    "fc_lbm_readback_field_range": (ctypes.c_int, [_P, _I32, _I32, _FP, _SZ]),
    "fc_lbm_readback_stats": (ctypes.c_int, [_P, ctypes.POINTER(_Stats)]),
    "fc_lbm_probe_slice_health": (ctypes.c_int, [_P, _I32, _I32P]),
    "fc_lbm_has_diverged": (ctypes.c_int, [_P, _I32P]),
    "fc_lbm_copy_solid_mask": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_uint8), _SZ]),
    "fc_lbm_is_valid": (ctypes.c_int, [_P]),
    "fc_lbm_model": (ctypes.c_int, [_P]),
    "fc_lbm_dims": (ctypes.c_int, [_P, _I32P, _I32P, _I32P]),
    "fc_lbm_sync": (ctypes.c_int, [_P, _I32]),
    "fc_lbm_get_stream": (ctypes.c_int, [_P, ctypes.POINTER(_P)]),
    "fc_lbm_boundary_info": (ctypes.c_int, [_P, _U64P, _U64P, _U64P]),
    "fc_lbm_launch_count": (ctypes.c_int, [_P, _U64P]),
    "fc_lbm_step_timed": (ctypes.c_int, [_P, _I32, _FP, _FP, _FP]),
    "fc_lbm_save_populations": (ctypes.c_int, [_P, _FP, _SZ]),
    "fc_lbm_load_populations": (ctypes.c_int, [_P, _FP, _SZ]),
    "fc_lbm_stats_noalloc": (ctypes.c_int, [_P, _P, _P, _I32, _I32, _I32, _I32, _I32, _P, _P]),
    "fc_lbm_aero_forces": (ctypes.c_int, [_P, ctypes.POINTER(_AeroForces)]),
    "fc_lbm_set_closure": (ctypes.c_int, [_P, ctypes.POINTER(_Closure)]),
    "fc_lbm_closure_probe": (ctypes.c_int, [_P, _FP, ctypes.POINTER(ctypes.c_uint8), _SZ]),
    "fc_lbm_wall_distance": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_uint8), _SZ]),
    "fc_lbm_closure_coverage": (ctypes.c_int, [_P, _U64P, _U64P]),
    "fc_lbm_layer_copy": (ctypes.c_int, [_P, _I32, _I32, _P, _I32, _P]),
    "fc_lbm_layer_copy_dir": (ctypes.c_int, [_P, _I32, _I32, _P, _I32, _I32, _P]),
    "fc_lbm_readback_field_async": (ctypes.c_int, [_P, _P, _SZ]),
    "fc_lbm_readback_wait": (ctypes.c_int, [_P, _I32]),
    "fc_lbm_alloc_pinned": (ctypes.c_int, [_SZ, ctypes.POINTER(ctypes.c_void_p)]),
    "fc_lbm_free_pinned": (ctypes.c_int, [_P]),
    "fc_lbm_particles_reset": (ctypes.c_int, [_P, _I32, _I32, ctypes.c_uint64, _I32, _I32]),
    "fc_lbm_particles_step": (ctypes.c_int, [_P, _I32, ctypes.c_float, ctypes.c_float, _I32, _I32, _I32]),
    "fc_lbm_particles_scatter": (ctypes.c_int, [_P, _I32, _I32]),
    "fc_lbm_particles_shift_plane": (ctypes.c_int, [_P, _I32, _I32]),
    "fc_lbm_particles_read": (ctypes.c_int, [_P, _FP, _SZ, _I32P, _SZ]),
    "fc_lbm_particles_set": (ctypes.c_int, [_P, _FP, _SZ]),
    "fc_lbm_batch_create": (ctypes.c_int, [ctypes.POINTER(_P), _I32, ctypes.POINTER(_P)]),
    "fc_lbm_batch_destroy": (None, [_P]),
    "fc_lbm_batch_last_error": (ctypes.c_char_p, [_P]),
    "fc_lbm_batch_step": (ctypes.c_int, [_P, _I32]),
    "fc_lbm_batch_config": (ctypes.c_int, [_P, _I32, _I32]),
    "fc_lbm_batch_tune": (ctypes.c_int, [_P, _I32, _I32P, _I32P, _FP]),
    "fc_lbm_closure_samples": (ctypes.c_int, [_P, ctypes.c_float, _P, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]),
    "fc_lbm_mlp_forward": (ctypes.c_int, [_P, _P, ctypes.c_int64, _P, _P]),
    "fc_lbm_mlp_grad": (ctypes.c_int, [_P, _P, _P, _P, ctypes.c_int64, _P, _P, _P, _P]),
    "fc_lbm_mlp_adam": (ctypes.c_int, [_P, _P, _P, _P, _I32, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                       ctypes.c_float, _P]),
    "fc_lbm_voxel_grid": (ctypes.c_int, [_P, _SZ, ctypes.POINTER(_VoxelParams), _I32, _I32P, _FP, _FP, _P]),
    "fc_lbm_voxelize": (ctypes.c_int, [_P, _SZ, _P, _SZ, _I32P, ctypes.c_float, _FP, _I32, _P, _P, _P]),
}

_lib = None


def load_library(path: str = LIB_PATH):
    """Loads libfc_lbm.so and binds every entry point; raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"CUDA library not built: {path} (run python -m flowcraft_b200.build)")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class LbmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{msg} (status {code})")
        self.code = code


@dataclass
class Params:
    """LbmSolver::Params (LbmSolver.h:61-100), same defaults."""
    tau: float = 0.8
    inletVelocity: float = 0.05
    reverseFlow: bool = False
    freeSlipY: bool = True
    freeSlipZ: bool = True
    smagorinskyCs: float = 0.12

    def _c(self) -> _Params:
        return _Params(self.tau, self.inletVelocity, int(self.reverseFlow), int(self.freeSlipY),
                       int(self.freeSlipZ), self.smagorinskyCs)


@dataclass
class VoxelGrid:
    """FlowCraft/VoxelGrid.h:13-61. ``solid`` / ``signedDistance`` are flat
    (or (nz, ny, nx)) numpy arrays, or CUDA torch tensors for device input."""
    nx: int = 0
    ny: int = 0
    nz: int = 0
    cellSize: float = 1.0
    origin: tuple = (0.0, 0.0, 0.0)
    solid: object = None
    signedDistance: object = None

    def CellCount(self) -> int:
        return self.nx * self.ny * self.nz

    def Index(self, x: int, y: int, z: int) -> int:
        return (z * self.ny + y) * self.nx + x


@dataclass
class Stats:
    """LbmSolver::Stats (LbmSolver.h:172-184) plus the FP64 sums."""
    avgDensity: float = 0.0
    minDensity: float = 0.0
    maxDensity: float = 0.0
    avgSpeed: float = 0.0
    maxSpeed: float = 0.0
    forceX: float = 0.0
    forceY: float = 0.0
    forceZ: float = 0.0
    maxStress: float = 0.0
    hasNaN: bool = False
    valid: bool = False
    totalMass: float = 0.0
    forceSum: tuple = (0.0, 0.0, 0.0)
    fluidCells: int = 0
    extra: dict = field(default_factory=dict)


@dataclass
class AerodynamicForces:
    """FieldOverlay::AerodynamicForces (FieldOverlay.h:186-195) plus the FP64
    sums the device integral produces."""
    forceX: float = 0.0
    forceY: float = 0.0
    forceZ: float = 0.0
    minStress: float = 0.0
    maxStress: float = 0.0
    centerOfPressure: tuple = (0.0, 0.0, 0.0)
    liftArrowBase: tuple = (0.0, 0.0, 0.0)
    hasNaN: bool = False
    forceSum: tuple = (0.0, 0.0, 0.0)
    liftWeightSum: float = 0.0
    forceWeightSum: float = 0.0
    solidCells: int = 0


def _stream_ptr(cmd) -> int | None:
    if cmd is None:
        return None
    if isinstance(cmd, int):
        return cmd
    handle = getattr(cmd, "cuda_stream", None)  # torch.cuda.Stream
    if handle is not None:
        return int(handle)
    raise TypeError("cmd must be None, an int cudaStream_t or a torch.cuda.Stream")


class LbmSolver:
    """CUDA-backed drop-in for the reference's SDL_GPU ``LbmSolver``."""

    def __init__(self):
        self._lib = load_library()
        h = ctypes.c_void_p()
        rc = self._lib.fc_lbm_create(ctypes.byref(h))
        if rc != FC_LBM_OK:
            raise LbmError(rc, "fc_lbm_create failed")
        self._h = h
        self._solid_cpu = np.zeros(0, dtype=np.uint8)
        self._model = LatticeModel.D3Q19
        self._device = 0
        self._keep = []

    # -- lifetime --------------------------------------------------------
    def __del__(self):
        try:
            if getattr(self, "_h", None):
                self._lib.fc_lbm_destroy(self._h)
                self._h = None
        except Exception:
            pass

    def close(self):
        if self._h:
            self._lib.fc_lbm_destroy(self._h)
            self._h = None

    def _check(self, rc: int, what: str):
        if rc != FC_LBM_OK:
            raise LbmError(rc, f"{what}: {self.LastError()}")

    @property
    def handle(self):
        return self._h

    def Init(self, device, grid: VoxelGrid, model: LatticeModel = LatticeModel.D3Q19,
             storage: Storage = Storage.FP32, streaming: Streaming = Streaming.PINGPONG, flags: int = 0) -> bool:
        """LbmSolver::Init (LbmSolver.cpp:205-366); ``device`` is a CUDA ordinal."""
        self._device = int(device)
        desc = _GridDesc()
        desc.nx, desc.ny, desc.nz = grid.nx, grid.ny, grid.nz
        desc.cell_size = grid.cellSize
        desc.origin[:] = list(grid.origin)
        solid, sdf = grid.solid, grid.signedDistance
        keep = []
        if hasattr(solid, "data_ptr"):  # torch tensor on a CUDA device
            desc.memory = FC_MEMORY_DEVICE
            solid = solid.contiguous()
            desc.solid = solid.data_ptr()
            keep.append(solid)
            if sdf is not None and sdf.numel() == grid.CellCount():
                sdf = sdf.contiguous()
                desc.signed_distance = sdf.data_ptr()
                keep.append(sdf)
            self._solid_cpu = None
        else:
            desc.memory = FC_MEMORY_HOST
            solid = np.ascontiguousarray(np.asarray(solid, dtype=np.uint8).ravel())
            desc.solid = solid.ctypes.data
            keep.append(solid)
            # a mis-sized SDF is treated as absent (LbmReference.cpp:162-166)
            if sdf is not None and np.asarray(sdf).size == grid.CellCount():
                sdf = np.ascontiguousarray(np.asarray(sdf, dtype=np.float32).ravel())
                desc.signed_distance = sdf.ctypes.data
                keep.append(sdf)
            self._solid_cpu = solid.copy()
        opts = _Options(int(device), int(storage), int(streaming), int(flags))
        rc = self._lib.fc_lbm_init(self._h, ctypes.byref(desc), int(model), ctypes.byref(opts))
        if rc == FC_LBM_OK:
            self._model = LatticeModel(model)
            if self._solid_cpu is None:
                self._solid_cpu = np.empty(grid.CellCount(), dtype=np.uint8)
                self._check(self._lib.fc_lbm_copy_solid_mask(
                    self._h, self._solid_cpu.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)),
                    self._solid_cpu.size), "copy solid mask")
        return rc == FC_LBM_OK

    def Shutdown(self):
        self._lib.fc_lbm_shutdown(self._h)

    def LastError(self) -> str:
        return self._lib.fc_lbm_last_error(self._h).decode()

    # -- state -----------------------------------------------------------
    def Reset(self, params: Params, seedAtMidSpeed: bool = False):
        self._check(self._lib.fc_lbm_reset(self._h, ctypes.byref(params._c()), int(seedAtMidSpeed)), "Reset")

    def ResetFromField(self, field) -> None:
        """Silently ignores a field of the wrong size, like LbmSolver.cpp:430."""
        f = np.ascontiguousarray(np.asarray(field, dtype=np.float32).ravel())
        rc = self._lib.fc_lbm_reset_from_field(self._h, f.ctypes.data_as(_FP), f.size)
        if rc not in (FC_LBM_OK, FC_LBM_ERR_INVALID_ARG):
            self._check(rc, "ResetFromField")

    def SetParams(self, params: Params) -> None:
        self._check(self._lib.fc_lbm_set_params(self._h, ctypes.byref(params._c())), "SetParams")

    def GetParams(self) -> Params:
        p = _Params()
        self._check(self._lib.fc_lbm_get_params(self._h, ctypes.byref(p)), "GetParams")
        return Params(p.tau, p.inlet_velocity, bool(p.reverse_flow), bool(p.free_slip_y), bool(p.free_slip_z),
                      p.smagorinsky_cs)

    # -- stepping --------------------------------------------------------
    def Step(self, cmd, numSubsteps: int):
        self._check(self._lib.fc_lbm_step(self._h, _stream_ptr(cmd), int(numSubsteps)), "Step")

    def StepRange(self, cmd, zStart: int, zCount: int):
        self._check(self._lib.fc_lbm_step_range(self._h, _stream_ptr(cmd), int(zStart), int(zCount)), "StepRange")

    def AdvanceSubstep(self):
        self._check(self._lib.fc_lbm_advance_substep(self._h), "AdvanceSubstep")

    def Sync(self, timeout_ms: int = -1):
        self._check(self._lib.fc_lbm_sync(self._h, int(timeout_ms)), "Sync")

    # -- readback --------------------------------------------------------
    def ReadbackField(self) -> np.ndarray:
        out = np.empty(self.CellCount() * 4, dtype=np.float32)
        self._check(self._lib.fc_lbm_readback_field(self._h, out.ctypes.data_as(_FP), out.size), "ReadbackField")
        return out

    def ReadbackFieldRange(self, zStart: int, zCount: int, outField: np.ndarray) -> None:
        if outField.dtype != np.float32 or not outField.flags.c_contiguous:
            raise TypeError("outField must be a contiguous float32 array of 4*CellCount()")
        self._check(self._lib.fc_lbm_readback_field_range(self._h, int(zStart), int(zCount),
                                                          outField.ctypes.data_as(_FP), outField.size),
                    "ReadbackFieldRange")

    def ReadbackStats(self) -> Stats:
        s = _Stats()
        self._check(self._lib.fc_lbm_readback_stats(self._h, ctypes.byref(s)), "ReadbackStats")
        return Stats(s.avg_density, s.min_density, s.max_density, s.avg_speed, s.max_speed, s.force_x, s.force_y,
                     s.force_z, s.max_stress, bool(s.has_nan), bool(s.valid), s.total_mass, tuple(s.force_sum),
                     int(s.fluid_cells), {"density_sum": s.density_sum, "speed_sum": s.speed_sum})

    def AerodynamicForces(self) -> AerodynamicForces:
        """FieldOverlay::ComputeAerodynamicForces (FieldOverlay.cpp:469-621) of
        the current state, integrated on the device in FP64 (no field readback)."""
        a = _AeroForces()
        self._check(self._lib.fc_lbm_aero_forces(self._h, ctypes.byref(a)), "AerodynamicForces")
        return AerodynamicForces(a.force[0], a.force[1], a.force[2], a.min_stress, a.max_stress,
                                 tuple(a.center_of_pressure), tuple(a.lift_arrow_base), bool(a.has_nan),
                                 tuple(a.force_sum), a.lift_weight_sum, a.force_weight_sum, int(a.solid_cells))

    def SetClosure(self, weights) -> None:
        """Installs a learned closure (flowcraft_b200.closure.ClosureWeights),
        or returns to Smagorinsky with None. Raises LbmError when the storage
        format or lattice cannot take it."""
        if weights is None:
            self._check(self._lib.fc_lbm_set_closure(self._h, None), "SetClosure")
            return
        keep = [np.ascontiguousarray(a, dtype=np.float32) for a in
                (weights.w1, weights.b1, weights.w2, weights.b2, weights.w3)]
        c = _Closure()
        c.w1, c.b1, c.w2, c.b2, c.w3 = (a.ctypes.data_as(_FPTR) for a in keep)
        c.b3 = float(weights.b3)
        c.out_scale = float(weights.out_scale)
        c.mean[:] = [float(v) for v in weights.mean]
        c.std[:] = [float(v) for v in weights.std]
        c.lo[:] = [float(v) for v in weights.lo]
        c.hi[:] = [float(v) for v in weights.hi]
        c.filter_width = float(weights.filter_width)
        c.min_wall_distance = float(getattr(weights, "wall_min", 0.0))
        c.trust_factor = float(getattr(weights, "trust", 0.0))
        self._check(self._lib.fc_lbm_set_closure(self._h, ctypes.byref(c)), "SetClosure")

    def ClosureProbe(self):
        """(inputs (N, 4), nu_t (N,), in_range (N,) bool) of the installed
        closure on the current populations as stored."""
        n = self.CellCount()
        out = np.empty(n * 5, dtype=np.float32)
        rng = np.empty(n, dtype=np.uint8)
        self._check(self._lib.fc_lbm_closure_probe(self._h, out.ctypes.data_as(_FP),
                                                   rng.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), n),
                    "ClosureProbe")
        out = out.reshape(n, 5)
        return out[:, :4], out[:, 4], rng.astype(bool)

    def ClosureSamples(self, filterWidth: float = 2.0, out=None):
        """Training samples of the closure from a 2x box filter of this
        lattice: a CUDA tensor (rows, 6) of inputs 0-4 and the target nu_t
        (allocated here when `out` is None)."""
        import torch
        cnt = ctypes.c_int64(0)
        rc = self._lib.fc_lbm_closure_samples(self._h, float(filterWidth), None, 0, ctypes.byref(cnt))
        if rc not in (FC_LBM_OK, FC_LBM_ERR_TOO_LARGE):
            self._check(rc, "ClosureSamples")
        n = int(cnt.value)
        if out is None:
            out = torch.empty((max(n, 1), 6), dtype=torch.float32, device=f"cuda:{self._device}")
        self._check(self._lib.fc_lbm_closure_samples(self._h, float(filterWidth), out.data_ptr(), out.shape[0],
                                                     ctypes.byref(cnt)), "ClosureSamples")
        return out[:n]

    def ClosureCoverage(self) -> dict:
        """Cells in the closure's training range and warps that run its MLP."""
        a, b = ctypes.c_uint64(), ctypes.c_uint64()
        self._check(self._lib.fc_lbm_closure_coverage(self._h, ctypes.byref(a), ctypes.byref(b)), "ClosureCoverage")
        n = self.CellCount()
        warps = (n + 63) // 64
        return {"cells_in_range": int(a.value), "cell_fraction": a.value / max(n, 1),
                "warps_with_mlp": int(b.value), "warp_fraction": b.value / max(warps, 1)}

    def ReadbackFieldAsync(self, out) -> None:
        """Starts a readback of the current field (4 floats per cell) into
        `out` (a float32 array of 4*CellCount(), ideally from PinnedBuffer)
        and returns; steps issued meanwhile overlap the copy. Keep `out`
        alive until ReadbackWait()."""
        if not isinstance(out, np.ndarray) or out.dtype != np.float32 or not out.flags.c_contiguous:
            raise TypeError("out must be a contiguous float32 array of 4*CellCount()")
        self._rb_out = out  # the copy lands here later
        self._check(self._lib.fc_lbm_readback_field_async(self._h, out.ctypes.data, out.size), "ReadbackFieldAsync")

    def ReadbackWait(self, timeout_ms: int = -1) -> None:
        self._check(self._lib.fc_lbm_readback_wait(self._h, int(timeout_ms)), "ReadbackWait")
        self._rb_out = None

    def LayerCopy(self, z: int, buffer_ptr: int, to_buffer: bool, next_set: bool = False, cmd=None,
                  ez: int = 0) -> None:
        """Packs (to_buffer) or unpacks z-layer `z` of the current (or, with
        next_set, the in-progress step's output) population set to / from a
        device buffer of Q*nx*ny elements; with ez = +1 or -1 only the 5
        planes with that e_z, as the buffer's first 5 rows."""
        if ez:
            self._check(self._lib.fc_lbm_layer_copy_dir(self._h, int(z), int(next_set), buffer_ptr, int(to_buffer),
                                                        int(ez), _stream_ptr(cmd)), "LayerCopy")
            return
        self._check(self._lib.fc_lbm_layer_copy(self._h, int(z), int(next_set), buffer_ptr, int(to_buffer),
                                                _stream_ptr(cmd)), "LayerCopy")

    def WallDistance(self) -> np.ndarray:
        """The closure's wall-distance input, bytes in 1/16-cell steps."""
        n = self.CellCount()
        out = np.empty(n, dtype=np.uint8)
        self._check(self._lib.fc_lbm_wall_distance(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), n),
                    "WallDistance")
        return out

    def ProbeSliceHealth(self, zLayer: int) -> bool:
        d = ctypes.c_int32()
        self._check(self._lib.fc_lbm_probe_slice_health(self._h, int(zLayer), ctypes.byref(d)), "ProbeSliceHealth")
        return bool(d.value)

    def HasDiverged(self) -> bool:
        d = ctypes.c_int32()
        self._check(self._lib.fc_lbm_has_diverged(self._h, ctypes.byref(d)), "HasDiverged")
        return bool(d.value)

    def SavePopulations(self) -> np.ndarray:
        q = 19 if self._model == LatticeModel.D3Q19 else 15
        out = np.empty(q * self.CellCount(), dtype=np.float32)
        self._check(self._lib.fc_lbm_save_populations(self._h, out.ctypes.data_as(_FP), out.size), "SavePopulations")
        return out.reshape(q, self.CellCount())

    def LoadPopulations(self, pops: np.ndarray) -> None:
        p = np.ascontiguousarray(np.asarray(pops, dtype=np.float32).ravel())
        self._check(self._lib.fc_lbm_load_populations(self._h, p.ctypes.data_as(_FP), p.size), "LoadPopulations")

    # -- queries ---------------------------------------------------------
    def SolidMask(self) -> np.ndarray:
        return self._solid_cpu

    def IsValid(self) -> bool:
        return bool(self._lib.fc_lbm_is_valid(self._h))

    def Model(self) -> LatticeModel:
        return self._model

    def _dims(self):
        x, y, z = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        self._lib.fc_lbm_dims(self._h, ctypes.byref(x), ctypes.byref(y), ctypes.byref(z))
        return x.value, y.value, z.value

    def Nx(self) -> int:
        return self._dims()[0]

    def Ny(self) -> int:
        return self._dims()[1]

    def Nz(self) -> int:
        return self._dims()[2]

    def CellCount(self) -> int:
        x, y, z = self._dims()
        return x * y * z

    def Stream(self) -> int:
        s = ctypes.c_void_p()
        self._check(self._lib.fc_lbm_get_stream(self._h, ctypes.byref(s)), "get_stream")
        return s.value or 0

    def BoundaryInfo(self) -> dict:
        a, b, c = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        self._lib.fc_lbm_boundary_info(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
        return {"boundary_cells": a.value, "bouzidi_links": b.value, "bulk_cells": c.value}

    def StepTimed(self, n: int) -> dict:
        """n substeps on the solver's stream with CUDA events around every
        launch: device ms of the sequence and of the bulk / boundary kernels."""
        t, b, d = ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
        self._check(self._lib.fc_lbm_step_timed(self._h, int(n), ctypes.byref(t), ctypes.byref(b), ctypes.byref(d)),
                    "StepTimed")
        return {"total_ms": t.value, "bulk_ms": b.value, "boundary_ms": d.value}

    def LaunchCount(self) -> int:
        v = ctypes.c_uint64()
        self._lib.fc_lbm_launch_count(self._h, ctypes.byref(v))
        return v.value


class PinnedBuffer:
    """Page-locked host float32 array (fc_lbm_alloc_pinned), for
    asynchronous readbacks. ``.array`` is the numpy view; free() or garbage
    collection releases it."""

    def __init__(self, count: int):
        self._lib = load_library()
        p = ctypes.c_void_p()
        rc = self._lib.fc_lbm_alloc_pinned(int(count) * 4, ctypes.byref(p))
        if rc != FC_LBM_OK:
            raise LbmError(rc, "fc_lbm_alloc_pinned failed")
        self._p = p.value
        buf = (ctypes.c_float * int(count)).from_address(self._p)
        self.array = np.ctypeslib.as_array(buf)

    def free(self):
        if getattr(self, "_p", None):
            self.array = None
            self._lib.fc_lbm_free_pinned(self._p)
            self._p = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass
