"""The C-ABI library loads here (no GPU), exports every entry point that
include/fc_lbm.h declares, and behaves per the header on calls that need no
device: creation, error strings, parameter validation, and a clean
initialization failure when no CUDA device is visible."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT, gpu_available

HEADER = os.path.join(ROOT, "include", "fc_lbm.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^FC_LBM_API\s+[\w\s\*]+?\b(fc_lbm_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_the_surface():
    names = declared_functions()
    for n in ("fc_lbm_create", "fc_lbm_init", "fc_lbm_reset", "fc_lbm_reset_from_field", "fc_lbm_set_params",
              "fc_lbm_step", "fc_lbm_step_range", "fc_lbm_advance_substep", "fc_lbm_readback_field",
              "fc_lbm_readback_field_range", "fc_lbm_readback_stats", "fc_lbm_probe_slice_health",
              "fc_lbm_sync", "fc_lbm_shutdown", "fc_lbm_destroy", "fc_lbm_last_error"):
        assert n in names


def test_library_exports_every_declared_symbol(cuda_lib):
    lib = ctypes.CDLL(os.path.join(ROOT, "flowcraft_b200", "libfc_lbm.so"))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_mirror_binds_every_declared_symbol(cuda_lib):
    from flowcraft_b200.lbm import SIGNATURES
    assert sorted(SIGNATURES) == declared_functions()


def test_create_destroy_and_defaults(cuda_lib):
    from flowcraft_b200.lbm import LbmSolver, Params
    s = LbmSolver()
    assert not s.IsValid()
    p = s.GetParams()
    # LbmSolver::Params defaults (FlowCraft/LbmSolver.h:61-100)
    assert p == Params(0.8, 0.05, False, True, True, 0.12) or (
        abs(p.tau - 0.8) < 1e-7 and abs(p.inletVelocity - 0.05) < 1e-7 and not p.reverseFlow
        and p.freeSlipY and p.freeSlipZ and abs(p.smagorinskyCs - 0.12) < 1e-7)
    assert s.Nx() == 0 and s.CellCount() == 0
    s.close()


def test_set_params_validation(cuda_lib):
    from flowcraft_b200.lbm import LbmError, LbmSolver, Params
    s = LbmSolver()
    s.SetParams(Params(tau=0.53, inletVelocity=0.1, smagorinskyCs=0.0))
    assert abs(s.GetParams().tau - 0.53) < 1e-7
    for bad in (Params(tau=0.5), Params(tau=0.3), Params(tau=float("nan")), Params(smagorinskyCs=-0.1),
                Params(inletVelocity=float("inf"))):
        with pytest.raises(LbmError):
            s.SetParams(bad)
        assert abs(s.GetParams().tau - 0.53) < 1e-7  # unchanged after a rejected call
    assert "tau" in s.LastError()


def test_calls_before_init_report_not_initialized(cuda_lib):
    from flowcraft_b200 import lbm
    s = lbm.LbmSolver()
    lib = cuda_lib
    out = np.zeros(4, dtype=np.float32)
    assert lib.fc_lbm_step(s.handle, None, 1) == lbm.FC_LBM_ERR_NOT_INITIALIZED
    assert lib.fc_lbm_readback_field(s.handle, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), 4) == \
        lbm.FC_LBM_ERR_NOT_INITIALIZED
    assert "not initialized" in s.LastError()
    assert lib.fc_lbm_step(None, None, 1) == lbm.FC_LBM_ERR_INVALID_ARG


@pytest.mark.skipif(gpu_available(), reason="checks the no-device error path")
def test_init_without_device_fails_cleanly(cuda_lib):
    from flowcraft_b200.lbm import LbmSolver, VoxelGrid
    s = LbmSolver()
    g = VoxelGrid(8, 4, 4, solid=np.zeros(128, np.uint8))
    assert s.Init(0, g) is False
    assert "CUDA" in s.LastError() or "device" in s.LastError()
    assert not s.IsValid()


def test_init_rejects_bad_grids(cuda_lib):
    from flowcraft_b200.lbm import LbmSolver, VoxelGrid
    s = LbmSolver()
    assert s.Init(0, VoxelGrid(0, 4, 4, solid=np.zeros(0, np.uint8))) is False
    assert "positive" in s.LastError()
    assert s.Init(0, VoxelGrid(2000, 2000, 1100, solid=np.zeros(1, np.uint8))) is False
    assert "2^32" in s.LastError()


def test_init_rejects_unknown_option_flags(cuda_lib):
    from flowcraft_b200.lbm import OPTION_TC_CLOSURE, OPTION_TMA_STAGING, LbmSolver, Storage, Streaming, VoxelGrid
    s = LbmSolver()
    g = VoxelGrid(8, 4, 4, solid=np.zeros(128, np.uint8))
    bad = (OPTION_TMA_STAGING | OPTION_TC_CLOSURE) << 1
    assert s.Init(0, g, storage=Storage.FP16_OFFSET, streaming=Streaming.PINGPONG, flags=bad) is False
    assert "option flags" in s.LastError()
    assert not s.IsValid()
