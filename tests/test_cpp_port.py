"""The C++ host mirror (include/fc_lbm_solver.hpp) compiles against the C ABI
and links; on a GPU, the restated reference test passes bit-for-bit and
fc::Voxelize matches the voxelizer oracle."""
import os
import subprocess

import pytest

from conftest import ROOT

SRC = os.path.join(ROOT, "tests", "cpp", "gpu_vs_cpu_test.cpp")


def _build(tmp_path):
    exe = str(tmp_path / "gpu_vs_cpu_test")
    lib_dir = os.path.join(ROOT, "flowcraft_b200")
    ora_dir = os.path.join(ROOT, "oracle")
    cmd = ["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-I" + os.path.join(ROOT, "include"), SRC, "-o", exe,
           "-L" + lib_dir, "-lfc_lbm", "-L" + ora_dir, "-l:liblbm_oracle32.so", "-l:libvoxel_oracle.so",
           "-Wl,-rpath," + lib_dir + ":" + ora_dir, "-pthread"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_cpp_mirror_compiles_and_links(cuda_lib, oracle_built, tmp_path):
    assert os.path.exists(_build(tmp_path))


@pytest.mark.gpu
def test_cpp_gpu_vs_cpu(gpu, oracle_built, tmp_path):
    exe = _build(tmp_path)
    res = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    print(res.stdout)
    assert res.returncode == 0, res.stdout + res.stderr
    assert res.stdout.count("PASS") == 3
