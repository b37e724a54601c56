"""The C++ interface (include/smina_b200.hpp), shaped like the reference's
gpusmina::GpuDocking, compiled against the public headers and linked with
the engine library; tests/cpp/gpu_docking_api_test.cpp checks its settings
validation, device-list parsing and error behaviour on a machine without a
device."""
import os
import subprocess

import pytest

from conftest import has_gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "gpu-smina_b200", "lib")


def _build(tmp_path):
    exe = str(tmp_path / "gpu_docking_api_test")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "gpu_docking_api_test.cpp"), "-L", LIBDIR, "-lsmina_b200",
           f"-Wl,-rpath,{LIBDIR}", "-pthread", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


@pytest.mark.skipif(has_gpu(), reason="checks the behaviour without a device")
def test_cpp_interface_without_a_device(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([exe, "host"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "0 failure(s)" in r.stdout


@pytest.mark.gpu
def test_cpp_interface_on_the_device(tmp_path):
    """parallel_mc (FP32 and FP64 engines), dock_batch, refine and
    minimize_batch through the GpuDocking-shaped class give, bit for bit,
    what the same work gives through the C ABI directly."""
    exe = _build(tmp_path)
    r = subprocess.run([exe, "device"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "device: 0 failure(s)" in r.stdout
