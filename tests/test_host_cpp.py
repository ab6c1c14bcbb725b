"""Runs the C++ test executable of the host library (ladds_b200/host/tests/test_host.cpp):
the interface mirror of the reference (Particle, ConfigReader, Integrator,
GpuCollisionFunctor, HotPathLoop)."""
import subprocess

import pytest


@pytest.fixture(scope="module")
def host_test():
    from ladds_b200 import build

    build.build_gpu()
    return build.build_host_tests()


def test_host_library_cpu(host_test):
    r = subprocess.run([host_test, "cpu"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr


@pytest.mark.gpu
def test_host_library_gpu(host_test):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    r = subprocess.run([host_test, "gpu"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
