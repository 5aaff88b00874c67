"""make_cuda_backend() (the ExecutionBackend contract of the C++ host layer on
the B200) through a C++ test program written like the reference's backend
tests: compiled here with g++ against include/ and run as a subprocess."""

import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "vikalp_b200")
BIN_DIR = os.path.join(ROOT, "tests", "cpp", "_bin")


@pytest.fixture(scope="module")
def test_binary():
    from vikalp_b200 import build
    build.build_host()
    os.makedirs(BIN_DIR, exist_ok=True)
    exe = os.path.join(BIN_DIR, "test_backend")
    src = os.path.join(ROOT, "tests", "cpp", "test_backend.cpp")
    cmd = [build.CXX, "-std=c++20", "-O1", "-I", os.path.join(ROOT, "include"), src, "-L", PKG, "-lvikalp",
           "-lvikalp_b200", f"-Wl,-rpath,{PKG}", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_backend_program_builds(test_binary):
    # compile-and-link check without a GPU: every symbol the backend uses resolves
    assert os.path.exists(test_binary)


@pytest.mark.gpu
def test_backend_on_gpu(test_binary):
    r = subprocess.run([test_binary, "gpu"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ALL CHECKS PASSED" in r.stdout
