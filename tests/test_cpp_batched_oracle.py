"""vikalp::BatchedRelaxationOracle (branch-and-bound node relaxations in one
device batch) through a C++ test program written like the reference's
branch-and-bound tests: compiled here with g++ against include/ and run as a
subprocess."""

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
    exe = os.path.join(BIN_DIR, "test_batched_oracle")
    src = os.path.join(ROOT, "tests", "cpp", "test_batched_oracle.cpp")
    cmd = [build.CXX, "-std=c++20", "-O1", "-I", os.path.join(ROOT, "include"), src, "-L", PKG, "-lvikalp",
           "-lvikalp_b200", f"-Wl,-rpath,{PKG}", "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_batched_oracle_routes_without_gpu(test_binary):
    r = subprocess.run([test_binary, "cpu"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ALL CHECKS PASSED" in r.stdout


@pytest.mark.gpu
def test_batched_oracle_on_gpu(test_binary):
    r = subprocess.run([test_binary, "gpu"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ALL CHECKS PASSED" in r.stdout
