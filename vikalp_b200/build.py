"""Builds the sm_100a CUDA library ``vikalp_b200/libvikalp_b200.so`` in-tree.

Usage: ``python -m vikalp_b200.build [--force] [--jobs N]``.

Every ``csrc/*.cu`` / ``csrc/*.cpp`` compiles with nvcc for
``-gencode arch=compute_100a,code=sm_100a`` into ``_build/`` (object files are
reused while newer than their source and every header), then links into one
shared library with the CUDA runtime linked statically.
"""

from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(PKG, "libvikalp_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-I", os.path.join(ROOT, "include"), "-I", CSRC]


def _headers() -> list[str]:
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))


def _stale(obj: str, src: str, newest_header: float) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return t < os.path.getmtime(src) or t < newest_header


def _compile(src: str, extra: list[str]) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    cmd = [NVCC, *ARCH, *FLAGS, *extra, "-c", src, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [NVCC, *FLAGS, *extra, "-x", "c++", "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj


def build(force: bool = False, jobs: int | None = None, verbose: bool = False, extra: list[str] | None = None) -> str:
    os.makedirs(BUILD, exist_ok=True)
    extra = extra or []
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    newest = max((os.path.getmtime(h) for h in _headers()), default=0.0)
    todo = [s for s in srcs if force or _stale(os.path.join(BUILD, os.path.basename(s) + ".o"), s, newest)]
    objs = [os.path.join(BUILD, os.path.basename(s) + ".o") for s in srcs]
    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
            for f in [ex.submit(_compile, s, extra) for s in todo]:
                f.result()
    if todo or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objs]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    build_host(force=force)
    if verbose:
        print(f"built {LIB} ({len(todo)} objects recompiled) and {HOST_LIB}")
    return LIB


HOST_LIB = os.path.join(PKG, "libvikalp.so")
# The system compiler, whose libstdc++ is the shared one every Python process
# here already has loaded (through numpy); a toolchain that links libstdc++
# statically would put a second copy of the C++ runtime (iostreams, locales)
# into the process.
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else os.environ.get("CXX", "g++")


def build_host(force: bool = False) -> str:
    """The C++20 host layer (vikalp::solve and the contracts) over the C ABI."""
    srcs = sorted(glob.glob(os.path.join(PKG, "host", "*.cpp")))
    hdrs = glob.glob(os.path.join(ROOT, "include", "**", "*.h*"), recursive=True)
    newest = max([os.path.getmtime(p) for p in srcs + hdrs + [LIB]], default=0.0)
    if not force and os.path.exists(HOST_LIB) and os.path.getmtime(HOST_LIB) >= newest:
        return HOST_LIB
    cmd = [CXX, "-std=c++20", "-O2", "-fPIC", "-shared", "-I", os.path.join(ROOT, "include"), *srcs,
           "-L", PKG, "-lvikalp_b200", "-Wl,-rpath,$ORIGIN", "-o", HOST_LIB]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"host build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return HOST_LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    a = ap.parse_args(argv)
    build(force=a.force, jobs=a.jobs, verbose=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
