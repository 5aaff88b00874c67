"""The dot product that allocates nothing (vk_vec_dot_device_noalloc).

It serves callers that cannot call cudaMalloc -- an allocator or memory pool
that owns all device memory, or a fixed memory budget. It must give exactly
what the allocating entry point (vk_vec_dot_device) gives: same kernels, same
order, so the results are compared bit for bit, on two calls in a row (the
second call reuses the fixed scratch the first one left behind). Inputs and
outputs are the caller's; the test allocates them with torch. This file is
named so pytest collects it last."""

import ctypes as C
import os
import subprocess
import sys
import textwrap

import pytest

import vikalp_b200 as vk

pytestmark = pytest.mark.gpu


def _call(fn, torch, x, y, out_slot):
    rc = fn(C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), x.numel(), C.c_void_p(out_slot.data_ptr()),
            C.c_void_p(torch.cuda.current_stream().cuda_stream))
    return rc


@pytest.mark.parametrize("n", [0, 1, 1000, 2049, 3_000_001, 8_388_608])
def test_noalloc_matches_allocating_dot(n):
    torch = pytest.importorskip("torch")
    L = vk.lib()
    g = torch.Generator(device="cuda").manual_seed(1234 + n)
    x = torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
    y = torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
    out = torch.full((3,), float("nan"), dtype=torch.float64, device="cuda")
    assert _call(L.vk_vec_dot_device, torch, x, y, out[0:1]) == vk.VK_OK, vk.last_error()
    assert _call(L.vk_vec_dot_device_noalloc, torch, x, y, out[1:2]) == vk.VK_OK, vk.last_error()
    assert _call(L.vk_vec_dot_device_noalloc, torch, x, y, out[2:3]) == vk.VK_OK, vk.last_error()
    torch.cuda.synchronize()
    a, b, c = (float(v) for v in out.cpu().tolist())
    assert b == a and c == a, (a, b, c)


def test_noalloc_second_call_with_different_inputs():
    # the shared scratch keeps the previous call's partials; a shorter call
    # must not see them
    torch = pytest.importorskip("torch")
    L = vk.lib()
    big = torch.ones(5_000_000, dtype=torch.float64, device="cuda")
    small = torch.full((10,), 2.0, dtype=torch.float64, device="cuda")
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    assert _call(L.vk_vec_dot_device_noalloc, torch, big, big, out[0:1]) == vk.VK_OK
    assert _call(L.vk_vec_dot_device_noalloc, torch, small, small, out[1:2]) == vk.VK_OK
    torch.cuda.synchronize()
    assert out.cpu().tolist() == [5_000_000.0, 40.0]


def test_noalloc_rejects_sizes_beyond_its_maximum():
    torch = pytest.importorskip("torch")
    L = vk.lib()
    x = torch.zeros(8_388_609, dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = _call(L.vk_vec_dot_device_noalloc, torch, x, x, out)
    assert rc == vk.VK_ERR_INVALID
    assert "exceeds its maximum of 8388608 elements" in vk.last_error()


_FRESH = textwrap.dedent("""
    import ctypes as C, sys
    import torch
    import vikalp_b200 as vk
    L = vk.lib()
    n = 3_000_001
    x = torch.randn(n, dtype=torch.float64, device="cuda")
    y = torch.randn(n, dtype=torch.float64, device="cuda")
    out = torch.zeros(8, dtype=torch.float64, device="cuda")
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    def call(k):
        return L.vk_vec_dot_device_noalloc(C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), n,
                                           C.c_void_p(out[k:k + 1].data_ptr()), s)
    # the first library call of this process: with lazy module loading the
    # driver loads the library's device code (and its fixed scratch) here
    assert call(0) == vk.VK_OK, vk.last_error()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for k in range(1, 8):
        assert call(k) == vk.VK_OK, vk.last_error()
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    v = out.cpu().tolist()
    ref = float(torch.dot(x, y))
    assert all(t == v[0] for t in v), v
    assert abs(v[0] - ref) <= 1e-9 * (float(torch.dot(x.abs(), y.abs())) + 1.0), (v[0], ref)
    print("free", free0, free1)
    sys.exit(0 if free0 == free1 else 3)
""")


def test_noalloc_first_call_in_a_fresh_process_allocates_nothing():
    # a fresh process whose first library call is the no-alloc entry point:
    # after that call (which may load the module), seven more calls leave the
    # device's free memory exactly where it was
    pytest.importorskip("torch")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, PYTHONPATH=root + os.pathsep + os.environ.get("PYTHONPATH", ""))
    r = subprocess.run([sys.executable, "-c", _FRESH], capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0, (r.returncode, r.stdout[-2000:], r.stderr[-2000:])
