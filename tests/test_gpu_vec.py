"""Device reductions of the ExecutionBackend contract (dot, norm_inf) against
numpy and the reference's known answers (test_backend.cpp:160-206)."""

import ctypes as C

import numpy as np
import pytest

import vikalp_b200 as vk

pytestmark = pytest.mark.gpu


def _dot(torch, x, y):
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = vk.lib().vk_vec_dot_device(C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), x.numel(),
                                    C.c_void_p(out.data_ptr()), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == vk.VK_OK, vk.last_error()
    torch.cuda.synchronize()
    return float(out.item())


def _ninf(torch, x):
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = vk.lib().vk_vec_norm_inf_device(C.c_void_p(x.data_ptr()), x.numel(), C.c_void_p(out.data_ptr()),
                                         C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == vk.VK_OK, vk.last_error()
    torch.cuda.synchronize()
    return float(out.item())


def test_known_answers():
    torch = pytest.importorskip("torch")
    t = lambda a: torch.tensor(a, dtype=torch.float64, device="cuda")  # noqa: E731
    assert _dot(torch, t([1.0, 2.0, 3.0]), t([4.0, 5.0, 6.0])) == 32.0
    assert _dot(torch, t([1.0, 0.0]), t([0.0, 1.0])) == 0.0
    assert _dot(torch, t([-1.0, -2.0]), t([3.0, 4.0])) == -11.0
    assert _ninf(torch, t([1.0, -5.0, 3.0])) == 5.0
    assert _ninf(torch, t([0.0, 0.0, 0.0])) == 0.0
    assert _ninf(torch, t([-7.5])) == 7.5
    # NaN entries are ignored, as std::max(result, |NaN|) keeps result
    assert _ninf(torch, t([1.0, float("nan"), -2.0])) == 2.0
    e = torch.zeros(1, dtype=torch.float64, device="cuda")
    assert _dot(torch, e[:0], e[:0]) == 0.0 and _ninf(torch, e[:0]) == 0.0


@pytest.mark.parametrize("n", [1, 255, 2049, 1_000_003, 9_000_000])
def test_against_numpy(n):
    torch = pytest.importorskip("torch")
    g = torch.Generator(device="cuda").manual_seed(n)
    x = torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
    y = torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
    xn, yn = x.cpu().numpy(), y.cpu().numpy()
    d = _dot(torch, x, y)
    assert abs(d - float(xn @ yn)) <= 1e-12 * float(np.abs(xn) @ np.abs(yn))
    assert _ninf(torch, x) == float(np.abs(xn).max())
    # deterministic: same bits on a second call
    assert _dot(torch, x, y) == d
