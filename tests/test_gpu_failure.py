"""Failure detection on the device without a fault.

Every wait inside the library's kernels is bounded: a pipelined sparse pass
that waits for a staged copy gives up after a poll limit, records a code in
the per-device error flag and returns; the host reads the flag after each
chunk and turns it into VK_ERR_CUDA. vk_diag_bounded_wait runs that path on
purpose -- its kernel waits on a barrier nothing arrives on, with a small poll
limit -- so the test can check the status the host gets and that the device
is still usable afterwards. Nothing faults and nothing waits without a bound."""

import numpy as np
import pytest

import vikalp_b200 as vk
from vikalp_b200 import synthetic

pytestmark = pytest.mark.gpu


def test_bounded_wait_runs_out_and_reports_cuda_error():
    L = vk.lib()
    assert L.vk_diag_bounded_wait(256) == vk.VK_ERR_CUDA
    assert "timed out" in vk.last_error()
    # the flag was cleared: an ordinary call on the same device succeeds
    inst = synthetic.lp_uniform(40, 90, 3, seed=5)
    x = np.random.default_rng(0).standard_normal(inst.n)
    y = vk.spmv(inst.row_offsets, inst.col_idx, inst.values, inst.m, inst.n, x)
    dense = inst.dense()
    assert np.allclose(y, dense @ x, rtol=1e-13, atol=1e-13)
    # and a whole solve runs to completion after it
    r = vk.solve(inst, algorithm="halpern", iteration_limit=20000, relative_tolerance=1e-6)
    assert r["status"] in ("Optimal", "IterationLimit"), r["message"]


def test_bounded_wait_twice_in_a_row():
    L = vk.lib()
    for _ in range(2):
        assert L.vk_diag_bounded_wait(64) == vk.VK_ERR_CUDA
    assert L.vk_diag_bounded_wait(0) == vk.VK_ERR_INVALID
