"""Transfers large enough to go through the staged host <-> device copies
(pinned buffers filled by several host threads, int64 -> int32 narrowing of
the CSR on the host): the uploaded pattern must be the caller's, bit for bit,
and downloaded results complete. The first large transfer of a process goes
the plain way while the pinned buffers are allocated in the background, so
each case runs twice, a moment apart (both paths)."""

import time

import numpy as np
import pytest

import vikalp_b200 as vk

pytestmark = pytest.mark.gpu


def test_staged_pattern_upload_sequential_bits(oracle):
    # 2.4M rows, ragged (0..5 nonzeros), 6M nonzeros: row offsets (19 MB of
    # int64) and column indices (48 MB) both exceed the staging threshold and
    # end in a partial chunk; SEQUENTIAL order is the reference's, bit for bit
    rng = np.random.default_rng(11)
    m, n = 2_400_001, 3_000_017
    lens = rng.integers(0, 6, size=m)
    ro = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    nnz = int(ro[-1])
    # strictly increasing columns per row: start + 8k + U{0..7}, k < 6, below n
    row_of = np.repeat(np.arange(m), lens)
    k = np.arange(nnz) - ro[row_of]
    start = rng.integers(0, n - 48, size=m)
    ci = (start[row_of] + 8 * k + rng.integers(0, 8, size=nnz)).astype(np.int64)
    assert ci.max() < n and np.all(np.diff(ci)[np.diff(row_of) == 0] > 0)
    v = rng.standard_normal(nnz)
    x = rng.standard_normal(n)
    want = oracle.spmv(ro, ci, v, x)
    for _ in range(2):
        got = vk.spmv(ro, ci, v, m, n, x, order="sequential")
        assert got.shape == want.shape and np.array_equal(got.view(np.uint64), want.view(np.uint64))
        time.sleep(2.0)


def test_staged_result_download():
    # 2.2M boxed variables and one non-binding row: x* sits on the bound its
    # cost points to; x (17.6 MB) and the variable duals come back staged
    rng = np.random.default_rng(5)
    n = 2_200_003

    class Box:
        pass

    p = Box()
    p.m, p.n = 1, n
    p.row_offsets = np.array([0, 2], np.int64)
    p.col_idx = np.array([0, 1], np.int64)
    p.values = np.array([1.0, 1.0])
    p.c = np.where(rng.integers(0, 2, size=n) == 1, 1.0, -1.0)
    p.var_lower, p.var_upper = np.full(n, -1.0), np.full(n, 2.0)
    p.row_lower, p.row_upper = np.array([-100.0]), np.array([100.0])
    p.objective_offset = 0.0
    p.q_row_offsets = p.q_col_idx = p.q_values = None
    p.q_nnz = 0
    want = np.where(p.c > 0, -1.0, 2.0)
    for _ in range(2):
        r = vk.solve(p, algorithm="halpern", relative_tolerance=1e-9, iteration_limit=20000)
        assert r["status"] == "Optimal"
        assert r["x"].shape == (n,) and np.array_equal(r["x"], want)
        assert np.allclose(r["var_lower_dual"], np.where(p.c > 0, 1.0, 0.0), atol=1e-6)
        assert np.allclose(r["var_upper_dual"], np.where(p.c < 0, 1.0, 0.0), atol=1e-6)
        time.sleep(2.0)
