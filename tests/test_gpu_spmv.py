"""GPU sparse products and CSR transpose through the C ABI, against the
reference's known answers (golden fixtures) and the CPU oracle.

SEQUENTIAL order must equal the reference bit for bit; FAST order (a
segmented warp scan) within 1e-13 of the row's absolute mass."""

import numpy as np
import pytest

import vikalp_b200 as vk
from conftest import same_bits
from vikalp_b200 import synthetic

pytestmark = pytest.mark.gpu


def _golden_spmv_names(golden):
    return sorted({k.split("__")[0] for k in golden.files if k.startswith("spmv_")})


@pytest.mark.parametrize("order", ["sequential", "fast"])
def test_spmv_golden(golden, oracle, order):
    for name in _golden_spmv_names(golden):
        g = lambda k: golden[f"{name}__{k}"]  # noqa: E731
        ro, n = g("ro"), int(g("n"))
        m = len(ro) - 1
        tr = bool(int(g("transpose")))
        got = vk.spmv(ro, g("ci"), g("v"), m, n, g("x"), g("y"), float(g("alpha")), float(g("beta")), tr, order)
        if order == "sequential":
            assert same_bits(got, g("out")), (name, got, g("out"))
        else:
            absv = np.abs(g("v"))
            ax = np.abs(g("x")) * abs(float(g("alpha")))
            mass = (oracle.spmv_t(ro, g("ci"), absv, n, ax) if tr else oracle.spmv(ro, g("ci"), absv, ax)) + \
                abs(float(g("beta"))) * np.abs(g("y"))
            assert np.all(np.abs(got - g("out")) <= 1e-13 * mass + 1e-300), name


def _ragged(seed, m=700, n=900, nnz=9000):
    inst = synthetic.lp_powerlaw(m, n, nnz, seed=seed)
    return inst.row_offsets, inst.col_idx, inst.values, inst.m, inst.n


def _with_long_rows(seed):
    # rows of 1, 40, 1500 (one tile of its own), 5000 (streamed from HBM) nonzeros
    rng = np.random.default_rng(seed)
    n = 6000
    lens = [1, 40, 0, 1500, 3, 5000, 7, 0, 33]
    ro = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    ci = np.concatenate([np.sort(rng.choice(n, size=k, replace=False)) for k in lens if k > 0]).astype(np.int64)
    v = rng.standard_normal(len(ci))
    return ro, ci, v, len(lens), n


@pytest.mark.parametrize("make", [_ragged, _with_long_rows])
@pytest.mark.parametrize("transpose", [False, True])
def test_spmv_matches_oracle(oracle, make, transpose):
    ro, ci, v, m, n = make(3)
    rng = np.random.default_rng(7)
    x = rng.standard_normal(m if transpose else n)
    y = rng.standard_normal(n if transpose else m)
    if transpose:
        want = oracle.spmv_t(ro, ci, v, n, x, 0.75, 1.5, y)
    else:
        want = oracle.spmv(ro, ci, v, x, 0.75, 1.5, y)
    got = vk.spmv(ro, ci, v, m, n, x, y, 0.75, 1.5, transpose, "sequential")
    assert same_bits(got, want)
    fast = vk.spmv(ro, ci, v, m, n, x, y, 0.75, 1.5, transpose, "fast")
    scale = np.abs(v).max() * np.abs(x).max() * (np.diff(ro).max() + 1) + np.abs(y).max()
    assert np.max(np.abs(fast - want)) <= 1e-13 * scale


def test_transpose_bit_exact(oracle):
    for make in (_ragged, _with_long_rows):
        ro, ci, v, m, n = make(5)
        tro, trow, tv, perm = vk.csr_transpose(ro, ci, v, m, n)
        wro, wrow, wv, wperm = oracle.transpose(ro, ci, v, n)
        assert np.array_equal(tro, wro)
        assert np.array_equal(trow, wrow)
        assert np.array_equal(perm, wperm)
        assert same_bits(tv, wv)


def test_transpose_edge_shapes(oracle):
    # empty matrix, all-empty rows, a single column
    for ro, ci, v, m, n in [
        (np.zeros(1, np.int64), np.zeros(0, np.int64), np.zeros(0), 0, 4),
        (np.zeros(6, np.int64), np.zeros(0, np.int64), np.zeros(0), 5, 3),
        (np.arange(8, dtype=np.int64), np.zeros(7, np.int64), np.arange(1.0, 8.0), 7, 1),
    ]:
        tro, trow, tv, perm = vk.csr_transpose(ro, ci, v, m, n)
        wro, wrow, wv, wperm = oracle.transpose(ro, ci, v, n)
        assert np.array_equal(tro, wro) and np.array_equal(trow, wrow) and np.array_equal(perm, wperm)


def test_spmv_invalid_pattern_raises():
    with pytest.raises(vk.VkError) as e:
        vk.spmv(np.array([0, 2]), np.array([1, 0]), np.ones(2), 1, 2, np.ones(2))
    assert e.value.code == vk.VK_ERR_INVALID


def test_spmat_device_apply(oracle):
    torch = pytest.importorskip("torch")
    ro, ci, v, m, n = _ragged(8, 2000, 3000, 40000)
    A = vk.SpMat(ro, ci, v, m, n, "fp64")
    x = torch.randn(n, dtype=torch.float64, device="cuda")
    y = torch.zeros(m, dtype=torch.float64, device="cuda")
    A.apply(x.data_ptr(), y.data_ptr(), False, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    want = oracle.spmv(ro, ci, v, x.cpu().numpy())
    assert np.max(np.abs(y.cpu().numpy() - want)) <= 1e-12 * np.abs(want).max()
    yt = torch.zeros(n, dtype=torch.float64, device="cuda")
    xt = torch.randn(m, dtype=torch.float64, device="cuda")
    A.apply(xt.data_ptr(), yt.data_ptr(), True, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    want_t = oracle.spmv_t(ro, ci, v, n, xt.cpu().numpy())
    assert np.max(np.abs(yt.cpu().numpy() - want_t)) <= 1e-12 * np.abs(want_t).max()
    B = vk.SpMat(ro, ci, v, m, n, "mixed")
    x32 = x.float()
    y32 = torch.zeros(m, dtype=torch.float32, device="cuda")
    B.apply(x32.data_ptr(), y32.data_ptr(), False, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    # fp32 storage and arithmetic: relative to the row's absolute mass
    mass = oracle.spmv(ro, ci, np.abs(v), np.abs(x.cpu().numpy()))
    assert np.all(np.abs(y32.cpu().numpy() - want) <= 1e-5 * (mass + 1e-30))
    assert A.bytes() == len(ci) * 12 + 4 * (m + 1) + 8 * n + 8 * m
    # every kernel variant the autotuner chooses from gives the same product
    assert 0 <= A.variant() < vk.FAST_VARIANTS and 0 <= A.variant(True) < vk.FAST_VARIANTS
    for var in range(vk.FAST_VARIANTS):
        A.set_variant(var)
        y.zero_()
        A.apply(x.data_ptr(), y.data_ptr(), False, torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        assert np.max(np.abs(y.cpu().numpy() - want)) <= 1e-12 * np.abs(want).max(), var
        A.set_variant(var, True)
        yt.zero_()
        A.apply(xt.data_ptr(), yt.data_ptr(), True, torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        assert np.max(np.abs(yt.cpu().numpy() - want_t)) <= 1e-12 * np.abs(want_t).max(), var
    with pytest.raises(vk.VkError):
        A.set_variant(vk.FAST_VARIANTS)


def _mostly_unit_rows(seed):
    # 5000 rows: most with one nonzero, some with 2-40, a few of 300, one of
    # 5000 and a few empty ones -- the mix a power-law column degree leaves
    # in A' (every hybrid-kernel path: lane-owned rows, sub-warp rows,
    # whole-warp rows)
    rng = np.random.default_rng(seed)
    n = 8000
    lens = np.ones(5000, dtype=np.int64)
    pick = rng.choice(5000, size=900, replace=False)
    lens[pick[:600]] = rng.integers(2, 41, size=600)
    lens[pick[600:640]] = 300
    lens[pick[640]] = 5000
    lens[pick[641:700]] = 0
    ro = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    ci = np.concatenate([np.sort(rng.choice(n, size=k, replace=False)) for k in lens if k > 0]).astype(np.int64)
    v = rng.standard_normal(len(ci))
    return ro, ci, v, len(lens), n


@pytest.mark.parametrize("make", [_with_long_rows, _mostly_unit_rows])
def test_every_variant_on_ragged_rows(oracle, make):
    torch = pytest.importorskip("torch")
    ro, ci, v, m, n = make(5)
    A = vk.SpMat(ro, ci, v, m, n, "fp64")
    rng = np.random.default_rng(11)
    xh, xth = rng.standard_normal(n), rng.standard_normal(m)
    x = torch.tensor(xh, device="cuda")
    xt = torch.tensor(xth, device="cuda")
    want = oracle.spmv(ro, ci, v, xh)
    want_t = oracle.spmv_t(ro, ci, v, n, xth)
    mass = oracle.spmv(ro, ci, np.abs(v), np.abs(xh)) + 1e-300
    mass_t = oracle.spmv_t(ro, ci, np.abs(v), n, np.abs(xth)) + 1e-300
    s = torch.cuda.current_stream().cuda_stream
    for var in range(vk.FAST_VARIANTS):
        A.set_variant(var)
        A.set_variant(var, True)
        y = torch.full((m,), np.nan, dtype=torch.float64, device="cuda")
        yt = torch.full((n,), np.nan, dtype=torch.float64, device="cuda")
        A.apply(x.data_ptr(), y.data_ptr(), False, s)
        A.apply(xt.data_ptr(), yt.data_ptr(), True, s)
        torch.cuda.synchronize()
        # every row written (empty rows as 0), each within 1e-13 of its absolute mass
        assert np.all(np.abs(y.cpu().numpy() - want) <= 1e-13 * mass), var
        assert np.all(np.abs(yt.cpu().numpy() - want_t) <= 1e-13 * mass_t), var
