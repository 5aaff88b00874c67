"""Column order of the FAST passes.

With FAST products the solver may rename the columns of A in order of
decreasing nonzero count (VIKALP_B200_COLUMN_ORDER = auto | keep | count;
auto renames skewed patterns of 2^20 nonzeros or more). The iteration is the
same arithmetic on renamed vectors, so every result comes back in the
caller's column order and equals the unrenamed solve up to the rounding of
re-associated sums; overrides and warm starts are taken in the caller's order.
The SEQUENTIAL order never renames: it stays bit-identical to the reference's
CPU code (pdhg.cpp:87-151)."""

import numpy as np
import pytest

import vikalp_b200 as vk
from conftest import same_bits
from vikalp_b200 import synthetic

pytestmark = pytest.mark.gpu

KEYS = ("x", "y", "row_lower_dual", "row_upper_dual", "var_lower_dual", "var_upper_dual")


@pytest.fixture
def order(monkeypatch):
    return lambda v: monkeypatch.setenv("VIKALP_B200_COLUMN_ORDER", v)


@pytest.fixture(scope="module")
def skewed():
    # power-law column counts (coefficient of variation well above 1)
    return synthetic.lp_powerlaw(3000, 8000, 60000, seed=5)


def _both(order, inst, *args, **kw):
    order("keep")
    a = vk.solve(inst, *args, **kw)
    order("count")
    b = vk.solve(inst, *args, **kw)
    return a, b


def _agree(a, b, tol):
    for k in KEYS:
        scale = 1.0 + np.abs(a[k]).max()
        assert np.max(np.abs(a[k] - b[k])) <= tol * scale, k
    assert abs(a["objective"] - b["objective"]) <= tol * (1.0 + abs(a["objective"]))


def test_counts_are_skewed(skewed):
    cnt = np.bincount(skewed.col_idx, minlength=skewed.n)
    assert cnt.std() / cnt.mean() >= 1.0


@pytest.mark.parametrize("algorithm", ["reference", "halpern"])
def test_renamed_columns_match_the_callers_order(order, skewed, algorithm):
    lim = (dict(iteration_limit=64, primal_tolerance=0.0, dual_tolerance=0.0) if algorithm == "reference" else
           dict(iteration_limit=64, relative_tolerance=0.0))
    a, b = _both(order, skewed, algorithm=algorithm, **lim)
    assert a["iterations"] == b["iterations"] == 64
    _agree(a, b, 1e-8)


def test_overrides_and_warm_start_in_callers_order(order, skewed):
    rng = np.random.default_rng(11)
    lo = skewed.var_lower.copy()
    hi = skewed.var_upper.copy()
    pick = rng.choice(skewed.n, 200, replace=False)
    lo[pick] = rng.uniform(0.0, 4.0, pick.size)
    hi[pick] = lo[pick] + rng.uniform(0.5, 3.0, pick.size)
    warm = np.clip(skewed.x0, lo, hi)
    lim = dict(iteration_limit=64, primal_tolerance=0.0, dual_tolerance=0.0)
    a, b = _both(order, skewed, warm, lo, hi, algorithm="reference", **lim)
    _agree(a, b, 1e-8)
    # x leaves the device as (scaled x) * D: within rounding of the bounds
    slack = 1e-12 * (1.0 + np.maximum(np.abs(lo), np.abs(hi)))
    assert np.all(b["x"] >= lo - slack) and np.all(b["x"] <= hi + slack)
    # the override really reached the renamed column: the unbounded solve differs there
    order("count")
    free = vk.solve(skewed, warm, algorithm="reference", **lim)
    assert np.max(np.abs(free["x"][pick] - b["x"][pick])) > 0.0


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_renamed_solve_reaches_the_same_optimum(order, skewed, oracle, precision):
    kw = dict(algorithm="halpern", precision=precision, iteration_limit=400000, relative_tolerance=1e-6)
    a, b = _both(order, skewed, **kw)
    assert a["status"] == b["status"] == "Optimal"
    for r in (a, b):
        k = oracle.rel_kkt(skewed, r["x"], r["y"])
        assert max(k["rel_primal"], k["rel_dual"], k["rel_gap"]) <= 1.05e-6, k
    # a 1e-6 relative KKT point on this six-decade instance fixes the
    # objective to a few 1e-5 (infeasibility times the duals' size)
    assert abs(a["objective"] - b["objective"]) <= 1e-4 * (1.0 + abs(a["objective"]))


def test_sequential_order_keeps_the_callers_columns(order, skewed, oracle):
    order("count")
    lim = dict(iteration_limit=100, primal_tolerance=0.0, dual_tolerance=0.0)
    got = vk.solve(skewed, algorithm="reference", spmv_order="sequential", **lim)
    want = oracle.pdhg_solve(skewed, **lim)
    for k in ("x", "row_lower_dual", "row_upper_dual", "var_lower_dual", "var_upper_dual"):
        assert same_bits(got[k], want[k]), k


def test_bad_setting_is_rejected(order, skewed):
    order("sideways")
    with pytest.raises(vk.VkError, match="VIKALP_B200_COLUMN_ORDER"):
        vk.solve(skewed, algorithm="reference", iteration_limit=1)
