"""The restarted reflected-Halpern engine (VK_ALGO_HALPERN) on the GPU.

* iterate agreement with the NumPy restatement (oracle/halpern.py) after a
  fixed number of iterations (two device-side checks, one restart decision),
  to 1e-8 relative -- the sparse sums are reassociated, nothing else differs;
* solutions: relative KKT <= 1e-6 as evaluated independently by the C oracle
  from the returned (x, y) (tolerance written in the test: 1.05e-6, the
  device and the oracle sum in different orders), and the objective within
  1e-6 relative of HiGHS (scipy) -- float64 and float32-mixed alike.
"""

import numpy as np
import pytest
import scipy.sparse as sp
from scipy.optimize import linprog

import vikalp_b200 as vk
from oracle import halpern
from vikalp_b200 import synthetic

pytestmark = pytest.mark.gpu

KKT_TOL = 1.05e-6


def highs_objective(inst, lower=None, upper=None):
    A = sp.csr_matrix((inst.values, inst.col_idx, inst.row_offsets), shape=(inst.m, inst.n))
    eq = np.isfinite(inst.row_lower) & (inst.row_lower == inst.row_upper)
    ub = ~eq
    lo = inst.var_lower if lower is None else lower
    hi = inst.var_upper if upper is None else upper
    r = linprog(inst.c, A_ub=A[ub], b_ub=inst.row_upper[ub], A_eq=A[eq], b_eq=inst.row_lower[eq],
                bounds=list(zip(lo, hi)), method="highs")
    assert r.status == 0
    return r.fun


@pytest.fixture(scope="module")
def lp_mid():
    return synthetic.lp_uniform(600, 1500, 6, seed=77)


def test_iterates_match_restatement(lp_mid):
    want = halpern.solve(lp_mid, tol=0.0, iteration_limit=128, check_every=64)
    got = vk.solve(lp_mid, algorithm="halpern", iteration_limit=128, relative_tolerance=0.0, check_every=64)
    assert got["iterations"] == want["iterations"] == 128
    assert got["restarts"] == want["restarts"]
    for k in ("x", "y"):
        scale = 1.0 + np.abs(want[k]).max()
        assert np.max(np.abs(got[k] - want[k])) <= 1e-8 * scale, k


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_solves_to_relative_kkt(lp_mid, oracle, precision):
    r = vk.solve(lp_mid, algorithm="halpern", precision=precision, iteration_limit=200000, relative_tolerance=1e-6)
    assert r["status"] == "Optimal", r["message"]
    k = oracle.rel_kkt(lp_mid, r["x"], r["y"])
    assert max(k["rel_primal"], k["rel_dual"], k["rel_gap"]) <= KKT_TOL, k
    # the device's own evaluation of the same quantity
    assert max(r["rel_primal"], r["rel_dual"], r["rel_gap"]) <= KKT_TOL
    ref = highs_objective(lp_mid)
    assert abs(r["objective"] - ref) <= 1e-6 * (1 + abs(ref))
    if precision == "mixed":
        assert r["fp32_iterations"] > 0


def test_small_workload_against_highs(oracle):
    inst = synthetic.workload_small_lp()
    r = vk.solve(inst, algorithm="halpern", iteration_limit=200000, relative_tolerance=1e-6)
    assert r["status"] == "Optimal"
    k = oracle.rel_kkt(inst, r["x"], r["y"])
    assert max(k["rel_primal"], k["rel_dual"], k["rel_gap"]) <= KKT_TOL
    # HiGHS optimum of this seeded instance (scipy 1.18 linprog(method="highs"))
    assert abs(r["objective"] - (-8206.12353127857)) <= 1e-6 * 8207


def test_overrides_and_warm_start(lp_mid, oracle):
    lo = lp_mid.var_lower.copy()
    hi = lp_mid.var_upper.copy()
    lo[:7] = 1.0
    hi[7:15] = 3.0
    with vk.Pdhg(lp_mid, algorithm="halpern", iteration_limit=200000, relative_tolerance=1e-6) as h:
        a = h.solve(lower=lo, upper=hi)
        assert a["status"] == "Optimal"
        assert np.all(a["x"] >= lo - 1e-9) and np.all(a["x"] <= hi + 1e-9)
        k = oracle.rel_kkt(lp_mid, a["x"], a["y"], lo, hi)
        assert max(k["rel_primal"], k["rel_dual"], k["rel_gap"]) <= KKT_TOL
        assert abs(a["objective"] - highs_objective(lp_mid, lo, hi)) <= 1e-6 * (1 + abs(a["objective"]))
        # a primal warm start (the duals start at zero again) reaches the same
        # optimum; it need not take fewer iterations
        b = h.solve(warm=a["x"], lower=lo, upper=hi)
        assert b["status"] == "Optimal"
        assert abs(b["objective"] - a["objective"]) <= 2e-6 * (1 + abs(a["objective"]))


def test_iteration_and_time_limits(lp_mid):
    r = vk.solve(lp_mid, algorithm="halpern", iteration_limit=64, relative_tolerance=1e-12)
    assert r["status"] == "IterationLimit" and r["iterations"] == 64
    r = vk.solve(lp_mid, algorithm="halpern", iteration_limit=10**9, relative_tolerance=0.0, time_limit_seconds=0.3)
    assert r["status"] == "TimeLimit" and r["solve_seconds"] < 5.0


@pytest.fixture(scope="module")
def qp_small():
    return synthetic.qp_sparse(300, 800, 5, b_rows=100, seed=1)


def test_qp_iterates_match_restatement(qp_small):
    # PDQP: Q pass + explicit gradient step, step sizes from |K| and
    # lambda_max(Q^), reflection cut below 1
    want = halpern.solve(qp_small, tol=0.0, iteration_limit=192, check_every=64)
    got = vk.solve(qp_small, algorithm="halpern", iteration_limit=192, relative_tolerance=0.0, check_every=64)
    assert got["iterations"] == want["iterations"] == 192
    assert got["restarts"] == want["restarts"]
    for k in ("x", "y"):
        scale = 1.0 + np.abs(want[k]).max()
        assert np.max(np.abs(got[k] - want[k])) <= 1e-8 * scale, k


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_qp_solves_to_relative_kkt(qp_small, oracle, precision):
    r = vk.solve(qp_small, algorithm="halpern", precision=precision, iteration_limit=400000, relative_tolerance=1e-6)
    assert r["status"] == "Optimal", r["message"]
    # the C oracle's KKT of the returned point: feasibility + zero gap certify
    # optimality of a convex QP
    k = oracle.rel_kkt(qp_small, r["x"], r["y"])
    assert max(k["rel_primal"], k["rel_dual"], k["rel_gap"]) <= KKT_TOL, k
    # objective of the restatement run to 1e-8 relative KKT (48.0767314906966)
    assert abs(r["objective"] - 48.0767314906966) <= 1e-5 * 49.0


def test_mixed_float32_answer_confirmed_in_float64(oracle):
    # the float32 phase reaches the tolerance by its own evaluation; the same
    # point, evaluated again in float64 (no float64 iteration), is accepted:
    # every iteration ran in float32 and the answer certifies at 1e-6
    inst = synthetic.workload_small_lp()
    r = vk.solve(inst, algorithm="halpern", precision="mixed", iteration_limit=200000, relative_tolerance=1e-6)
    assert r["status"] == "Optimal", r["message"]
    assert r["fp32_iterations"] == r["iterations"] > 0
    k = oracle.rel_kkt(inst, r["x"], r["y"])
    assert max(k["rel_primal"], k["rel_dual"], k["rel_gap"]) <= KKT_TOL, k
    assert max(r["rel_primal"], r["rel_dual"], r["rel_gap"]) <= 1e-6
    assert abs(r["objective"] - (-8206.12353127857)) <= 1e-6 * 8207
