"""The CPU oracle pinned against the reference (CPU only, no GPU).

* against the committed golden fixtures, which the reference itself produced
  (tests/golden/make_golden.py): the reference's SpMV known answers
  (test_backend.cpp:257-378) and PDHG / PDQP runs (test_pdhg.cpp:105-159 plus
  seeded histories), compared bit for bit;
* against the live reference build (oracle/_ref) on fresh seeded inputs, when
  that build is present.
"""

import os

import numpy as np
import pytest

from conftest import same_bits
from vikalp_b200 import synthetic

REF_SO = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "libvkref.so")


def test_spmv_kats_match_golden(golden, oracle):
    names = sorted({k.split("__")[0] for k in golden.files if k.startswith("spmv_")})
    assert len(names) >= 10
    for name in names:
        g = lambda k: golden[f"{name}__{k}"]  # noqa: E731
        if int(g("transpose")):
            got = oracle.spmv_t(g("ro"), g("ci"), g("v"), int(g("n")), g("x"), float(g("alpha")), float(g("beta")),
                                g("y"))
        else:
            got = oracle.spmv(g("ro"), g("ci"), g("v"), g("x"), float(g("alpha")), float(g("beta")), g("y"))
        assert same_bits(got, g("out")), name


def test_spmv_hand_values(golden):
    # the literal expectations written in test_backend.cpp
    assert list(golden["spmv_n_ax__out"]) == [4.0, 15.0]
    assert list(golden["spmv_n_alphabeta__out"]) == [20.0, 75.0]
    assert list(golden["spmv_t_aty__out"]) == [2.0, 7.0, 4.0]
    assert list(golden["spmv_t_alphabeta__out"]) == [5.0, 17.5, 10.0]
    assert list(golden["spmv_empty_row__out"]) == [2.0, 0.0, 15.0]
    assert list(golden["spmv_one_n__out"]) == [21.0]
    assert list(golden["spmv_zero_x__out"]) == [0.0, 0.0]


@pytest.mark.parametrize("name", ["lp_bounded", "lp_row", "lp_row_warm_override", "qp_scalar", "qp_scalar_override",
                                  "lp_it0", "lp_it1", "lp_it2", "lp_it7", "lp_it51", "lp_it52", "lp_it300",
                                  "lp_box_it200", "lp_warm_ovr_it120", "lp_tol_stop", "qp_it1", "qp_it60",
                                  "qp_it200"])
def test_pdhg_matches_golden(golden_cases, oracle, name):
    case = golden_cases[name]
    ex = case.extra
    res = oracle.pdhg_solve(case.model, warm=ex.get("warm"), lower=ex.get("lower"), upper=ex.get("upper"),
                            **case.opts)
    out = case.out
    assert res["status"] == out["status"]
    assert res["iterations"] == int(out["iterations"])
    for k in ("x", "y", "row_lower_dual", "row_upper_dual", "var_lower_dual", "var_upper_dual"):
        assert same_bits(res[k], out[k]), k
    for k in ("objective", "primal_residual", "stationarity_residual", "complementarity_residual"):
        assert same_bits(res[k], out[k]), k


def test_pdhg_kat_values(golden_cases):
    # the literal expectations of test_pdhg.cpp:113-159
    o = golden_cases["lp_bounded"].out
    assert o["status"] == "Optimal" and abs(o["x"][0] - 10.0) <= 1e-5 and abs(o["objective"] + 10.0) <= 1e-5
    assert abs(golden_cases["lp_row"].out["x"][0] - 3.0) <= 1e-4
    assert abs(golden_cases["lp_row_warm_override"].out["x"][0] - 3.0) <= 1e-4
    q = golden_cases["qp_scalar"].out
    assert q["status"] == "Optimal" and abs(q["x"][0] - 5.0) <= 1e-4 and abs(q["objective"] + 25.0) <= 1e-4
    assert abs(golden_cases["qp_scalar_override"].out["x"][0] - 4.0) <= 1e-4


def test_transpose_order_is_reference_scatter_order(oracle):
    # Summing each transposed row left to right reproduces the reference's
    # row-order scatter (cpu_ops.cpp:444-458) exactly.
    inst = synthetic.lp_powerlaw(300, 700, 6000, seed=11)
    tro, trow, tv, perm = oracle.transpose(inst.row_offsets, inst.col_idx, inst.values, inst.n)
    assert np.array_equal(np.diff(tro), np.bincount(inst.col_idx, minlength=inst.n))
    for j in range(inst.n):
        assert np.all(np.diff(trow[tro[j]:tro[j + 1]]) > 0)
    assert np.array_equal(tv, inst.values[perm])
    y = np.random.default_rng(0).standard_normal(inst.m)
    seq = np.zeros(inst.n)
    for j in range(inst.n):
        acc = 0.0
        for t in range(tro[j], tro[j + 1]):
            acc += tv[t] * y[trow[t]]
        seq[j] = acc
    assert same_bits(seq, oracle.spmv_t(inst.row_offsets, inst.col_idx, inst.values, inst.n, y))


def test_rel_kkt_of_an_exact_solution(oracle):
    # x* of the bounded LP min -x, 0<=x<=10 with no rows: lambda = c = -1 at the upper bound.
    class M:
        m, n = 0, 1
        row_offsets = np.zeros(1, np.int64)
        col_idx = np.zeros(0, np.int64)
        values = np.zeros(0)
        c = np.array([-1.0])
        var_lower, var_upper = np.array([0.0]), np.array([10.0])
        row_lower = row_upper = np.zeros(0)
        objective_offset = 0.0
        q_nnz = 0
    k = oracle.rel_kkt(M, np.array([10.0]), np.zeros(0))
    assert k["rel_primal"] == 0.0 and k["rel_dual"] == 0.0 and k["rel_gap"] == 0.0
    k = oracle.rel_kkt(M, np.array([5.0]), np.zeros(0))
    assert k["rel_gap"] > 0.1


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference build absent")
@pytest.mark.parametrize("seed", [21, 22])
def test_oracle_matches_live_reference(oracle, seed):
    from oracle.oracle import Reference
    ref = Reference()
    inst = synthetic.lp_powerlaw(150, 400, 3000, seed=seed)
    for it in (3, 101):
        a = oracle.pdhg_solve(inst, iteration_limit=it, primal_tolerance=0.0, dual_tolerance=0.0)
        b = ref.solve_continuous(inst, iteration_limit=it, primal_tolerance=0.0, dual_tolerance=0.0)
        assert a["status"] == b["status"] and a["iterations"] == b["iterations"]
        assert same_bits(a["x"], b["x"]) and same_bits(a["y"], b["y"])
        assert same_bits(a["objective"], b["objective"])
    q = synthetic.qp_sparse(40, 100, 3, b_rows=20, seed=seed)
    a = oracle.pdhg_solve(q, iteration_limit=77, primal_tolerance=0.0, dual_tolerance=0.0)
    b = ref.solve_continuous(q, qp=True, iteration_limit=77, primal_tolerance=0.0, dual_tolerance=0.0)
    assert same_bits(a["x"], b["x"]) and same_bits(a["y"], b["y"])


def test_adjoint_oracle_against_finite_differences():
    # the active-set KKT gradient against central differences of HiGHS re-solves
    from oracle import adjoint

    inst = synthetic.lp_uniform(120, 240, 6, seed=41)
    x, y = adjoint.highs_solve(inst)
    rng = np.random.default_rng(3)
    g = rng.standard_normal(inst.n)
    for w_obj in (0.0, 1.0):
        gr = adjoint.kkt_gradient(inst, x, y, g, w_obj=w_obj)
        assert gr["rows_active"] == gr["cols_free"]  # a nondegenerate vertex
        for key, size in (("b", inst.m), ("A", inst.nnz), ("c", inst.n)):
            d = rng.standard_normal(size)
            fd = adjoint.fd_directional(inst, g, {key: d}, w_obj=w_obj)
            assert abs(fd - gr[key] @ d) <= 1e-5 * max(1.0, abs(fd)), (w_obj, key)
