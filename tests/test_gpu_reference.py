"""The reference scheme on the GPU (VK_ALGO_REFERENCE) against the reference's
own runs (golden fixtures) and the CPU oracle.

With VK_SPMV_SEQUENTIAL every iterate, dual, objective and residual must equal
the reference bit for bit (compared with ==, so -0.0 == +0.0); with the FAST
product order the iterates agree to 1e-9 relative."""

import numpy as np
import pytest

import vikalp_b200 as vk
from conftest import same_bits
from vikalp_b200 import synthetic

pytestmark = pytest.mark.gpu

CASES = ["lp_bounded", "lp_row", "lp_row_warm_override", "qp_scalar", "qp_scalar_override", "lp_it0", "lp_it1",
         "lp_it2", "lp_it7", "lp_it51", "lp_it52", "lp_it300", "lp_box_it200", "lp_warm_ovr_it120", "lp_tol_stop",
         "qp_it1", "qp_it60", "qp_it200"]


def run(case, order):
    ex = case.extra
    return vk.solve(case.model, warm=ex.get("warm"), lower=ex.get("lower"), upper=ex.get("upper"),
                    algorithm="reference", spmv_order=order, **case.opts)


@pytest.mark.parametrize("name", CASES)
def test_bit_exact_against_reference_runs(golden_cases, name):
    case = golden_cases[name]
    res = run(case, "sequential")
    out = case.out
    assert res["status"] == out["status"], res["message"]
    assert res["iterations"] == int(out["iterations"])
    for k in ("x", "row_lower_dual", "row_upper_dual", "var_lower_dual", "var_upper_dual"):
        assert same_bits(res[k], out[k]), k
    for k in ("objective", "primal_residual", "stationarity_residual", "complementarity_residual"):
        if case.model.q_nnz > 0 and k == "objective":
            assert abs(res[k] - out[k]) <= 1e-12 * (1 + abs(out[k]))
        else:
            assert same_bits(res[k], out[k]), (k, res[k], out[k])


@pytest.mark.parametrize("name", ["lp_it300", "lp_box_it200", "lp_warm_ovr_it120", "qp_it200"])
def test_fast_order_close(golden_cases, name):
    case = golden_cases[name]
    res = run(case, "fast")
    out = case.out
    scale = 1.0 + np.abs(out["x"]).max()
    assert np.max(np.abs(res["x"] - out["x"])) <= 1e-9 * scale


def test_larger_instance_against_oracle(oracle):
    # ragged power-law LP with rows long enough for the warp and long-row paths
    inst = synthetic.lp_powerlaw(3000, 8000, 120000, seed=31)
    for it in (5, 157):
        want = oracle.pdhg_solve(inst, iteration_limit=it, primal_tolerance=0.0, dual_tolerance=0.0)
        got = vk.solve(inst, algorithm="reference", spmv_order="sequential", iteration_limit=it,
                       primal_tolerance=0.0, dual_tolerance=0.0)
        assert got["iterations"] == want["iterations"]
        assert same_bits(got["x"], want["x"])
        assert same_bits(got["y"], want["y"])
        assert same_bits(got["objective"], want["objective"])


@pytest.mark.parametrize("seed", [31, 32])
def test_fast_order_against_oracle_through_policy_iterations(oracle, seed):
    # The FAST order extrapolates K xbar = 2 K x+ - K x and does the primal
    # step in the column pass except on the every-50th control step; 157 and
    # 331 iterations cross several step-rule decisions and graph boundaries.
    # Every iterate must stay within 1e-9 (relative to the largest |x|, |y|)
    # of the oracle's, with the same step-rule restarts.
    inst = synthetic.lp_powerlaw(3000, 8000, 120000, seed=seed)
    for it in (1, 2, 51, 52, 157, 331):
        want = oracle.pdhg_solve(inst, iteration_limit=it, primal_tolerance=0.0, dual_tolerance=0.0)
        got = vk.solve(inst, algorithm="reference", spmv_order="fast", iteration_limit=it,
                       primal_tolerance=0.0, dual_tolerance=0.0)
        assert got["iterations"] == want["iterations"] == it
        assert got["restarts"] == want["restarts"]
        sx = 1.0 + np.abs(want["x"]).max()
        sy = 1.0 + np.abs(want["y"]).max()
        assert np.max(np.abs(got["x"] - want["x"])) <= 1e-9 * sx, it
        assert np.max(np.abs(got["y"] - want["y"])) <= 1e-9 * sy, it


def test_fast_order_tolerance_stop_matches_reference(golden_cases):
    # the reference run that stops on its absolute metric (and is then
    # downgraded by the original-coordinate check): the FAST order stops on
    # the same iteration with the same status
    case = golden_cases["lp_tol_stop"]
    res = run(case, "fast")
    out = case.out
    assert res["status"] == out["status"]
    assert abs(res["iterations"] - int(out["iterations"])) <= 1
    assert abs(res["objective"] - out["objective"]) <= 1e-6 * (1 + abs(out["objective"]))


@pytest.mark.parametrize("order", ["fast", "sequential"])
def test_pass_profile(order):
    inst = synthetic.lp_powerlaw(20000, 50000, 400000, seed=5)
    with vk.Pdhg(inst, algorithm="reference", spmv_order=order) as h:
        prof = h.profile(60)
        r = h.solve(iteration_limit=300, primal_tolerance=0.0, dual_tolerance=0.0)
    assert [p["launches"] for p in prof] == [60, 60, 60]
    assert all(p["ms"] > 0 for p in prof)
    nnz = inst.nnz
    assert prof[0]["bytes"] >= 12 * nnz and prof[2]["bytes"] >= 12 * nnz
    # the profiled passes account for the graph-launched iteration within 2x
    per_iter = sum(p["ms"] for p in prof) * 1e-3
    assert 0.5 * per_iter <= r["iterate_seconds"] / 300 <= 2.0 * per_iter
    with vk.Pdhg(inst, algorithm="halpern") as h:
        with pytest.raises(vk.VkError) as e:
            h.profile(4)
        assert e.value.code == vk.VK_ERR_UNSUPPORTED


def test_reference_cuda_backend_runs_on_b200(oracle):
    # the reference's own CUDA backend (cuSPARSE; the bench's GPU-to-GPU
    # comparison) replays the reference iteration on this GPU with the same
    # iterates as its CPU backend, to rounding
    from oracle.oracle import Reference, ReferenceCuda
    try:
        cuda = ReferenceCuda()
    except (FileNotFoundError, OSError) as e:
        pytest.skip(f"reference CUDA build absent: {e}")
    inst = synthetic.lp_uniform(300, 800, 5, seed=3)
    step = 0.99 / max(1.0, oracle.operator_bound(inst.row_offsets, inst.col_idx, inst.values, inst.n))
    _, xc, yc = Reference().pdhg_replay(inst, step, 40)
    _, xg, yg = cuda.pdhg_replay_cuda(inst, step, 40)
    assert np.max(np.abs(xg - xc)) <= 1e-9 * (1 + np.abs(xc).max())
    assert np.max(np.abs(yg - yc)) <= 1e-9 * (1 + np.abs(yc).max())


def test_repeated_solves_on_one_handle(golden_cases):
    # one device model, several solves with different overrides (the
    # branch-and-bound pattern, RelaxationOracle.hpp:17-22)
    case = golden_cases["lp_warm_ovr_it120"]
    with vk.Pdhg(case.model, algorithm="reference", spmv_order="sequential", **case.opts) as h:
        a = h.solve(case.extra["warm"], case.extra["lower"], case.extra["upper"])
        b = h.solve()
        c = h.solve(case.extra["warm"], case.extra["lower"], case.extra["upper"])
    assert same_bits(a["x"], case.out["x"]) and same_bits(c["x"], a["x"])
    assert not same_bits(b["x"], a["x"])


def test_solve_time_errors(golden_cases):
    case = golden_cases["lp_it7"]
    with vk.Pdhg(case.model, algorithm="reference") as h:
        n = case.model.n
        bad = np.zeros(n)
        bad[3] = np.inf
        r = h.solve(warm=bad)
        assert r["status"] == "InvalidModel" and r["message"] == "warm start must be empty or finite and sized to the model"
        lo = case.model.var_lower.copy()
        lo[0] = 11.0
        r = h.solve(lower=lo)
        assert r["status"] == "InvalidModel" and r["message"] == "variable bound overrides contain an invalid interval"
        lo[0] = np.nan
        r = h.solve(lower=lo)
        assert r["message"] == "variable bound overrides must be empty or sized and non-NaN"


def test_time_limit(golden_cases):
    case = golden_cases["lp_it7"]
    r = vk.solve(case.model, algorithm="reference", iteration_limit=10**9, time_limit_seconds=0.2,
                 primal_tolerance=0.0, dual_tolerance=0.0)
    assert r["status"] == "TimeLimit"
    assert r["iterations"] > 0 and r["solve_seconds"] < 5.0
