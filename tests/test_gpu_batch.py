"""Independent LPs solved as one batch (vk_batch_solve) on the GPU.

* per-instance iterate agreement with the NumPy restatement of the Halpern
  scheme (oracle/halpern.py) after 128 iterations (two checks, one restart
  decision each), to 1e-8 relative: each instance of the batch must follow its
  own single-instance trajectory (own scaling, step size, primal weight);
* every instance solved to relative KKT <= 1e-6 as evaluated by the C oracle
  from the returned (x, y) (tolerance written here: 1.05e-6, sums reordered),
  with the objective within 1e-6 relative of HiGHS -- float64 and mixed;
* degenerate members (a 1x1 LP, an LP with an empty row and an empty column)
  and members that converge at very different times (tiles of finished
  instances are skipped, which must leave their answers untouched).
"""

import numpy as np
import pytest
import scipy.sparse as sp

import vikalp_b200 as vk
from oracle import halpern
from oracle.highs import objective as highs_objective
from vikalp_b200 import synthetic

pytestmark = pytest.mark.gpu

KKT_TOL = 1.05e-6


@pytest.fixture(scope="module")
def members():
    return [synthetic.lp_uniform(200, 500, 6, seed=11), synthetic.lp_uniform(600, 1500, 6, seed=77),
            synthetic.lp_uniform(40, 90, 4, seed=5), synthetic.lp_uniform(1200, 2400, 8, seed=13),
            synthetic.lp_uniform(300, 800, 5, seed=3)]


def _degenerate():
    one = synthetic.Instance(m=1, n=1, row_offsets=np.array([0, 1], np.int64), col_idx=np.array([0], np.int64),
                             values=np.array([2.0]), c=np.array([-1.0]), var_lower=np.array([0.0]),
                             var_upper=np.array([10.0]), row_lower=np.array([-np.inf]), row_upper=np.array([4.0]),
                             x0=np.array([1.0]), name="1x1")
    base = synthetic.lp_uniform(50, 120, 4, seed=21)
    # drop row 7 (empty row) and every entry of column 3 (empty column)
    ro, ci, v = base.row_offsets, base.col_idx, base.values
    keep = np.ones(base.nnz, bool)
    keep[ro[7]:ro[8]] = False
    keep &= ci != 3
    rows = np.repeat(np.arange(base.m), np.diff(ro))[keep]
    new_ro = np.zeros(base.m + 1, np.int64)
    np.add.at(new_ro, rows + 1, 1)
    new_ro = np.cumsum(new_ro)
    inst = synthetic.Instance(m=base.m, n=base.n, row_offsets=new_ro, col_idx=ci[keep].copy(), values=v[keep].copy(),
                              c=base.c.copy(), var_lower=base.var_lower.copy(), var_upper=base.var_upper.copy(),
                              row_lower=base.row_lower.copy(), row_upper=base.row_upper.copy(), x0=base.x0,
                              name="holes")
    ax = synthetic.csr_matvec(inst.row_offsets, inst.col_idx, inst.values, base.x0)
    inst.row_lower = np.where(np.isfinite(inst.row_lower), np.minimum(inst.row_lower, ax), inst.row_lower)
    inst.row_upper = np.maximum(inst.row_upper, ax)
    inst.row_lower[7], inst.row_upper[7] = -1.0, 1.0
    return [one, inst]


def test_batch_follows_each_single_trajectory(members):
    outs = vk.batch_solve(members, iteration_limit=128, relative_tolerance=0.0, check_every=64)
    for inst, got in zip(members, outs):
        want = halpern.solve(inst, tol=0.0, iteration_limit=128, check_every=64)
        assert got["iterations"] == want["iterations"] == 128
        assert got["restarts"] == want["restarts"]
        for k in ("x", "y"):
            scale = 1.0 + np.abs(want[k]).max()
            assert np.max(np.abs(got[k] - want[k])) <= 1e-8 * scale, (inst.name, k)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_solves_every_member(members, oracle, precision):
    outs = vk.batch_solve(members, precision=precision, iteration_limit=200000, relative_tolerance=1e-6)
    iters = []
    for inst, r in zip(members, outs):
        assert r["status"] == "Optimal", inst.name
        k = oracle.rel_kkt(inst, r["x"], r["y"])
        assert max(k["rel_primal"], k["rel_dual"], k["rel_gap"]) <= KKT_TOL, (inst.name, k)
        assert max(r["rel_primal"], r["rel_dual"], r["rel_gap"]) <= KKT_TOL
        ref = highs_objective(inst)
        assert abs(r["objective"] - ref) <= 1e-6 * (1 + abs(ref)), inst.name
        iters.append(r["iterations"])
    # members stop on their own schedules
    assert len(set(iters)) > 1


def test_batch_matches_single_solves(members):
    outs = vk.batch_solve(members, iteration_limit=200000, relative_tolerance=1e-6)
    for inst, r in zip(members, outs):
        s = vk.solve(inst, algorithm="halpern", iteration_limit=200000, relative_tolerance=1e-6)
        assert s["status"] == r["status"] == "Optimal"
        # same scheme, sums reordered: the stopping check may land one chunk apart
        assert abs(s["iterations"] - r["iterations"]) <= 64 * 4, inst.name
        assert abs(s["objective"] - r["objective"]) <= 2e-6 * (1 + abs(s["objective"]))


def test_batch_degenerate_members(oracle):
    insts = _degenerate() + [synthetic.lp_uniform(100, 250, 5, seed=9)]
    outs = vk.batch_solve(insts, iteration_limit=200000, relative_tolerance=1e-6)
    for inst, r in zip(insts, outs):
        assert r["status"] == "Optimal", inst.name
        k = oracle.rel_kkt(inst, r["x"], r["y"])
        assert max(k["rel_primal"], k["rel_dual"], k["rel_gap"]) <= KKT_TOL, (inst.name, k)
        assert abs(r["objective"] - highs_objective(inst)) <= 1e-6 * (1 + abs(r["objective"])), inst.name
    assert abs(outs[0]["x"][0] - 2.0) <= 1e-5


def test_batch_limits(members):
    outs = vk.batch_solve(members, iteration_limit=64, relative_tolerance=1e-12)
    assert all(r["status"] == "IterationLimit" and r["iterations"] == 64 for r in outs)


# ---- relaxations of one LP that differ in variable bounds (shared A) -------------


@pytest.fixture(scope="module")
def node_lp():
    inst = synthetic.lp_uniform(600, 1500, 6, seed=77)
    lo, hi = synthetic.bnb_nodes(inst, 8, seed=3)
    return inst, lo, hi


def test_shared_follows_each_single_trajectory(node_lp):
    inst, lo, hi = node_lp
    outs = vk.batch_solve_shared(inst, len(lo), lo, hi, iteration_limit=128, relative_tolerance=0.0, check_every=64)
    for b, got in enumerate(outs):
        want = halpern.solve(inst, tol=0.0, iteration_limit=128, check_every=64, lower=lo[b], upper=hi[b])
        assert got["iterations"] == want["iterations"] == 128
        assert got["restarts"] == want["restarts"]
        for k in ("x", "y"):
            scale = 1.0 + np.abs(want[k]).max()
            assert np.max(np.abs(got[k] - want[k])) <= 1e-8 * scale, (b, k)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_shared_solves_every_node(node_lp, oracle, precision):
    inst, lo, hi = node_lp
    outs = vk.batch_solve_shared(inst, len(lo), lo, hi, precision=precision, iteration_limit=200000,
                                 relative_tolerance=1e-6)
    for b, r in enumerate(outs):
        assert r["status"] == "Optimal", (b, r["message"])
        assert np.all(r["x"] >= lo[b] - 1e-9) and np.all(r["x"] <= hi[b] + 1e-9)
        k = oracle.rel_kkt(inst, r["x"], r["y"], lo[b], hi[b])
        assert max(k["rel_primal"], k["rel_dual"], k["rel_gap"]) <= KKT_TOL, (b, k)
        ref = highs_objective(inst, lo[b], hi[b])
        assert abs(r["objective"] - ref) <= 1e-6 * (1 + abs(ref)), b
        if precision == "mixed":
            assert r["fp32_iterations"] > 0


def test_shared_wide_batch_vector_lanes(oracle):
    # 130 nodes: 16-byte lane packs (4 float32 / 2 float64 instances per lane)
    # and a padded instance dimension (130 -> 256)
    inst = synthetic.lp_uniform(150, 400, 5, seed=19)
    lo, hi = synthetic.bnb_nodes(inst, 130, seed=4)
    outs = vk.batch_solve_shared(inst, 130, lo, hi, precision="mixed", iteration_limit=200000,
                                 relative_tolerance=1e-6)
    for b in list(range(0, 130, 9)) + [129]:
        r = outs[b]
        assert r["status"] == "Optimal", b
        k = oracle.rel_kkt(inst, r["x"], r["y"], lo[b], hi[b])
        assert max(k["rel_primal"], k["rel_dual"], k["rel_gap"]) <= KKT_TOL, (b, k)
        assert abs(r["objective"] - highs_objective(inst, lo[b], hi[b])) <= 1e-6 * (1 + abs(r["objective"])), b
    assert all(r["status"] == "Optimal" for r in outs)


def test_shared_invalid_member_and_warm_start(node_lp):
    inst, lo, hi = node_lp
    lo, hi = lo.copy(), hi.copy()
    lo[2, 5], hi[2, 5] = 3.0, 1.0
    outs = vk.batch_solve_shared(inst, len(lo), lo, hi, iteration_limit=200000, relative_tolerance=1e-6)
    assert outs[2]["status"] == "InvalidModel"
    assert outs[2]["message"] == "variable bound overrides contain an invalid interval"
    assert all(r["status"] == "Optimal" for b, r in enumerate(outs) if b != 2)
    # warm starts (primal, as RelaxationOracle passes them): each instance
    # follows the restatement's warm-started trajectory
    lo[2, 5], hi[2, 5] = inst.var_lower[5], inst.var_upper[5]
    warm = np.stack([r["x"] if b != 2 else np.zeros(inst.n) for b, r in enumerate(outs)])
    warm += np.random.default_rng(1).uniform(-0.5, 0.5, warm.shape)
    again = vk.batch_solve_shared(inst, len(lo), lo, hi, warm, iteration_limit=128, relative_tolerance=0.0)
    for b in range(len(lo)):
        want = halpern.solve(inst, tol=0.0, iteration_limit=128, lower=lo[b], upper=hi[b], warm=warm[b])
        assert again[b]["restarts"] == want["restarts"]
        for k in ("x", "y"):
            assert np.max(np.abs(again[b][k] - want[k])) <= 1e-8 * (1.0 + np.abs(want[k]).max()), (b, k)


# ---- duals and residuals of batch members -----------------------------------------


def _post_reference(inst, x, y, lo, hi, atol=1e-6):
    """The post-processing of pdhg.cpp:153-264 in numpy (split row duals, variable
    duals at bounds within active_tol, the three infinity-norm residuals)."""
    A = sp.csr_matrix((inst.values, inst.col_idx, inst.row_offsets), shape=(inst.m, inst.n))
    ax = A @ x
    rl, ru = inst.row_lower, inst.row_upper
    ld, ud = np.maximum(0, -y), np.maximum(0, y)
    s = inst.c + A.T @ y
    at_lo = np.isfinite(lo) & (x - lo <= atol)
    at_hi = np.isfinite(hi) & (hi - x <= atol)
    vld = np.where(at_lo, np.maximum(0, s), 0.0)
    vud = np.where(at_hi, np.maximum(0, -s), 0.0)
    with np.errstate(invalid="ignore"):
        pres = max(np.max(np.where(np.isfinite(rl), rl - ax, 0), initial=0.0),
                   np.max(np.where(np.isfinite(ru), ax - ru, 0), initial=0.0),
                   np.max(np.where(np.isfinite(lo), lo - x, 0), initial=0.0),
                   np.max(np.where(np.isfinite(hi), x - hi, 0), initial=0.0))
    stat = np.max(np.abs(x - np.clip(x - s, lo, hi)), initial=0.0)
    return dict(row_lower_dual=ld, row_upper_dual=ud, var_lower_dual=vld, var_upper_dual=vud,
                primal_residual=pres, stationarity_residual=stat)


def test_batch_members_duals_and_residuals(members, node_lp):
    # the options' primal tolerance (1e-7) gives active_tol = max(10 * 1e-7, 1e-8) = 1e-6
    outs = vk.batch_solve(members, duals=True, iteration_limit=200000, relative_tolerance=1e-6)
    inst, lo, hi = node_lp
    nodes = vk.batch_solve_shared(inst, len(lo), lo, hi, duals=True, iteration_limit=200000, relative_tolerance=1e-6)
    cases = [(m, r, m.var_lower, m.var_upper) for m, r in zip(members, outs)]
    cases += [(inst, r, lo[b], hi[b]) for b, r in enumerate(nodes)]
    for model, r, l, u in cases:
        want = _post_reference(model, r["x"], r["y"], l, u)
        for k in ("row_lower_dual", "row_upper_dual", "var_lower_dual", "var_upper_dual"):
            assert np.allclose(r[k], want[k], rtol=1e-12, atol=1e-12), k
        for k in ("primal_residual", "stationarity_residual"):
            assert abs(r[k] - want[k]) <= 1e-12 * (1 + abs(want[k])), (k, r[k], want[k])
        assert np.isfinite(r["complementarity_residual"])
    # without dual arrays the residuals stay NaN
    plain = vk.batch_solve(members[:2], iteration_limit=200000, relative_tolerance=1e-6)
    assert np.isnan(plain[0]["primal_residual"])


# ---- a node batch and independent LPs in flight together ---------------------------


def test_together_equals_the_two_batches(members, node_lp):
    inst, lo, hi = node_lp
    opts = dict(precision="mixed", iteration_limit=200000, relative_tolerance=1e-6)
    nodes, lps = vk.batch_solve_together(inst, len(lo), members, lo, hi, **opts)
    n_alone = vk.batch_solve_shared(inst, len(lo), lo, hi, **opts)
    l_alone = vk.batch_solve(members, **opts)
    for got, want in list(zip(nodes, n_alone)) + list(zip(lps, l_alone)):
        assert got["status"] == want["status"] == "Optimal"
        assert got["iterations"] == want["iterations"]
        assert np.array_equal(got["x"], want["x"]) and np.array_equal(got["y"], want["y"])
