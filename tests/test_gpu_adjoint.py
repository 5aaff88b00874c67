"""The LP adjoint (vk_lp_adjoint) on the GPU.

Pins (the reference has no differentiation):
* the CPU FP64 active-set KKT gradient (oracle/adjoint.py) at the same
  (x, y): the device LSQR must reproduce the sparse-LU / LSQR answer to 1e-8;
* end to end from the device's own solves (batched, float64, 1e-9 relative
  KKT) against the oracle gradient at HiGHS's optimum: <= 1e-4 relative;
* central finite differences (h = 1e-6, HiGHS re-solves) along random
  directions: <= 1e-4 relative;
* a thin torch.autograd.Function over the C ABI (this harness only): the
  gradients autograd returns equal the oracle's.
"""

import numpy as np
import pytest
import torch

import vikalp_b200 as vk
from oracle import adjoint as oadj
from vikalp_b200 import synthetic

pytestmark = pytest.mark.gpu

GRAD_TOL = 1e-4


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def lps():
    return [synthetic.lp_uniform(200, 400, 8, seed=31 + s) for s in range(6)]


@pytest.fixture(scope="module")
def highs(lps):
    return [oadj.highs_solve(inst) for inst in lps]


def test_lsqr_matches_oracle_at_the_same_point(lps, highs):
    rng = np.random.default_rng(5)
    gs = [rng.standard_normal(i.n) for i in lps]
    got = vk.lp_adjoint(lps, [h[0] for h in highs], [h[1] for h in highs], gs, active_tolerance=1e-8)
    for inst, (x, y), g, r in zip(lps, highs, gs, got):
        want = oadj.kkt_gradient(inst, x, y, g, tol=1e-8)
        assert r["status"] == "Optimal"
        assert r["rows_active"] == want["rows_active"] and r["cols_free"] == want["cols_free"]
        for k in ("b", "A"):
            assert rel(r[k], want[k]) <= 1e-8, (k, rel(r[k], want[k]))
        assert np.all(r["c"] == 0.0)


@pytest.mark.parametrize("w_obj", [0.0, 1.0])
def test_end_to_end_against_oracle_and_fd(lps, highs, w_obj):
    sols = vk.batch_solve(lps, iteration_limit=500000, relative_tolerance=1e-9)
    assert all(s["status"] == "Optimal" for s in sols)
    rng = np.random.default_rng(11)
    gs = [rng.standard_normal(i.n) for i in lps]
    got = vk.lp_adjoint(lps, [s["x"] for s in sols], [s["y"] for s in sols], gs, dL_dobj=w_obj)
    for b, (inst, (x, y), g, r) in enumerate(zip(lps, highs, gs, got)):
        want = oadj.kkt_gradient(inst, x, y, g, w_obj=w_obj)
        for k in ("b", "A", "c"):
            if np.linalg.norm(want[k]) > 0:
                assert rel(r[k], want[k]) <= GRAD_TOL, (b, k, rel(r[k], want[k]))
        if b < 2:  # finite differences (two HiGHS re-solves per direction)
            for k, size in (("b", inst.m), ("A", inst.nnz), ("c", inst.n)):
                d = rng.standard_normal(size)
                fd = oadj.fd_directional(inst, g, {k: d}, w_obj=w_obj)
                an = float(r[k] @ d)
                assert abs(fd - an) <= GRAD_TOL * max(1.0, abs(fd)), (b, k, fd, an)


class LPLayer(torch.autograd.Function):
    """x* = argmin c'x s.t. A x <= / = b, l <= x <= u, differentiable in
    (c, b, A values) through vk_lp_adjoint. Test harness only."""

    @staticmethod
    def forward(ctx, c, b, avals, inst):
        m = synthetic.Instance(**{**inst.__dict__})
        m.c = c.detach().double().numpy()
        eq = np.isfinite(inst.row_lower) & (inst.row_lower == inst.row_upper)
        m.row_upper = b.detach().double().numpy().copy()
        m.row_lower = np.where(eq, m.row_upper, inst.row_lower)
        m.values = avals.detach().double().numpy()
        s = vk.batch_solve([m], iteration_limit=500000, relative_tolerance=1e-9)[0]
        ctx.model, ctx.x, ctx.y = m, s["x"], s["y"]
        return torch.from_numpy(s["x"].copy())

    @staticmethod
    def backward(ctx, gx):
        r = vk.lp_adjoint([ctx.model], [ctx.x], [ctx.y], [gx.double().numpy()])[0]
        return torch.from_numpy(r["c"]), torch.from_numpy(r["b"]), torch.from_numpy(r["A"]), None


def test_autograd_function(lps, highs):
    inst = lps[0]
    c = torch.tensor(inst.c, requires_grad=True)
    b = torch.tensor(inst.row_upper, requires_grad=True)
    a = torch.tensor(inst.values, requires_grad=True)
    g = torch.from_numpy(np.random.default_rng(2).standard_normal(inst.n))
    x = LPLayer.apply(c, b, a, inst)
    (x * g).sum().backward()
    want = oadj.kkt_gradient(inst, *highs[0], g.numpy())
    assert rel(b.grad.numpy(), want["b"]) <= GRAD_TOL
    assert rel(a.grad.numpy(), want["A"]) <= GRAD_TOL
    assert torch.all(c.grad == 0)
