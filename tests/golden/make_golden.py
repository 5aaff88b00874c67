"""Generates tests/golden/*.npz from the reference itself.

Run from the repository root where the reference tree is present:

    make -C oracle REF=<reference tree> && python tests/golden/make_golden.py

It drives the reference's own CPU code (oracle/_ref/libvkref.so, compiled by
oracle/Makefile from the reference sources) on
  * the known-answer cases of the reference's tests/test_backend.cpp
    (SpMV N / T with alpha, beta, an empty row, 1x1, a zero vector),
  * the known-answer cases of tests/solver/continuous/test_pdhg.cpp
    (bounded LP, row-bounded LP, warm start + override, convex QP),
  * seeded small LPs and a QP run for fixed iteration counts with zero
    tolerance, so the full iterate history is pinned,
and stores inputs and outputs. The fixtures are small (a few hundred KB).
"""

from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.oracle import Reference  # noqa: E402
from vikalp_b200 import synthetic  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
INF = np.inf


def spmv_kats(ref: Reference) -> dict:
    """The SpMV known answers of test_backend.cpp:257-378, recomputed by the reference."""
    out = {}
    # A = [1 2 0; 0 3 4]
    ro, ci, v = np.array([0, 2, 4]), np.array([0, 1, 1, 2]), np.array([1.0, 2.0, 3.0, 4.0])
    cases = [
        ("n_ax", ro, ci, v, 3, [2.0, 1.0, 3.0], [0.0, 0.0], 1.0, 0.0, False),
        ("n_alphabeta", ro, ci, v, 3, [2.0, 1.0, 3.0], [4.0, 15.0], 2.0, 3.0, False),
        ("t_aty", ro, ci, v, 3, [2.0, 1.0], [0.0, 0.0, 0.0], 1.0, 0.0, True),
        ("t_alphabeta", ro, ci, v, 3, [2.0, 1.0], [2.0, 7.0, 4.0], 0.5, 2.0, True),
        ("one_n", np.array([0, 1]), np.array([0]), np.array([7.0]), 1, [3.0], [0.0], 1.0, 0.0, False),
        ("one_t", np.array([0, 1]), np.array([0]), np.array([7.0]), 1, [3.0], [0.0], 1.0, 0.0, True),
        ("empty_row", np.array([0, 1, 1, 2]), np.array([0, 1]), np.array([1.0, 5.0]), 2, [2.0, 3.0],
         [0.0, 0.0, 0.0], 1.0, 0.0, False),
        ("zero_x", ro, ci, v, 3, [0.0, 0.0, 0.0], [0.0, 0.0], 1.0, 0.0, False),
    ]
    for name, ro_, ci_, v_, n, x, y, a, b, t in cases:
        y_out = ref.multiply(ro_, ci_, v_, n, np.array(x), np.array(y), alpha=a, beta=b, transpose=t)
        out[f"spmv_{name}"] = dict(ro=ro_, ci=ci_, v=v_, n=n, x=np.array(x), y=np.array(y), alpha=a, beta=b,
                                   transpose=int(t), out=y_out)
    # a seeded rectangular matrix with ragged rows, both directions
    inst = synthetic.lp_uniform(60, 90, 3, seed=5)
    rng = np.random.default_rng(9)
    x = rng.standard_normal(inst.n)
    yv = rng.standard_normal(inst.m)
    for t, xx, yy in ((False, x, yv), (True, yv, x)):
        y_out = ref.multiply(inst.row_offsets, inst.col_idx, inst.values, inst.n, xx, yy, 1.25, -0.5, t)
        out[f"spmv_seeded_{int(t)}"] = dict(ro=inst.row_offsets, ci=inst.col_idx, v=inst.values, n=inst.n,
                                           x=xx, y=yy, alpha=1.25, beta=-0.5, transpose=int(t), out=y_out)
    return out


class Tiny:
    """A small hand-written model in synthetic.Instance form."""

    def __init__(self, c, lo, hi, A=None, rl=(), ru=(), Q=None):
        n = len(c)
        self.n = n
        self.c = np.array(c, float)
        self.var_lower = np.array(lo, float)
        self.var_upper = np.array(hi, float)
        if A is None:
            self.m = 0
            self.row_offsets = np.zeros(1, np.int64)
            self.col_idx = np.zeros(0, np.int64)
            self.values = np.zeros(0)
        else:
            self.m, self.row_offsets, self.col_idx, self.values = A
        self.row_lower = np.array(rl, float)
        self.row_upper = np.array(ru, float)
        self.objective_offset = 0.0
        if Q is None:
            self.q_row_offsets = self.q_col_idx = self.q_values = None
        else:
            self.q_row_offsets, self.q_col_idx, self.q_values = Q
        self.x0 = np.zeros(n)

    @property
    def nnz(self):
        return int(self.col_idx.shape[0])

    @property
    def q_nnz(self):
        return 0 if self.q_col_idx is None else int(len(self.q_col_idx))


def tiny_cases() -> dict:
    """test_pdhg.cpp:105-159 models."""
    return {
        "lp_bounded": (Tiny([-1.0], [0.0], [10.0]), dict(iteration_limit=5000, primal_tolerance=1e-5,
                                                         dual_tolerance=1e-5), {}),
        "lp_row": (Tiny([-1.0], [0.0], [20.0], A=(1, np.array([0, 1]), np.array([0]), np.array([1.0])),
                        rl=[-INF], ru=[3.0]),
                   dict(iteration_limit=5000, primal_tolerance=1e-5, dual_tolerance=1e-5), {}),
        "lp_row_warm_override": (Tiny([-1.0], [0.0], [20.0], A=(1, np.array([0, 1]), np.array([0]),
                                                                 np.array([1.0])), rl=[-INF], ru=[3.0]),
                                 dict(iteration_limit=5000, primal_tolerance=1e-5, dual_tolerance=1e-5),
                                 dict(warm=np.array([2.0]), upper=np.array([4.0]))),
        "qp_scalar": (Tiny([-10.0], [0.0], [10.0], Q=(np.array([0, 1]), np.array([0]), np.array([2.0]))),
                      dict(iteration_limit=1000, primal_tolerance=1e-6, dual_tolerance=1e-6), {}),
        "qp_scalar_override": (Tiny([-10.0], [0.0], [10.0], Q=(np.array([0, 1]), np.array([0]), np.array([2.0]))),
                               dict(iteration_limit=1000, primal_tolerance=1e-6, dual_tolerance=1e-6),
                               dict(warm=np.array([1.0]), upper=np.array([4.0]))),
    }


def seeded_cases() -> dict:
    lp = synthetic.lp_uniform(120, 300, 4, seed=1)
    lp_box = synthetic.lp_uniform(80, 200, 5, seed=2, lo=-3.0, hi=7.0)
    qp = synthetic.qp_sparse(60, 150, 3, b_rows=30, seed=3)
    rng = np.random.default_rng(4)
    warm = rng.uniform(0, 10, lp.n)
    lo = lp.var_lower.copy()
    hi = lp.var_upper.copy()
    lo[:5] = 2.0
    hi[5:10] = 4.0
    cases = {}
    for it in (0, 1, 2, 7, 51, 52, 300):
        cases[f"lp_it{it}"] = (lp, dict(iteration_limit=it, primal_tolerance=0.0, dual_tolerance=0.0), {})
    cases["lp_box_it200"] = (lp_box, dict(iteration_limit=200, primal_tolerance=0.0, dual_tolerance=0.0), {})
    cases["lp_warm_ovr_it120"] = (lp, dict(iteration_limit=120, primal_tolerance=0.0, dual_tolerance=0.0),
                                  dict(warm=warm, lower=lo, upper=hi))
    cases["lp_tol_stop"] = (lp, dict(iteration_limit=20000, primal_tolerance=2e-2, dual_tolerance=2e-2), {})
    for it in (1, 60, 200):
        cases[f"qp_it{it}"] = (qp, dict(iteration_limit=it, primal_tolerance=0.0, dual_tolerance=0.0), {})
    return cases


def model_arrays(inst) -> dict:
    d = dict(m=inst.m, n=inst.n, ro=inst.row_offsets, ci=inst.col_idx, v=inst.values, c=inst.c,
             vl=inst.var_lower, vu=inst.var_upper, rl=inst.row_lower, ru=inst.row_upper)
    if inst.q_nnz > 0:
        d.update(qro=inst.q_row_offsets, qci=inst.q_col_idx, qv=inst.q_values)
    return d


def main() -> int:
    ref = Reference()
    arrays = {}
    for name, case in spmv_kats(ref).items():
        for k, v in case.items():
            arrays[f"{name}__{k}"] = np.asarray(v)
    names = []
    for name, (inst, opts, extra) in {**tiny_cases(), **seeded_cases()}.items():
        qp = inst.q_nnz > 0
        res = ref.solve_continuous(inst, qp=qp, **extra, **opts)
        assert res["rc"] == 0, res["message"]
        for k, v in model_arrays(inst).items():
            arrays[f"pdhg_{name}__model_{k}"] = np.asarray(v)
        for k, v in opts.items():
            arrays[f"pdhg_{name}__opt_{k}"] = np.asarray(v)
        for k, v in extra.items():
            arrays[f"pdhg_{name}__extra_{k}"] = np.asarray(v)
        for k in ("x", "y", "row_lower_dual", "row_upper_dual", "var_lower_dual", "var_upper_dual", "iterations",
                  "objective", "primal_residual", "stationarity_residual", "complementarity_residual"):
            arrays[f"pdhg_{name}__out_{k}"] = np.asarray(res[k])
        arrays[f"pdhg_{name}__out_status"] = np.asarray(res["status"])
        names.append(name)
    arrays["pdhg_cases"] = np.asarray(names)
    path = os.path.join(OUT, "reference_golden.npz")
    np.savez_compressed(path, **arrays)
    print(f"wrote {path} ({os.path.getsize(path)} bytes, {len(names)} solver cases)")
    return 0


if __name__ == "__main__":
    sys.exit(main())
