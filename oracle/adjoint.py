"""LP sensitivities -- TEST INFRASTRUCTURE ONLY (tests/ use it as the checker of
the library's adjoint; nothing else imports it).

The reference has no differentiation, so there is no reference code to follow:
these are the two independent pins the library's adjoint is checked against.

Problem (the reference's canonical form, Model.hpp:38-44):
    min c'x  s.t.  rl <= A x <= ru,  l <= x <= u,
with row multipliers y in the reference's sign convention (y > 0: upper row
bound active, c + A'y - lambda = 0; SolveResult.hpp:31-33).

1. kkt_gradient: the FP64 active-set KKT gradient. At an optimum with active
   rows R (equality rows and rows at a bound) and free columns F (strictly
   inside their bounds), x_F solves A_RF x_F = b_R - A_RN x_N and
   c_F + A_RF' y_R = 0. For L = g'x* + w_obj * (c'x*):
       w = argmin_min-norm |A_RF' w - g_F|       (the adjoint solve)
       dL/dc = w_obj * x
       dL/db_i = w_i - w_obj * y_i               (b_i: the active side of row i)
       dL/dA_ij = -w_i x_j + w_obj * y_i x_j     (every stored entry)
   (the c-sensitivity of x* is zero on a nondegenerate vertex; the objective
   terms are the envelope theorem).
2. fd_directional: central finite differences of L along random directions,
   re-solving the perturbed LPs with HiGHS (scipy), h = 1e-6.
"""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp
from scipy.optimize import linprog
from scipy.sparse.linalg import lsqr, splu


def _csr(inst):
    return sp.csr_matrix((inst.values, inst.col_idx, inst.row_offsets), shape=(inst.m, inst.n))


def highs_solve(inst, c=None, rl=None, ru=None, values=None):
    """HiGHS optimum (x, y) of the LP with optional replaced c / row bounds /
    A values; y in the reference's sign convention."""
    c = inst.c if c is None else c
    rl = inst.row_lower if rl is None else rl
    ru = inst.row_upper if ru is None else ru
    A = sp.csr_matrix((inst.values if values is None else values, inst.col_idx, inst.row_offsets),
                      shape=(inst.m, inst.n))
    eq = np.isfinite(rl) & (rl == ru)
    up = ~eq & np.isfinite(ru)
    dn = ~eq & np.isfinite(rl)
    blocks, rhs, which = [], [], []
    if up.any():
        blocks.append(A[up])
        rhs.append(ru[up])
        which.append(("up", np.flatnonzero(up)))
    if dn.any():
        blocks.append(-A[dn])
        rhs.append(-rl[dn])
        which.append(("dn", np.flatnonzero(dn)))
    r = linprog(c, A_ub=sp.vstack(blocks).tocsr() if blocks else None, b_ub=np.concatenate(rhs) if rhs else None,
                A_eq=A[eq] if eq.any() else None, b_eq=rl[eq] if eq.any() else None,
                bounds=list(zip(inst.var_lower, inst.var_upper)), method="highs",
                options={"primal_feasibility_tolerance": 1e-10, "dual_feasibility_tolerance": 1e-10})
    assert r.status == 0, r.message
    y = np.zeros(inst.m)
    if eq.any():
        y[eq] = -r.eqlin.marginals
    off = 0
    for kind, rows in which:
        mg = r.ineqlin.marginals[off:off + rows.size]
        off += rows.size
        # d obj / d ru = -y (y > 0 upper active); d obj / d rl = -y on a lower-active row
        y[rows] += -mg if kind == "up" else mg
    return r.x, y


def active_set(inst, x, y, tol=1e-8):
    """Active rows R and free columns F of an optimum (x, y)."""
    A = _csr(inst)
    ax = A @ x
    rl, ru = inst.row_lower, inst.row_upper
    scale_r = 1.0 + np.maximum(np.where(np.isfinite(rl), np.abs(rl), 0), np.where(np.isfinite(ru), np.abs(ru), 0))
    at_lo = np.isfinite(rl) & (np.abs(ax - rl) <= tol * scale_r)
    at_hi = np.isfinite(ru) & (np.abs(ax - ru) <= tol * scale_r)
    R = at_lo | at_hi
    lo, hi = inst.var_lower, inst.var_upper
    free = ~((np.isfinite(lo) & (x - lo <= tol * (1 + np.abs(lo)))) | (np.isfinite(hi) & (hi - x <= tol * (1 + np.abs(hi)))))
    return R, free


def kkt_gradient(inst, x, y, g, w_obj=0.0, tol=1e-8):
    """The FP64 active-set gradient (see the module docstring)."""
    A = _csr(inst)
    R, F = active_set(inst, x, y, tol)
    B = A[R][:, F]  # |R| x |F|
    gF = g[F]
    if B.shape[0] == B.shape[1] and B.shape[0] > 0:
        w_R = splu(B.T.tocsc()).solve(gF)
    elif B.shape[0] > 0:
        w_R = lsqr(B.T.tocsr(), gF, atol=1e-15, btol=1e-15, iter_lim=100000)[0]
    else:
        w_R = np.zeros(0)
    w = np.zeros(inst.m)
    w[R] = w_R
    rows = np.repeat(np.arange(inst.m), np.diff(inst.row_offsets))
    dA = (-w[rows] + w_obj * y[rows]) * x[inst.col_idx]
    return {"c": w_obj * x, "b": w - w_obj * y, "A": dA, "rows_active": int(R.sum()), "cols_free": int(F.sum())}


def fd_directional(inst, g, direction, h=1e-6, w_obj=0.0):
    """Central difference of L = g'x* + w_obj c'x* along `direction`, a dict
    with any of 'c' [n], 'b' [m] (moves the active side: ru, and rl too on
    equality rows), 'A' [nnz]."""
    def L(t):
        c = inst.c + t * direction["c"] if "c" in direction else inst.c
        rl, ru = inst.row_lower.copy(), inst.row_upper.copy()
        if "b" in direction:
            eq = np.isfinite(rl) & (rl == ru)
            ru = ru + t * direction["b"]
            rl = np.where(eq, ru, rl)
        vals = inst.values + t * direction["A"] if "A" in direction else None
        x, _ = highs_solve(inst, c=c, rl=rl, ru=ru, values=vals)
        return g @ x + w_obj * (c @ x)
    return (L(h) - L(-h)) / (2 * h)
