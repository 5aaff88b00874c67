"""HiGHS (scipy.optimize.linprog, method="highs") objective of an LP -- TEST
INFRASTRUCTURE ONLY: an independent optimum to compare the device solutions
against (tests/ only)."""

import numpy as np
import scipy.sparse as sp
from scipy.optimize import linprog


def objective(inst, lower=None, upper=None) -> float:
    A = sp.csr_matrix((inst.values, inst.col_idx, inst.row_offsets), shape=(inst.m, inst.n))
    eq = np.isfinite(inst.row_lower) & (inst.row_lower == inst.row_upper)
    lo = inst.var_lower if lower is None else lower
    hi = inst.var_upper if upper is None else upper
    # rows with two finite sides split into <= and >= parts
    ub_rows, ub_rhs = [], []
    up = ~eq & np.isfinite(inst.row_upper)
    if up.any():
        ub_rows.append(A[up])
        ub_rhs.append(inst.row_upper[up])
    dn = ~eq & np.isfinite(inst.row_lower)
    if dn.any():
        ub_rows.append(-A[dn])
        ub_rhs.append(-inst.row_lower[dn])
    A_ub = sp.vstack(ub_rows).tocsr() if ub_rows else None
    b_ub = np.concatenate(ub_rhs) if ub_rhs else None
    r = linprog(inst.c, A_ub=A_ub, b_ub=b_ub, A_eq=A[eq] if eq.any() else None,
                b_eq=inst.row_lower[eq] if eq.any() else None, bounds=list(zip(lo, hi)), method="highs")
    assert r.status == 0, r.message
    return float(r.fun) + float(getattr(inst, "objective_offset", 0.0))
