"""Seeded synthetic LP / QP instances for the PDHG hot path.

Every instance is in VIKALP's canonical minimisation form (``Model.hpp:38-44`` in
the reference):

    min c'x + 0.5 x'Qx   s.t.  row_lower <= A x <= row_upper,  var_lower <= x <= var_upper

with ``A`` in CSR (int64 offsets / indices, float64 values, strictly increasing
columns per row, as ``Model::validate`` requires, ``src/contracts/Model.cpp:13-54``).

The generators use numpy's PCG64 (``np.random.default_rng(seed)``). The shapes
follow the five workloads the path is measured on:

* ``lp_uniform``      -- fixed nnz per column at uniformly random distinct rows,
                          values N(0,1); a seeded feasible point x0 ~ U[lo,hi] fixes
                          the row bounds: even rows ``[r, r]``, odd rows
                          ``[-inf, r + U[0,1]]`` with ``r = A x0``; c ~ U[-1,1].
* ``lp_powerlaw``     -- column degrees Zipf(1.5) clamped at 2000 and thinned
                          binomially so the mean degree is ``target_nnz / n``
                          (min 1); values +-10^U[-3,3].
* ``qp_sparse``       -- ``lp_uniform``-style A plus Q = D + B'B with D ~ U[0.1,1]
                          diagonal and B a sparse (4 nnz/row, N(0,1/4)) matrix.
* ``bnb_nodes``       -- per-node bound overrides for branch-and-bound relaxations
                          that share one A.
"""

from __future__ import annotations

import dataclasses

import numpy as np


@dataclasses.dataclass
class Instance:
    """One LP/QP in CSR form (original, unscaled coordinates)."""

    m: int
    n: int
    row_offsets: np.ndarray  # int64 [m+1]
    col_idx: np.ndarray  # int64 [nnz]
    values: np.ndarray  # float64 [nnz]
    c: np.ndarray  # float64 [n]
    var_lower: np.ndarray  # float64 [n]
    var_upper: np.ndarray  # float64 [n]
    row_lower: np.ndarray  # float64 [m]
    row_upper: np.ndarray  # float64 [m]
    x0: np.ndarray  # the seeded feasible point the row bounds were built around
    q_row_offsets: np.ndarray | None = None  # int64 [n+1] (QP only, full symmetric CSR)
    q_col_idx: np.ndarray | None = None
    q_values: np.ndarray | None = None
    objective_offset: float = 0.0
    name: str = ""

    @property
    def nnz(self) -> int:
        return int(self.col_idx.shape[0])

    @property
    def q_nnz(self) -> int:
        return 0 if self.q_col_idx is None else int(self.q_col_idx.shape[0])

    def dense(self) -> np.ndarray:
        a = np.zeros((self.m, self.n))
        rows = np.repeat(np.arange(self.m), np.diff(self.row_offsets))
        a[rows, self.col_idx] = self.values
        return a


def _distinct_rows(rng: np.random.Generator, m: int, degrees: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Row index lists, one per column, ``degrees[j]`` distinct rows each.

    Draws with replacement, then redraws the (rare) duplicated (row, column)
    pairs until every column's rows are distinct.
    """
    n = degrees.shape[0]
    degrees = np.minimum(degrees, m)
    dense = degrees > max(8, m // 8)  # near-full columns: draw without replacement directly
    cols = np.repeat(np.arange(n, dtype=np.int64), np.where(dense, 0, degrees))
    rows = rng.integers(0, m, size=cols.shape[0], dtype=np.int64)
    for _ in range(256):
        key = cols * m + rows
        order = np.argsort(key, kind="stable")
        dup = np.zeros(key.shape[0], dtype=bool)
        sk = key[order]
        dup[order[1:]] = sk[1:] == sk[:-1]
        nd = int(dup.sum())
        if nd == 0:
            break
        rows[dup] = rng.integers(0, m, size=nd, dtype=np.int64)
    else:  # pragma: no cover - probability ~0 for the sizes used here
        raise RuntimeError("could not draw distinct rows")
    if dense.any():
        dj = np.flatnonzero(dense)
        extra_r = [rng.choice(m, size=int(degrees[j]), replace=False) for j in dj]
        rows = np.concatenate([rows, *extra_r]).astype(np.int64)
        cols = np.concatenate([cols, np.repeat(dj, degrees[dj])]).astype(np.int64)
    return rows, cols


def _to_csr(m: int, n: int, rows: np.ndarray, cols: np.ndarray, vals: np.ndarray):
    key = rows * n + cols
    order = np.argsort(key, kind="stable")
    r = rows[order]
    offsets = np.zeros(m + 1, dtype=np.int64)
    np.cumsum(np.bincount(r, minlength=m), out=offsets[1:])
    return offsets, cols[order].astype(np.int64), vals[order].astype(np.float64)


def csr_matvec(row_offsets, col_idx, values, x) -> np.ndarray:
    """Row-sequential CSR product (numpy, float64)."""
    m = row_offsets.shape[0] - 1
    rows = np.repeat(np.arange(m), np.diff(row_offsets))
    return np.bincount(rows, weights=values * x[col_idx], minlength=m)


def _row_bounds(rng, m, ax0):
    rl = ax0.copy()
    ru = ax0.copy()
    odd = np.arange(m) % 2 == 1
    rl[odd] = -np.inf
    ru[odd] = ax0[odd] + rng.uniform(0.0, 1.0, size=int(odd.sum()))
    return rl, ru


def lp_uniform(m: int, n: int, per_col: int = 8, seed: int = 12345, lo: float = 0.0,
               hi: float = 10.0, name: str = "") -> Instance:
    """``per_col`` distinct uniform rows per column, N(0,1) values, box [lo, hi]."""
    rng = np.random.default_rng(seed)
    rows, cols = _distinct_rows(rng, m, np.full(n, per_col, dtype=np.int64))
    vals = rng.standard_normal(rows.shape[0])
    offsets, cidx, v = _to_csr(m, n, rows, cols, vals)
    x0 = rng.uniform(lo, hi, size=n)
    ax0 = csr_matvec(offsets, cidx, v, x0)
    rl, ru = _row_bounds(rng, m, ax0)
    c = rng.uniform(-1.0, 1.0, size=n)
    return Instance(m, n, offsets, cidx, v, c, np.full(n, lo), np.full(n, hi), rl, ru, x0,
                    name=name or f"lp_uniform(m={m},n={n},k={per_col},seed={seed})")


def lp_powerlaw(m: int, n: int, target_nnz: int, seed: int = 12345, zipf_a: float = 1.5,
                cap: int = 2000, lo: float = 0.0, hi: float = 10.0, name: str = "") -> Instance:
    """Zipf column degrees (clamped at ``cap``) thinned to ``target_nnz`` on average.

    Values are sign * 10^U[-3,3] (six decades of magnitude).
    """
    rng = np.random.default_rng(seed)
    deg = np.minimum(rng.zipf(zipf_a, size=n), cap).astype(np.int64)
    p = min(1.0, target_nnz / float(deg.sum()))
    deg = np.maximum(rng.binomial(deg, p), 1).astype(np.int64)
    rows, cols = _distinct_rows(rng, m, deg)
    mag = 10.0 ** rng.uniform(-3.0, 3.0, size=rows.shape[0])
    sign = np.where(rng.integers(0, 2, size=rows.shape[0]) == 1, 1.0, -1.0)
    offsets, cidx, v = _to_csr(m, n, rows, cols, mag * sign)
    x0 = rng.uniform(lo, hi, size=n)
    ax0 = csr_matvec(offsets, cidx, v, x0)
    rl, ru = _row_bounds(rng, m, ax0)
    c = rng.uniform(-1.0, 1.0, size=n)
    return Instance(m, n, offsets, cidx, v, c, np.full(n, lo), np.full(n, hi), rl, ru, x0,
                    name=name or f"lp_powerlaw(m={m},n={n},nnz~{target_nnz},seed={seed})")


def qp_sparse(m: int, n: int, per_col: int = 6, b_rows: int | None = None, b_per_row: int = 4,
              seed: int = 2024, box: float = 5.0, name: str = "") -> Instance:
    """Convex QP: ``lp_uniform``-style A, Q = D + B'B (full symmetric CSR), x in [-box, box], c ~ N(0,1)."""
    rng = np.random.default_rng(seed)
    rows, cols = _distinct_rows(rng, m, np.full(n, per_col, dtype=np.int64))
    vals = rng.standard_normal(rows.shape[0])
    offsets, cidx, v = _to_csr(m, n, rows, cols, vals)
    x0 = rng.uniform(-box, box, size=n)
    ax0 = csr_matvec(offsets, cidx, v, x0)
    rl, ru = _row_bounds(rng, m, ax0)
    c = rng.standard_normal(n)
    nb = b_rows if b_rows is not None else max(1, n // 10)
    # B: nb x n, b_per_row distinct columns per row, N(0, 1/4) values.
    bc, br = _distinct_rows(rng, n, np.full(nb, b_per_row, dtype=np.int64))
    bv = rng.normal(0.0, 0.5, size=bc.shape[0])
    # Q = D + B'B assembled as COO, summed per (i, j).
    order = np.argsort(br, kind="stable")
    br, bc, bv = br[order], bc[order], bv[order]
    k = b_per_row
    bc2 = bc.reshape(nb, k)
    bv2 = bv.reshape(nb, k)
    qi = np.repeat(bc2, k, axis=1).ravel()
    qj = np.tile(bc2, (1, k)).ravel()
    qv = (np.repeat(bv2, k, axis=1) * np.tile(bv2, (1, k))).ravel()
    d = rng.uniform(0.1, 1.0, size=n)
    qi = np.concatenate([qi, np.arange(n)])
    qj = np.concatenate([qj, np.arange(n)])
    qv = np.concatenate([qv, d])
    key = qi * n + qj
    uk, inv = np.unique(key, return_inverse=True)
    sv = np.zeros(uk.shape[0])
    np.add.at(sv, inv, qv)
    ui = uk // n
    uj = uk % n
    q_off = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(ui, minlength=n), out=q_off[1:])
    return Instance(m, n, offsets, cidx, v, c, np.full(n, -box), np.full(n, box), rl, ru, x0,
                    q_row_offsets=q_off, q_col_idx=uj.astype(np.int64), q_values=sv,
                    name=name or f"qp_sparse(m={m},n={n},seed={seed})")


def bnb_nodes(inst: Instance, count: int, seed: int = 7, max_vars: int = 12,
              max_shift: float = 2.0) -> tuple[np.ndarray, np.ndarray]:
    """Bound overrides for ``count`` branch-and-bound nodes of ``inst``.

    Each node tightens 1..max_vars random variables: a "down" branch sets
    ``upper = floor(x0_j + d)``, an "up" branch sets ``lower = ceil(x0_j - d)`` with
    ``d ~ U[0, max_shift]``, both clipped into the original box. Returns
    ``(lower[count, n], upper[count, n])``.
    """
    rng = np.random.default_rng(seed)
    lo = np.tile(inst.var_lower, (count, 1))
    hi = np.tile(inst.var_upper, (count, 1))
    for b in range(count):
        k = int(rng.integers(1, max_vars + 1))
        js = rng.choice(inst.n, size=k, replace=False)
        d = rng.uniform(0.0, max_shift, size=k)
        down = rng.integers(0, 2, size=k) == 1
        for j, dj, dn in zip(js, d, down):
            if dn:
                hi[b, j] = min(inst.var_upper[j], max(inst.var_lower[j], np.floor(inst.x0[j] + dj)))
            else:
                lo[b, j] = max(inst.var_lower[j], min(inst.var_upper[j], np.ceil(inst.x0[j] - dj)))
    return lo, hi


# Named workloads: the sizes the path is measured and tested on.
def workload_small_lp(seed: int = 12345) -> Instance:
    """m=2,000, n=5,000, 8 nnz per column (40,000 nnz): the CPU-runnable LP."""
    return lp_uniform(2000, 5000, 8, seed=seed, name=f"lp m=2000 n=5000 nnz=40000 seed={seed}")


def workload_large_lp(seed: int = 12345) -> Instance:
    """m=1,000,000, n=2,000,000, ~20M nnz power-law LP."""
    return lp_powerlaw(1_000_000, 2_000_000, 20_000_000, seed=seed,
                       name=f"lp m=1e6 n=2e6 nnz~20M zipf1.5 seed={seed}")


def workload_independent_lps(count: int = 256, seed: int = 2024, m_min: int = 500, m_max: int = 20000,
                             per_col: int = 8) -> list[Instance]:
    """``count`` independent LPs, m log-uniform on [m_min, m_max], n = 2m,
    ``per_col`` nonzeros per column (lp_uniform each, seeds seed+b): the
    independent half of the batched workload (256 LPs: ~1.35M rows,
    ~2.7M columns, ~21.7M nonzeros in expectation)."""
    rng = np.random.default_rng(seed)
    ms = np.exp(rng.uniform(np.log(m_min), np.log(m_max), size=count)).astype(np.int64)
    return [lp_uniform(int(m), int(2 * m), per_col, seed=seed + b, name=f"lp m={m} n={2 * m} seed={seed + b}")
            for b, m in enumerate(ms)]


def workload_qp(seed: int = 2024) -> Instance:
    """The large convex QP: n=500,000, m=200,000, A with 6 nonzeros per column
    (3M), Q = D + B'B with B 50,000 x n, 4 per row, x in [-5, 5], c ~ N(0,1)."""
    return qp_sparse(200_000, 500_000, 6, b_rows=50_000, b_per_row=4, seed=seed,
                     name=f"qp m=2e5 n=5e5 A nnz=3M Q=D+B'B seed={seed}")
