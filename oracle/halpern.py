"""NumPy restatement of the restarted reflected-Halpern PDHG -- TEST INFRASTRUCTURE ONLY.

This is the checker for the library's VK_ALGO_HALPERN engine (no reference
counterpart: the reference runs the fixed every-50-iterations scheme of
pdhg.cpp:133-145). It follows the same definitions, float64 throughout:

* scaling: 10 Ruiz infinity-norm passes then one Pock-Chambolle (alpha=1) pass
  (R, D), K = R A D, c^ = D c, variable bounds / D, row bounds * R;
* eta = 0.99 / sigma_max(K) (power iteration), omega_0 = |c^| / |b^|;
* the PDHG step with the reference's sign convention for y and the reflected
  Halpern update with lambda = (k+1)/(k+2);
* every `check_every` iterations: relative KKT of (x^, y^) in original units,
  stop at `tol`, restart rule on the fixed-point residual, primal weight
  update on restart (OMEGA_START, THETA, RESTART below: the library's rule).

Used by tests/ and the bench's CPU baseline only.
"""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp


def _csr(inst):
    return sp.csr_matrix((inst.values, inst.col_idx, inst.row_offsets), shape=(inst.m, inst.n))


def scaling(A: sp.csr_matrix, passes: int = 10):
    m, n = A.shape
    r = np.ones(m)
    d = np.ones(n)
    absA = abs(A)
    for p in range(passes + 1):
        K = sp.diags(r) @ absA @ sp.diags(d)
        if p < passes:
            rn = np.asarray(K.max(axis=1).todense()).ravel() if m else np.zeros(0)
            cn = np.asarray(K.max(axis=0).todense()).ravel()
        else:
            rn = np.asarray(K.sum(axis=1)).ravel()
            cn = np.asarray(K.sum(axis=0)).ravel()
        r = np.where(rn > 0, r / np.sqrt(np.where(rn > 0, rn, 1)), r)
        d = np.where(cn > 0, d / np.sqrt(np.where(cn > 0, cn, 1)), d)
    return r, d


def sigma_max(K: sp.csr_matrix, iters: int = 200) -> float:
    n = K.shape[1]
    i = np.arange(n, dtype=np.uint64)
    h = (i * np.uint64(2654435761) + np.uint64(12345)) & np.uint64(0xFFFFFFFF)
    h ^= h >> np.uint64(13)
    h = (h * np.uint64(2246822519)) & np.uint64(0xFFFFFFFF)
    h ^= h >> np.uint64(16)
    v = 0.5 + (h & np.uint64(0xFFFF)).astype(np.float64) / 65536.0
    v /= np.linalg.norm(v)
    prev = 0.0
    for it in range(iters):
        z = K.T @ (K @ v)
        nz = np.linalg.norm(z)
        est = np.sqrt(nz)
        v = z / nz if nz > 0 else z
        if it > 10 and abs(est - prev) <= 1e-6 * est:
            return est
        prev = est
    return prev


def _q(inst):
    """Q as a scipy CSR matrix, or None for an LP."""
    if getattr(inst, "q_col_idx", None) is None or inst.q_nnz == 0:
        return None
    return sp.csr_matrix((inst.q_values, inst.q_col_idx, inst.q_row_offsets), shape=(inst.n, inst.n))


def lambda_max(Q: sp.csr_matrix, iters: int = 200) -> float:
    """Largest eigenvalue of a PSD matrix by power iteration (same start vector
    and stopping rule as sigma_max)."""
    n = Q.shape[0]
    i = np.arange(n, dtype=np.uint64)
    h = (i * np.uint64(2654435761) + np.uint64(12345)) & np.uint64(0xFFFFFFFF)
    h ^= h >> np.uint64(13)
    h = (h * np.uint64(2246822519)) & np.uint64(0xFFFFFFFF)
    h ^= h >> np.uint64(16)
    v = 0.5 + (h & np.uint64(0xFFFF)).astype(np.float64) / 65536.0
    v /= np.linalg.norm(v)
    prev = 0.0
    for it in range(iters):
        z = Q @ v
        est = np.linalg.norm(z)
        v = z / est if est > 0 else z
        if it > 10 and abs(est - prev) <= 1e-6 * est:
            return est
        prev = est
    return prev


def step_params(knorm: float, lq: float, omega: float):
    """(eta, rho) for primal weight omega: tau = eta/omega, sigma = eta*omega.

    LP (lq == 0): eta = 0.99/|K|, rho = 1 (fully reflected). QP: the explicit
    gradient step on 0.5 x'Qx needs 1/tau - sigma |K|^2 >= L (L = lambda_max of
    the scaled Q); eta solves tau L + eta^2 |K|^2 = 0.99^2, and the reflection
    is cut to rho = 0.99 (1 - 1/(2 kappa)), kappa = (1/tau - sigma |K|^2) / L,
    which keeps (1+rho) T - rho I nonexpansive (Condat's relaxation bound)."""
    if lq <= 0:
        return (0.99 / knorm if knorm > 0 else 1.0), 1.0
    k2, b, c = knorm * knorm, lq / omega, 0.9801
    eta = 2.0 * c / (b + np.sqrt(b * b + 4.0 * k2 * c))
    tau = eta / omega
    kappa = (1.0 - eta * eta * k2) / (tau * lq)
    return eta, min(1.0, 0.99 * (1.0 - 1.0 / (2.0 * kappa)))


def rel_kkt(inst, x, y, lower=None, upper=None):
    """Relative KKT of (x, y) in original units (same definition as the C oracle)."""
    A = _csr(inst)
    Q = _q(inst)
    lo = inst.var_lower if lower is None else lower
    hi = inst.var_upper if upper is None else upper
    ax = A @ x
    rl, ru = inst.row_lower, inst.row_upper
    rp = np.linalg.norm(ax - np.clip(ax, rl, ru)) + np.linalg.norm(x - np.clip(x, lo, hi))
    b = np.maximum(np.where(np.isfinite(rl), np.abs(rl), 0), np.where(np.isfinite(ru), np.abs(ru), 0))
    qx = Q @ x if Q is not None else np.zeros_like(x)
    quad = float(x @ qx)
    lam = inst.c + qx + A.T @ y
    yl, yu = np.maximum(0, -y), np.maximum(0, y)
    vl, vu = np.maximum(0, lam), np.maximum(0, -lam)
    viol = np.sum(np.where((yl > 0) & ~np.isfinite(rl), yl, 0) ** 2) + np.sum(np.where((yu > 0) & ~np.isfinite(ru), yu, 0) ** 2)
    rd2 = np.sum(np.where((vl > 0) & ~np.isfinite(lo), vl, 0) ** 2) + np.sum(np.where((vu > 0) & ~np.isfinite(hi), vu, 0) ** 2)
    fin = lambda v, w: np.where((w > 0) & np.isfinite(v), np.where(np.isfinite(v), v, 0.0) * w, 0.0)  # noqa: E731
    off = float(getattr(inst, "objective_offset", 0.0))
    dobj = np.sum(fin(rl, yl)) - np.sum(fin(ru, yu)) + np.sum(fin(lo, vl)) - np.sum(fin(hi, vu)) - 0.5 * quad + off
    pobj = inst.c @ x + 0.5 * quad + off
    return dict(rel_primal=rp / (1 + np.linalg.norm(b)), rel_dual=np.sqrt(rd2 + viol) / (1 + np.linalg.norm(inst.c)),
                rel_gap=abs(pobj - dobj) / (1 + abs(pobj) + abs(dobj)), primal_objective=pobj, dual_objective=dobj)


# The library's default primal-weight / restart rule (PrimalWeightRule,
# vk_engine.cuh): omega starts at OMEGA_START x |c^| / |b^|, is smoothed with
# THETA at each restart, restart thresholds RESTART = (sufficient, necessary,
# artificial).
OMEGA_START = 1.0
THETA = 0.2
FREEZE = 0.0  # no primal-weight update once the relative KKT error is below this
RESTART = (0.2, 0.8, 0.2)


def solve(inst, tol=1e-6, iteration_limit=100000, check_every=64, rho=None, warm=None, lower=None, upper=None,
          trace=False, theta=None, omega0=None, omega_start=None, restart=None, freeze=None):
    """rho: reflection override (default: step_params' choice, 1 for an LP).
    theta / omega_start / restart: the rule (defaults: THETA, OMEGA_START,
    RESTART); omega0 replaces the starting primal weight outright."""
    theta = THETA if theta is None else theta
    freeze = FREEZE if freeze is None else freeze
    omega_start = OMEGA_START if omega_start is None else omega_start
    b_suff, b_nec, b_art = RESTART if restart is None else restart
    A = _csr(inst)
    Q = _q(inst)
    m, n = A.shape
    lo0 = inst.var_lower if lower is None else lower
    hi0 = inst.var_upper if upper is None else upper
    r, d = scaling(A)
    K = (sp.diags(r) @ A @ sp.diags(d)).tocsr()
    KT = K.T.tocsr()
    Qs = (sp.diags(d) @ Q @ sp.diags(d)).tocsr() if Q is not None else None
    c = inst.c * d
    with np.errstate(invalid="ignore", divide="ignore"):
        lo = np.where(np.isfinite(lo0), lo0 / d, lo0)
        hi = np.where(np.isfinite(hi0), hi0 / d, hi0)
        rl = np.where(np.isfinite(inst.row_lower), inst.row_lower * r, inst.row_lower)
        ru = np.where(np.isfinite(inst.row_upper), inst.row_upper * r, inst.row_upper)
    b_orig = np.maximum(np.where(np.isfinite(inst.row_lower), np.abs(inst.row_lower), 0),
                        np.where(np.isfinite(inst.row_upper), np.abs(inst.row_upper), 0))
    bnorm, cnorm = np.linalg.norm(b_orig), np.linalg.norm(inst.c)
    cs2, bs2 = np.sum(c * c), np.sum((b_orig * r) ** 2)
    omega = np.sqrt(cs2) / np.sqrt(bs2) if (cs2 > 1e-20 and bs2 > 1e-20) else 1.0
    omega *= omega_start
    if omega0 is not None:
        omega = omega0
    smax = sigma_max(K) if K.nnz else 0.0
    lq = lambda_max(Qs) if Qs is not None and Qs.nnz else 0.0
    eta, rho_k = step_params(smax, lq, omega)
    rho_k = rho_k if rho is None else rho
    tau, sigma = eta / omega, eta * omega
    x = np.clip(np.zeros(n) if warm is None else warm / d, lo, hi)
    y = np.zeros(m)
    x0, y0 = x.copy(), y.copy()
    k_base, total, restarts = 0, 0, 0
    r_restart, r_prev = -1.0, np.inf
    status, hist = "IterationLimit", []
    xh = yh = None
    while True:
        for it in range(check_every):
            lam = (k_base + it + 1.0) / (k_base + it + 2.0)
            g = c + KT @ y if Qs is None else c + Qs @ x + KT @ y
            xh = np.clip(x - tau * g, lo, hi)
            xb = 2 * xh - x
            xn = lam * ((1 + rho_k) * xh - rho_k * x) + (1 - lam) * x0
            v = y + sigma * (K @ xb)
            yh = v - np.clip(v, sigma * rl, sigma * ru)
            yn = lam * ((1 + rho_k) * yh - rho_k * y) + (1 - lam) * y0
            if it == check_every - 1:
                dx2, dx0 = np.sum((xh - x) ** 2), np.sum((xh - x0) ** 2)
                dy2, dy0 = np.sum((yh - y) ** 2), np.sum((yh - y0) ** 2)
            x, y = xn, yn
        total += check_every
        kk = rel_kkt(inst, xh * d, yh * r, lo0, hi0)
        kkt = max(kk["rel_primal"], kk["rel_dual"], kk["rel_gap"])
        if trace:
            hist.append((total, kkt, restarts, omega, kk["rel_primal"], kk["rel_dual"], kk["rel_gap"]))
        if kkt <= tol:
            status = "Optimal"
            break
        if total >= iteration_limit:
            break
        rr = np.sqrt(omega * dx2 + dy2 / omega)
        k = k_base + check_every
        restart = False
        if r_restart < 0:
            r_restart = rr
        else:
            restart = rr <= b_suff * r_restart or (rr <= b_nec * r_restart and rr > r_prev) or k >= b_art * total
        r_prev = rr
        if restart:
            mx, my = np.sqrt(dx0), np.sqrt(dy0)
            if mx > 1e-10 and my > 1e-10 and theta > 0 and kkt >= freeze:
                omega = np.exp(theta * np.log(my / mx) + (1 - theta) * np.log(omega))
            eta, rho_k = step_params(smax, lq, omega)
            rho_k = rho_k if rho is None else rho
            tau, sigma = eta / omega, eta * omega
            k_base = 0
            restarts += 1
            r_restart = rr
            x, x0, y, y0 = xh.copy(), xh.copy(), yh.copy(), yh.copy()
        else:
            k_base = k
    out = dict(status=status, iterations=total, restarts=restarts, x=xh * d, y=yh * r, kkt=kkt, omega=omega, eta=eta)
    out.update(kk)
    if trace:
        out["trace"] = hist
    return out
