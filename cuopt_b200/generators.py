"""Seeded synthetic LPs with an optimum known by construction (the benchmark workloads).

Every generator returns an ``LP`` with CSR constraint matrix, bounds, and the constructed primal /
dual optimum (x_star, y_star) and reduced costs (s_star) that satisfy the KKT conditions exactly:
    A x* within [con_lo, con_up],   var_lo <= x* <= var_up,
    c = A^T y* + s*,   s*_j >= 0 where x*_j = var_lo_j,  s*_j <= 0 where x*_j = var_up_j, else 0,
    y*_i >= 0 only on active lower row bounds, y*_i <= 0 only on active upper row bounds.
So c.x* is the optimal objective.  Random numbers come from numpy's PCG64 seeded with
``config_id * 1000 + instance``.

Workloads (sizes are parameters so the tests can run them small):
  constructed_lp   the 2000 x 5000 and 1M x 2M LPs: equality rows, [0, 10] bounds, k non-zeros per column at
                   uniform rows, N(0,1) values; 30% of x* at 0, the rest U(0.5, 5).
  skewed_lp        the 500k-row skewed LP: Zipf(1.3) row lengths on [1, 5000], uniform columns, log-uniform
                   magnitudes in [1e-3, 1e3] with random signs, 50% 'E' / 50% 'L' rows
                   (a slack column each with explicit_slacks, as that workload is specified;
                   otherwise a ranged row), bounds [0, U(1,100)], 10% free columns.
  batch_lps        the 512-LP batch: constructed_lp instances with m log-uniform in [200, 20000], n = 2.5 m,
                   non-zeros per column uniform in 6..12.
"""
from __future__ import annotations

from dataclasses import dataclass

from typing import Optional

import numpy as np


@dataclass
class LP:
    m: int
    n: int
    row_off: np.ndarray  # int32 [m+1]
    col_idx: np.ndarray  # int32 [nnz]
    val: np.ndarray      # float64 [nnz]
    c: np.ndarray
    con_lo: np.ndarray
    con_up: np.ndarray
    var_lo: np.ndarray
    var_up: np.ndarray
    x_star: np.ndarray
    y_star: np.ndarray
    s_star: np.ndarray
    name: str = "lp"
    basic: Optional[np.ndarray] = None  # basic columns of a non-degenerate vertex (vertex_lp)

    @property
    def nnz(self) -> int:
        return int(self.row_off[-1])

    @property
    def optimal_objective(self) -> float:
        return float(np.dot(self.c, self.x_star))

    def matvec(self, x: np.ndarray) -> np.ndarray:
        """A @ x with numpy (row sums)."""
        rows = np.repeat(np.arange(self.m), np.diff(self.row_off))
        return np.bincount(rows, weights=self.val * x[self.col_idx], minlength=self.m)

    def rmatvec(self, y: np.ndarray) -> np.ndarray:
        """A^T @ y with numpy."""
        rows = np.repeat(np.arange(self.m), np.diff(self.row_off))
        return np.bincount(self.col_idx, weights=self.val * y[rows], minlength=self.n)


def _csr_from_columns(m: int, n: int, rows: np.ndarray, cols: np.ndarray, vals: np.ndarray):
    """CSR (rows sorted, columns ascending inside a row) from coordinate lists."""
    order = np.lexsort((cols, rows))
    rows, cols, vals = rows[order], cols[order], vals[order]
    counts = np.bincount(rows, minlength=m)
    row_off = np.zeros(m + 1, dtype=np.int64)
    np.cumsum(counts, out=row_off[1:])
    return row_off.astype(np.int32), cols.astype(np.int32), vals.astype(np.float64)


def _distinct_rows_per_column(rng: np.random.Generator, m: int, n: int, k: int) -> np.ndarray:
    """[n, k] row indices, distinct inside each column, uniform over [0, m)."""
    if k > m:
        raise ValueError("more non-zeros per column than rows")
    r = rng.integers(0, m, size=(n, k), dtype=np.int64)
    while True:
        s = np.sort(r, axis=1)
        bad = np.any(s[:, 1:] == s[:, :-1], axis=1)
        if not bad.any():
            return r
        r[bad] = rng.integers(0, m, size=(int(bad.sum()), k), dtype=np.int64)


def constructed_lp(m: int, n: int, nnz_per_col: int = 8, seed: int = 0, upper: float = 10.0,
                   name: str = "constructed") -> LP:
    """min c.x s.t. A x = b, 0 <= x <= upper, with a constructed (degenerate) optimum."""
    rng = np.random.default_rng(seed)
    rows = _distinct_rows_per_column(rng, m, n, nnz_per_col)
    vals = rng.standard_normal((n, nnz_per_col))
    cols = np.repeat(np.arange(n, dtype=np.int64), nnz_per_col)
    row_off, col_idx, val = _csr_from_columns(m, n, rows.ravel(), cols, vals.ravel())
    x = rng.uniform(0.5, 5.0, size=n)
    zero = rng.random(n) < 0.3
    x[zero] = 0.0
    y = rng.standard_normal(m)
    s = np.where(zero, rng.uniform(0.1, 1.0, size=n), 0.0)
    lp = LP(m, n, row_off, col_idx, val, np.zeros(n), np.zeros(m), np.zeros(m),
            np.zeros(n), np.full(n, float(upper)), x, y, s, name)
    b = lp.matvec(x)
    lp.con_lo = b.copy()
    lp.con_up = b.copy()
    lp.c = lp.rmatvec(y) + s
    return lp


def vertex_lp(m: int, n: int, nnz_per_col: int = 8, seed: int = 0, upper: float = 10.0,
              name: str = "vertex") -> LP:
    """The constructed_lp recipe with a unique, non-degenerate optimal vertex (the adjoint batch).

    m basic variables lie strictly inside [0, upper]; basic column basic[i] holds row i with a
    value of magnitude in [1, 2], so the basis matrix is non-singular.  Every other variable sits
    on a bound (80 % at 0, 20 % at `upper`) with a reduced cost of the matching sign and magnitude
    in [0.1, 1], so the optimum is unique and its derivatives with respect to c, b and A exist.
    """
    rng = np.random.default_rng(seed)
    rows = _distinct_rows_per_column(rng, m, n, nnz_per_col)
    vals = rng.standard_normal((n, nnz_per_col))
    basic = rng.permutation(n)[:m]
    diag = np.arange(m)
    pos = np.argmax(rows[basic] == diag[:, None], axis=1)
    has = (rows[basic] == diag[:, None]).any(axis=1)
    pos[~has] = 0
    rows[basic[~has], 0] = diag[~has]
    vals[basic, pos] = np.where(rng.random(m) < 0.5, -1.0, 1.0) * rng.uniform(1.0, 2.0, size=m)
    cols = np.repeat(np.arange(n, dtype=np.int64), nnz_per_col)
    row_off, col_idx, val = _csr_from_columns(m, n, rows.ravel(), cols, vals.ravel())
    is_basic = np.zeros(n, dtype=bool)
    is_basic[basic] = True
    at_up = (~is_basic) & (rng.random(n) < 0.2)
    x = np.zeros(n)
    x[basic] = rng.uniform(0.5, upper - 0.5, size=m)
    x[at_up] = upper
    s = np.zeros(n)
    at_lo = (~is_basic) & (~at_up)
    s[at_lo] = rng.uniform(0.1, 1.0, size=int(at_lo.sum()))
    s[at_up] = -rng.uniform(0.1, 1.0, size=int(at_up.sum()))
    y = rng.standard_normal(m)
    lp = LP(m, n, row_off, col_idx, val, np.zeros(n), np.zeros(m), np.zeros(m),
            np.zeros(n), np.full(n, float(upper)), x, y, s, name)
    b = lp.matvec(x)
    lp.con_lo = b.copy()
    lp.con_up = b.copy()
    lp.c = lp.rmatvec(y) + s
    lp.basic = np.sort(basic)
    return lp


def _truncated_zipf(rng: np.random.Generator, a: float, cap: int, size: int) -> np.ndarray:
    """Samples of P(k) proportional to k^-a on k = 1..cap (mean 150.8 for a = 1.3, cap = 5000)."""
    k = np.arange(1, cap + 1, dtype=np.float64)
    cdf = np.cumsum(k ** -a)
    cdf /= cdf[-1]
    return np.searchsorted(cdf, rng.random(size), side="right").astype(np.int64) + 1


def skewed_lp(m: int, n: int, seed: int = 2000, zipf_a: float = 1.3, cap: int = 5000,
              name: str = "skewed", explicit_slacks: bool = False) -> LP:
    """Skewed-sparsity LP (row lengths Zipf(a) on [1, cap], mixed senses, free columns).

    With explicit_slacks, every '<=' row gets a slack column (coefficient +1, bounds [0, inf),
    cost 0) and becomes an equality, as the 500k-row skewed workload is specified (n grows by the number
    of such rows); the constructed optimum carries over (slack = the row's slack, reduced cost
    -y_i)."""
    rng = np.random.default_rng(seed)
    lens = np.minimum(_truncated_zipf(rng, zipf_a, cap, m), n)
    rows = np.repeat(np.arange(m, dtype=np.int64), lens)
    key = rows * n + rng.integers(0, n, size=int(lens.sum()), dtype=np.int64)
    del rows
    key.sort()
    keep = np.ones(key.size, dtype=bool)
    keep[1:] = key[1:] != key[:-1]  # drop duplicate (row, column) pairs
    key = key[keep]
    rows, cols = key // n, key % n
    del key
    mag = 10.0 ** rng.uniform(-3.0, 3.0, size=rows.size)
    sign = np.where(rng.random(rows.size) < 0.5, -1.0, 1.0)
    counts = np.bincount(rows, minlength=m)
    row_off = np.zeros(m + 1, dtype=np.int64)
    np.cumsum(counts, out=row_off[1:])
    row_off, col_idx, val = row_off.astype(np.int32), cols.astype(np.int32), mag * sign
    del rows, cols
    ub = rng.uniform(1.0, 100.0, size=n)
    lb = np.zeros(n)
    free = rng.random(n) < 0.1
    lb[free], ub[free] = -np.inf, np.inf
    # x*: bounded columns 30% at lower, 10% at upper, rest interior; free columns N(0, 1).
    u = rng.random(n)
    at_lo = (~free) & (u < 0.3)
    at_up = (~free) & (u >= 0.3) & (u < 0.4)
    x = np.where(free, rng.standard_normal(n), rng.uniform(0.1, 0.9, size=n) * np.where(free, 1.0, ub))
    x[at_lo] = 0.0
    x[at_up] = ub[at_up]
    s = np.zeros(n)
    s[at_lo] = rng.uniform(0.1, 1.0, size=int(at_lo.sum()))
    s[at_up] = -rng.uniform(0.1, 1.0, size=int(at_up.sum()))
    lp = LP(m, n, row_off, col_idx, val, np.zeros(n), np.zeros(m), np.zeros(m), lb, ub, x,
            np.zeros(m), s, name)
    ax = lp.matvec(x)
    eq = rng.random(m) < 0.5
    active = rng.random(m) < 0.5
    y = np.where(eq, rng.standard_normal(m), 0.0)
    le_active = (~eq) & active
    y[le_active] = -rng.uniform(0.1, 1.0, size=int(le_active.sum()))
    slack = np.where((~eq) & (~active), rng.uniform(0.1, 1.0, size=m) * (1.0 + np.abs(ax)), 0.0)
    lp.con_lo = np.where(eq, ax, -np.inf)
    lp.con_up = ax + slack
    lp.y_star = y
    lp.c = lp.rmatvec(y) + s
    if explicit_slacks:
        le = ~eq
        k = int(le.sum())
        ends = lp.row_off[1:].astype(np.int64)[le]
        col_idx = np.insert(lp.col_idx, ends, (n + np.arange(k)).astype(np.int32))
        val = np.insert(lp.val, ends, 1.0)
        row_off = (lp.row_off.astype(np.int64) +
                   np.concatenate([[0], np.cumsum(le)])).astype(np.int32)
        b = lp.con_up
        lp = LP(m, n + k, row_off, col_idx.astype(np.int32), val,
                np.concatenate([lp.c, np.zeros(k)]), b.copy(), b.copy(),
                np.concatenate([lb, np.zeros(k)]), np.concatenate([ub, np.full(k, np.inf)]),
                np.concatenate([x, slack[le]]), y, np.concatenate([s, -y[le]]), name)
    return lp


def _batch_shapes(count, seed, m_lo, m_hi):
    rng = np.random.default_rng(seed)
    ms = np.exp(rng.uniform(np.log(m_lo), np.log(m_hi), size=count)).astype(int)
    ks = rng.integers(6, 13, size=count)
    return ms, ks


def batch_lps(count: int = 512, seed: int = 3000, m_lo: int = 200, m_hi: int = 20000):
    """The batch workload: `count` constructed_lp instances of uneven sizes."""
    ms, ks = _batch_shapes(count, seed, m_lo, m_hi)
    return [constructed_lp(int(m), int(2.5 * m), int(k), seed=seed + 1 + i, name=f"batch{i}")
            for i, (m, k) in enumerate(zip(ms, ks))]


def batch_instance(i: int, count: int = 512, seed: int = 3000, m_lo: int = 200,
                   m_hi: int = 20000):
    """Instance i of batch_lps(count, seed, ...) alone."""
    ms, ks = _batch_shapes(count, seed, m_lo, m_hi)
    return constructed_lp(int(ms[i]), int(2.5 * ms[i]), int(ks[i]), seed=seed + 1 + i,
                          name=f"batch{i}")


def kkt_relative_error(lp: LP, x: np.ndarray, y: np.ndarray) -> dict:
    """Relative KKT errors of (x, y) with the reference's definitions
    (convergence_information.cu:492-811): primal residual against the row bounds, dual residual
    with the reduced cost taken as the projection of c - A^T y onto the normal cone of the
    variable bounds at x, and the primal/dual objective gap."""
    ax = lp.matvec(x)
    rp = ax - np.clip(ax, lp.con_lo, lp.con_up)
    g = lp.c - lp.rmatvec(y)
    # reduced cost allowed only where the bound is active
    rc = np.where(np.isfinite(lp.var_lo) & (x <= lp.var_lo) & (g > 0), g, 0.0) + \
        np.where(np.isfinite(lp.var_up) & (x >= lp.var_up) & (g < 0), g, 0.0)
    rd = g - rc
    fin = lambda v: np.where(np.isfinite(v), v, 0.0)
    pobj = float(lp.c @ x)
    dobj = float(np.sum(np.maximum(y, 0) * fin(lp.con_lo) + np.minimum(y, 0) * fin(lp.con_up))
                 + np.sum(np.maximum(rc, 0) * fin(lp.var_lo) + np.minimum(rc, 0) * fin(lp.var_up)))
    bnorm = np.sqrt(np.sum(np.where(np.isfinite(lp.con_lo) & (lp.con_lo != lp.con_up),
                                    fin(lp.con_lo) ** 2, 0.0) + fin(lp.con_up) ** 2))
    return {
        "rel_primal": float(np.linalg.norm(rp) / (1.0 + bnorm)),
        "rel_dual": float(np.linalg.norm(rd) / (1.0 + np.linalg.norm(lp.c))),
        "rel_gap": abs(pobj - dobj) / (1.0 + abs(pobj) + abs(dobj)),
        "primal_objective": pobj,
        "dual_objective": dobj,
    }
