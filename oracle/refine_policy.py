"""CPU restatement of the limits-adaptive refinement (TEST INFRASTRUCTURE ONLY).

The reference has no refinement: its adaptive grid is the limit vector of
init() (adaptive_sparse_grid_bench.c:82-83, c:113-129).  This file restates
the refinement policy of the library's sg_refine_step / sg_refine in plain
Python over the oracle (`Oracle`, sg_oracle.c), so the tests can check the
library's host step and its GPU driver:
  - per-subspace max |surplus| in compact subspace order;
  - a subspace is active when that maximum exceeds tol; each child l + e_k
    (l_k < max_level) of an active subspace must be in the next grid, the
    smallest (n', limits') containing the current grid and those children,
    with n' capped at 16 levels.
Only the test suite imports this module.
"""
from __future__ import annotations

import numpy as np

from .oracle import Oracle

MAX_LEVELS = 16


def subspace_levels(o: Oracle):
    """Level vectors of all subspaces in compact order (group s ascending,
    idx2l positions inside a group)."""
    out = []
    for s in range(o.n):
        cnt = (int(o.lidx[s + 1]) - int(o.lidx[s])) >> s
        for pos in range(cnt):
            out.append((s, tuple(int(v) for v in o.idx2l(pos, s))))
    return out


def subspace_maxabs(o: Oracle, values) -> np.ndarray:
    """max |value| per subspace of compact-order values (N floats)."""
    v = np.abs(np.asarray(values, np.float32))
    res = []
    for s in range(o.n):
        seg = v[int(o.lidx[s]):int(o.lidx[s + 1])]
        if seg.size:
            res.append(seg.reshape(-1, 1 << s).max(axis=1))
    return np.concatenate(res) if res else np.zeros(0, np.float32)


def refine_step(o: Oracle, limits, maxabs, tol: float, max_level: int):
    """(n', limits', changed) for grid (o.d, o.n, limits)."""
    lim = [min(int(x), o.n - 1) for x in limits]
    new_lim = list(lim)
    nn = o.n
    for (s, lv), m in zip(subspace_levels(o), maxabs):
        if not float(m) > tol:
            continue
        for k in range(o.d):
            if lv[k] >= max_level:
                continue
            new_lim[k] = max(new_lim[k], lv[k] + 1)
            nn = max(nn, s + 2)
    nn = min(nn, MAX_LEVELS)
    new_lim = [min(x, nn - 1) for x in new_lim]
    return nn, new_lim, (nn != o.n or new_lim != lim)


def refine(d: int, n0: int, nodal_values, tol: float, max_level: int, max_points: int, max_iters: int,
           limits0=None, precision: str = "fp32"):
    """The driver's loop with the oracle's hierarchization (FP32, or FP64
    rounded once to FP32).  nodal_values(d, n, limits) -> compact FP32 values
    of f at that grid's points.  Returns (n, limits, iterations, surpluses of
    the last grid)."""
    n = n0
    lim = list(limits0) if limits0 is not None else [n0 - 1] * d
    it = 0
    while True:
        it += 1
        o = Oracle(d, n, lim)
        lim = [min(x, n - 1) for x in lim]
        v = nodal_values(d, n, lim)
        if precision == "fp64":
            surplus = o.hierarchize_f64(np.asarray(v, np.float64)).astype(np.float32)
        else:
            surplus = o.hierarchize_f32(v)
        if it == max_iters:
            return n, lim, it, surplus
        nn, nl, changed = refine_step(o, lim, subspace_maxabs(o, surplus), tol, max_level)
        if not changed or Oracle(d, nn, nl).N > max_points:
            return n, lim, it, surplus
        n, lim = nn, nl
