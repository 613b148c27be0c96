"""Limits-adaptive refinement over the C ABI (sg_refine_step, sg_refine).

The reference's adaptive grid is a per-dimension level limit vector
(adaptive_sparse_grid_bench.c:82-83, c:113-129); these calls grow (n, limits)
from the per-subspace maximum |surplus| so that every grid produced is one
the reference's init()/hierarchize0() reproduce for the same limits.
Levels are 0-based as in the reference.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from ._lib import check
from .grid import Grid


def refine_step(d: int, n: int, limits, maxabs, tol: float, max_level: int):
    """One step on the host: returns (n_out, limits_out, changed)."""
    lim = np.ascontiguousarray(limits if limits is not None else [n - 1] * d, np.int32)
    m = np.ascontiguousarray(maxabs, np.float32)
    n_out = C.c_int()
    lim_out = np.zeros(d, np.int32)
    changed = C.c_int()
    check(L.lib().sg_refine_step(int(d), int(n), lim.ctypes.data, m.ctypes.data, float(tol), int(max_level),
                                 C.byref(n_out), lim_out.ctypes.data, C.byref(changed)))
    return n_out.value, lim_out, bool(changed.value)


def refine(d: int, n0: int, fn: int, params=(), tol: float = 1e-4, max_level: int = 13,
           max_points: int = 1 << 28, max_iters: int = 32, limits0=None, precision: str = "fp32"):
    """The driver: returns (hierarchized Grid, number of grids built)."""
    p = np.ascontiguousarray(params, np.float64)
    lim = None if limits0 is None else np.ascontiguousarray(limits0, np.int32)
    h = C.c_void_p()
    it = C.c_int()
    prec = L.SG_HIER_FP64 if precision == "fp64" else L.SG_HIER_FP32
    check(L.lib().sg_refine(int(d), int(n0), lim.ctypes.data if lim is not None else None, int(fn),
                            p.ctypes.data if p.size else None, int(p.size), float(tol), int(max_level),
                            int(max_points), int(max_iters), prec, C.byref(h), C.byref(it)))
    return Grid.from_handle(h), it.value
