"""Limits-adaptive refinement on the GPU through the C ABI: the per-subspace
statistic (sg_subspace_maxabs) bit-exact against the oracle, and the driver
(sg_refine) choosing exactly the grids the restated loop chooses
(oracle/refine_policy.py, fed the same device-sampled nodal values), with
the final surpluses bit-exact (FP32: hierarchize0, c:557-571; FP64: the FP64
oracle rounded once)."""
import numpy as np
import pytest

import adaptive_sparse_grid_bench_b200 as sg
from adaptive_sparse_grid_bench_b200 import _lib
from oracle import refine_policy as rp
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

BUMP = (0.3, 50.0)


def _device_nodal(d, n, lim):
    g = sg.Grid(d, n, lim)
    g.sample_function(_lib.SG_FN_BUMP, BUMP)
    v = g.get_values()
    g.close()
    return v


@pytest.mark.parametrize("d,n,lim", [(1, 9, None), (2, 8, [3, 7]), (3, 7, None), (6, 5, [4, 1, 4, 2, 3, 4]),
                                     (10, 4, None), (4, 9, None)])
def test_subspace_maxabs_exact(cuda, d, n, lim):
    g = sg.Grid(d, n, lim)
    g.sample_function(_lib.SG_FN_BUMP, BUMP)
    g.hierarchize()
    got = g.subspace_maxabs()
    want = rp.subspace_maxabs(Oracle(d, n, lim), g.get_values())
    assert got.shape == (g.num_subspaces,)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    # twice in a row: the shared scratch is cleared between calls
    assert np.array_equal(g.subspace_maxabs().view(np.uint32), want.view(np.uint32))


CASES = [  # d, n0, limits0, tol, max_level, max_points, max_iters, precision
    (2, 3, None, 1e-3, 13, 1 << 20, 20, "fp32"),
    (3, 3, [1, 2, 0], 3e-3, 13, 1 << 20, 20, "fp32"),
    (6, 4, None, 1e-4, 6, 2_000_000, 8, "fp32"),
    (4, 3, None, 1e-4, 13, 1 << 20, 3, "fp32"),       # stops at the iteration cap
    (5, 3, None, 1e-5, 13, 200_000, 30, "fp32"),      # stops before the point cap
    (3, 3, None, 1e-3, 9, 1 << 20, 20, "fp64"),
]


@pytest.mark.parametrize("case", CASES)
def test_driver_matches_restated_loop(cuda, case):
    d, n0, lim0, tol, max_level, max_points, max_iters, prec = case
    g, it = sg.refine(d, n0, _lib.SG_FN_BUMP, BUMP, tol, max_level, max_points, max_iters, lim0, prec)
    n, lim, it_w, surplus = rp.refine(d, n0, _device_nodal, tol, max_level, max_points, max_iters, lim0, prec)
    assert (g.n, list(g.limits), it) == (n, lim, it_w)
    assert g.num_points <= max_points or it == 1
    assert np.array_equal(g.get_values().view(np.uint32), surplus.view(np.uint32))
    g.close()
