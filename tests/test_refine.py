"""Limits-adaptive refinement on the CPU: the library's host step
(sg_refine_step) against the restated policy (oracle/refine_policy.py), its
caps, and a refinement loop whose final grid is pinned to the reference's own
init()/hierarchize0() for the limits it chose (structure and FP32 surpluses
bit-exact: the reference's adaptive grid is exactly such a limit vector,
adaptive_sparse_grid_bench.c:82-83, c:113-129)."""
import numpy as np
import pytest

import adaptive_sparse_grid_bench_b200 as sg
from adaptive_sparse_grid_bench_b200 import inputs
from oracle import refine_policy as rp
from oracle.oracle import Oracle, Reference

SHAPES = [(1, 7, None), (2, 5, None), (3, 6, [2, 5, 4]), (4, 4, None), (6, 4, None), (5, 5, [0, 4, 1, 4, 2]),
          (3, 8, [7, 1, 3])]


@pytest.mark.parametrize("d,n,lim", SHAPES)
def test_step_matches_restatement(d, n, lim):
    o = Oracle(d, n, lim)
    limits = lim if lim is not None else [n - 1] * d
    rng = np.random.default_rng(d * 100 + n)
    for trial in range(12):
        # magnitudes spread over decades so every tol splits the subspaces
        m = (10.0 ** rng.uniform(-7, 0, o.S)).astype(np.float32)
        if trial % 4 == 0:
            m[rng.integers(0, o.S)] = 0.0
        tol = float(10.0 ** rng.uniform(-6, -1))
        max_level = int(rng.integers(0, 10))
        got = sg.refine_step(d, n, limits, m, tol, max_level)
        want = rp.refine_step(o, limits, m, tol, max_level)
        assert got[0] == want[0] and list(got[1]) == want[1] and got[2] == want[2], (trial, tol, max_level)


def test_step_fixed_point_and_caps():
    # nothing active: same grid
    n2, l2, ch = sg.refine_step(3, 5, None, np.zeros(35, np.float32), 1e-4, 13)
    assert (n2, list(l2), ch) == (5, [4, 4, 4], False)
    # everything active: one more level sum, limits follow
    o = Oracle(2, 4)
    n2, l2, ch = sg.refine_step(2, 4, None, np.ones(o.S, np.float32), 1e-4, 13)
    assert (n2, list(l2), ch) == (5, [4, 4], True)
    # max_level 1: only children l_k = 0 -> 1; (0,3) -> (1,3) still raises n
    n2, l2, ch = sg.refine_step(2, 4, [1, 3], np.ones(Oracle(2, 4, [1, 3]).S, np.float32), 0.0, 1)
    assert (n2, list(l2), ch) == (5, [1, 3], True)
    # max_level 0: no children at all
    n2, l2, ch = sg.refine_step(2, 4, [1, 3], np.ones(Oracle(2, 4, [1, 3]).S, np.float32), 0.0, 0)
    assert (n2, list(l2), ch) == (4, [1, 3], False)
    o = Oracle(1, 16)
    n2, l2, ch = sg.refine_step(1, 16, None, np.ones(o.S, np.float32), 0.0, 30)
    assert (n2, list(l2), ch) == (16, [15], False)
    with pytest.raises(sg.SgError):
        sg.refine_step(2, 4, None, np.ones(10, np.float32), -1.0, 3)


def _bump_values(d, n, lim):
    X = Oracle(d, n, lim).grid_points().astype(np.float64)
    return inputs.f_bump(X).astype(np.float32)


@pytest.mark.parametrize("d,n0,lim0,tol", [(2, 3, None, 1e-3), (3, 3, [1, 2, 0], 3e-3), (1, 2, None, 1e-5)])
def test_refinement_loop_pinned_to_reference(d, n0, lim0, tol):
    n, lim, it, surplus = rp.refine(d, n0, _bump_values, tol, 13, 1 << 20, 20, lim0)
    assert it >= 2  # it refined at least once
    o = Oracle(d, n, lim)
    # the final grid has no active subspace with a missing child
    n2, l2, ch = rp.refine_step(o, lim, rp.subspace_maxabs(o, surplus), tol, 13)
    assert not ch or Oracle(d, n2, l2).N > (1 << 20) or it == 20
    if not Reference.available():
        pytest.skip("oracle/_ref not built")
    r = Reference(d, n, lim)
    assert (r.N, r.S) == (o.N, o.S)
    dp, lidx = r.tables()
    assert np.array_equal(dp.astype(np.int64), o.dp) and np.array_equal(lidx.astype(np.int64), o.lidx[:n])
    r.set_values(_bump_values(d, n, lim))
    r.hierarchize(0)
    assert np.array_equal(r.values().view(np.uint32), surplus.view(np.uint32))
