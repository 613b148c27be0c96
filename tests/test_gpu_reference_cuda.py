"""The reference's own CUDA kernels, compiled by oracle/Makefile, on the GPU.
Evaluation (evaluate5, adaptive_sparse_grid_bench_cuda.cu:1522-1598): its
results agree with the FP64 oracle at the reference's FP32 accuracy and with
this library's evaluation.  Tolerance: 1e-4 of max|u| (the reference sums in
FP32 without compensation, in evaluate0's order, c:1237-1274).
Hierarchization (hierarchize7, cu:1053-1160, with the warp barriers it lacks
added): surpluses bit-identical to hierarchize0 and to this library.  So
timing them next to the library compares like with like."""
import numpy as np
import pytest

import adaptive_sparse_grid_bench_b200 as sg
from adaptive_sparse_grid_bench_b200 import inputs
from oracle.oracle import Oracle, ReferenceCUDA

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("d,n,P", [(4, 8, 32), (4, 8, 64), (6, 6, 128), (10, 5, 256)])
def test_reference_evaluate5_agrees(cuda, d, n, P):
    assert ReferenceCUDA.available(), "oracle/_ref/libasgb_refcuda.so is not built (make -C oracle)"
    g = sg.Grid(d, n)
    g.set_values(inputs.grid_values(g, inputs.f_gauss))
    g.hierarchize()
    surplus = g.get_values()
    X = inputs.uniform_points(21 + d, 8 * P * 3, d)
    out, tk, tt = ReferenceCUDA.evaluate5(d, n, surplus, X, P, reps=2)
    assert tk > 0 and tt >= tk
    ref64 = Oracle(d, n).evaluate_f64(surplus.astype(np.float64), X)
    scale = np.abs(ref64).max()
    assert np.abs(out - ref64).max() <= 1e-4 * scale
    assert np.abs(out - g.evaluate(X)).max() <= 1e-4 * scale


@pytest.mark.parametrize("d,n", [(4, 8), (6, 6), (2, 10), (10, 7)])
def test_reference_hierarchize7_bitexact(cuda, d, n):
    """The reference's hierarchize7 (cu:1053-1160, with the warp barriers
    added) gives surpluses bit-identical to hierarchize0 (c:557-571) and to
    this library's hierarchization: its timing compares like with like."""
    assert ReferenceCUDA.available(), "oracle/_ref/libasgb_refcuda.so is not built (make -C oracle)"
    g = sg.Grid(d, n)
    vals = inputs.grid_values(g, inputs.f_gauss)
    out, tk, tt = ReferenceCUDA.hierarchize7(d, n, vals, reps=2)
    assert tk > 0 and tt >= tk
    want = Oracle(d, n).hierarchize_f32(vals)
    assert np.array_equal(out.view(np.uint32), want.view(np.uint32))
    g.set_values(vals)
    g.hierarchize()
    assert np.array_equal(g.get_values().view(np.uint32), out.view(np.uint32))
