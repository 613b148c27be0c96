"""The reference's own CUDA evaluation kernel (evaluate5,
adaptive_sparse_grid_bench_cuda.cu:1522-1598), compiled in place, on the
GPU: its results agree with the FP64 oracle at the reference's FP32 accuracy
and with this library's evaluation, so timing it next to the library
compares like with like.  Tolerance: 1e-4 of max|u| (the reference sums in
FP32 without compensation, in evaluate0's order, c:1237-1274)."""
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
