"""The no-allocation evaluation entry point, sg_evaluate_device_noalloc.

It exists for callers that cannot call cudaMalloc when they evaluate: serving
loops whose device memory is reserved up front by their own pool,
latency-bound request paths that cannot afford an allocation's device
synchronisation, and plugin hosts that forbid device allocations.  Its sort
scratch is a fixed array inside the library instead of a buffer grown with
cudaMalloc.  This file is collected last so that a run stopping at the first
failure has run every other test before it; it also passes alone.
"""
import ctypes as C

import numpy as np
import pytest

import adaptive_sparse_grid_bench_b200 as sg
from adaptive_sparse_grid_bench_b200 import _lib, inputs

pytestmark = pytest.mark.gpu

# the evaluation tolerance of the parity tests
EVAL_RTOL_NORM = 1e-5
EVAL_ATOL = 2e-7


def _close(a, b):
    a = a.astype(np.float64)
    b = b.astype(np.float64)
    bound = EVAL_RTOL_NORM * max(np.max(np.abs(b)), 1e-30) + EVAL_ATOL
    return float(np.max(np.abs(a - b))) <= bound


def test_noalloc_matches_evaluate_device_twice(cuda):
    import torch
    d, n = 10, 7
    g = sg.Grid(d, n)
    g.sample_function(_lib.SG_FN_GAUSS)
    g.hierarchize()
    m1, m2 = 100_003, _lib.SG_NOALLOC_MAX_POINTS
    X1 = torch.from_numpy(inputs.uniform_points(21, m1, d)).to(cuda)
    X2 = torch.from_numpy(inputs.uniform_points(22, m2, d)).to(cuda)
    ref1 = torch.empty(m1, device=cuda)
    ref2 = torch.empty(m2, device=cuda)
    g.evaluate_device(X1, ref1)
    g.evaluate_device(X2, ref2)
    g.sync()
    out0 = torch.empty(m2, device=cuda)
    out1 = torch.empty(m1, device=cuda)
    out2 = torch.empty(m2, device=cuda)
    bytes_before = g.device_bytes()
    # the first call on a device looks up the fixed array, which makes the
    # CUDA runtime place it on this device (SG_NOALLOC_SCRATCH_BYTES, held
    # until exit); later calls must not change free device memory at all
    g.evaluate_device_noalloc(X2, out0)
    g.sync()
    free_before = torch.cuda.mem_get_info()[0]
    # two calls in a row: the second reuses the array the first left behind
    g.evaluate_device_noalloc(X1, out1)
    g.evaluate_device_noalloc(X2, out2)
    g.sync()
    free_after = torch.cuda.mem_get_info()[0]
    assert g.device_bytes() == bytes_before
    assert free_after == free_before
    assert _close(out0.cpu().numpy(), ref2.cpu().numpy())
    assert _close(out1.cpu().numpy(), ref1.cpu().numpy())
    assert _close(out2.cpu().numpy(), ref2.cpu().numpy())


def test_noalloc_after_value_change(cuda):
    """New values reach the no-allocation path (the block layout is rebuilt
    in place)."""
    import torch
    d, n = 4, 8
    g = sg.Grid(d, n)
    X = torch.from_numpy(inputs.uniform_points(3, 4096, d)).to(cuda)
    out = torch.empty(4096, device=cuda)
    ref = torch.empty(4096, device=cuda)
    for fn in (_lib.SG_FN_PROD4, _lib.SG_FN_GAUSS):
        g.sample_function(fn)
        g.hierarchize()
        g.evaluate_device_noalloc(X, out)
        g.evaluate_device(X, ref)
        g.sync()
        assert _close(out.cpu().numpy(), ref.cpu().numpy())


def test_noalloc_rejects_what_it_cannot_do(cuda):
    import torch
    lib = sg.lib()
    g = sg.Grid(3, 4)
    x = torch.zeros((8, 3), device=cuda)
    o = torch.zeros(8, device=cuda)
    # no device state yet: refusing is the only way not to allocate
    assert lib.sg_evaluate_device_noalloc(g.handle, x.data_ptr(), o.data_ptr(), 8, None) == _lib.SG_ERR_STATE
    g.sample_function(_lib.SG_FN_PROD4)
    m = _lib.SG_NOALLOC_MAX_POINTS + 1
    assert lib.sg_evaluate_device_noalloc(g.handle, x.data_ptr(), o.data_ptr(), m, None) == _lib.SG_ERR_RANGE
    assert b"SG_NOALLOC_MAX_POINTS" in lib.sg_last_error()
    assert lib.sg_evaluate_device_noalloc(g.handle, x.data_ptr(), o.data_ptr(), 0, None) == _lib.SG_OK
