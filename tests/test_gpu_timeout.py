"""The bounded device-side waits of the staged hierarchization sweeps.

With SG_OPT_TEST_WAIT the first staged chain of every CTA announces its copy
bytes but never starts a copy, so the CTA's wait on that stage can only run
out (no copy is in flight towards it, nothing else waits on it).  The kernel
must give up after the short limit, set the error flag and return; the host
reads the flag in sg_sync (SG_ERR_TIMEOUT), the context stays usable, and
the same handle then hierarchizes normally, bit-identical to hierarchize0
(c:557-571).
"""
import time

import numpy as np
import pytest

import adaptive_sparse_grid_bench_b200 as sg
from adaptive_sparse_grid_bench_b200 import _lib, inputs
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("d,n", [(3, 8), (6, 5)])
def test_wait_runs_out_reports_timeout_and_recovers(cuda, d, n):
    import torch
    g = sg.Grid(d, n)
    v = inputs.uniform01(55 + d, g.num_points) * 2 - 1
    g.set_values(v)
    g.set_option(_lib.SG_OPT_HIER_KERNEL, 1)
    g.set_option(_lib.SG_OPT_TEST_WAIT, 8)  # 8 * 2^20 cycles, a few ms per wait
    t0 = time.perf_counter()
    with pytest.raises(sg.SgError) as e:
        g.hierarchize()
    assert e.value.code == _lib.SG_ERR_TIMEOUT
    assert time.perf_counter() - t0 < 30.0  # every wait ended on its own
    # the error flag was read and cleared; the context is usable
    g.sync()
    x = torch.arange(1000, device=cuda, dtype=torch.float32)
    assert float(x.sum()) == 499500.0
    g.set_option(_lib.SG_OPT_TEST_WAIT, 0)
    g.set_values(v)
    g.hierarchize()
    want = Oracle(d, n).hierarchize_f32(v)
    assert np.array_equal(g.get_values().view(np.uint32), want.view(np.uint32))


def test_wait_option_is_checked(cuda):
    g = sg.Grid(3, 4)
    for bad in (-1, 2049):
        with pytest.raises(sg.SgError):
            g.set_option(_lib.SG_OPT_TEST_WAIT, bad)
