"""Batches of grids on the GPU: hierarchization bit-identical to the oracle
(FP32: hierarchize0, c:557-571; FP64: the FP64 oracle rounded once) and to
the single-grid path, evaluation within conftest.check_eval's bounds of the
FP64 oracle and equal to the single-grid evaluation, in both precisions,
with and without CUDA graphs."""
import numpy as np
import pytest

import adaptive_sparse_grid_bench_b200 as sg
from adaptive_sparse_grid_bench_b200 import _lib, inputs
from conftest import check_eval
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

MIXED = [  # (d, n, limits): small grids (shared-memory path) and larger ones (sweeps)
    (2, 3, None), (4, 8, None), (3, 7, [6, 2, 4]), (6, 6, None), (10, 5, None), (1, 9, None),
    (12, 4, None), (5, 9, None), (3, 12, None), (8, 7, None), (2, 9, [8, 3]), (4, 9, None)]


def _batch(shapes):
    dims = [s[0] for s in shapes]
    levels = [s[1] for s in shapes]
    limits = None
    if any(s[2] is not None for s in shapes):
        limits = [s[2] if s[2] is not None else [s[1] - 1] * s[0] for s in shapes]
    return sg.Batch(dims, levels, limits)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("graph,kernel,group", [(1, 0, None), (0, 0, None), (1, 1, None), (1, 3, None),
                                                (1, 0, 0), (1, 0, 1), (0, 3, 1 << 15)])
def test_batch_hierarchize_matches_single_grids(cuda, precision, graph, kernel, group):
    # kernel 0: auto (short chains one warp per chain), 1: staged chains
    # everywhere, 3: one warp per chain wherever the chains fit; group: values
    # per sweep group (None: default, 0: every sweep over the whole batch,
    # 1: one group per grid, run on several streams)
    b = _batch(MIXED)
    if group is not None:
        b.set_option(_lib.SG_OPT_SWEEP_GROUP, group)
    b.set_option(_lib.SG_OPT_USE_GRAPH, graph)
    b.set_option(_lib.SG_OPT_HIER_KERNEL, kernel)
    b.set_option(_lib.SG_OPT_HIER_PRECISION, _lib.SG_HIER_FP64 if precision == "fp64" else _lib.SG_HIER_FP32)
    vals = inputs.uniform01(77, b.num_values) * 2 - 1
    for rep in range(2):  # the second run replays the graph
        b.set_values(vals)
        b.hierarchize()
        got = b.get_values()
    for g, (d, n, lim) in enumerate(MIXED):
        one = sg.Grid(d, n, lim)
        one.precision = precision
        one.set_values(b.grid_values(vals, g))
        one.hierarchize()
        want = one.get_values()
        assert np.array_equal(b.grid_values(got, g).view(np.uint32), want.view(np.uint32)), f"grid {g} {d} {n}"


@pytest.mark.parametrize("ppt,sort,blocking", [(1, 1, 0), (2, 1, 0), (2, 0, 0), (2, 1, 2), (1, 1, 2), (2, 0, 1)])
def test_batch_evaluate_matches_single_grids(cuda, ppt, sort, blocking):
    # the batch under each subspace blocking gives the bits of the single
    # grids under the default one
    import torch
    b = _batch(MIXED)
    b.set_option(_lib.SG_OPT_EVAL_PPT, ppt)
    b.set_option(_lib.SG_OPT_EVAL_SORT, sort)
    b.set_option(_lib.SG_OPT_EVAL_BLOCKING, blocking)
    vals = inputs.uniform01(78, b.num_values) * 2 - 1
    b.set_values(vals)
    b.hierarchize()
    counts = [0, 1, 513, 1000, 257, 33, 2048, 600, 70, 511, 512, 1025]
    po = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    Xs = [inputs.uniform_points(100 + g, counts[g], MIXED[g][0]) for g in range(len(MIXED))]
    coords = torch.from_numpy(np.concatenate([x.reshape(-1) for x in Xs]).astype(np.float32)).to(cuda)
    out = torch.full((int(po[-1]),), np.nan, device=cuda)
    for rep in range(2):
        b.evaluate_device(po, coords, out)
        b.sync()
    res = out.cpu().numpy()
    surplus = b.get_values()
    for g, (d, n, lim) in enumerate(MIXED):
        if counts[g] == 0:
            continue
        one = sg.Grid(d, n, lim)
        one.set_values(b.grid_values(surplus, g))
        want = one.evaluate(Xs[g])
        got = res[po[g]:po[g + 1]]
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), f"grid {g}"


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_batch_against_oracle(cuda, precision):
    """Every grid of the mixed batch against the oracle directly: surpluses
    bit for bit, evaluation of the batch's surpluses within tolerance of the
    FP64 evaluation of the same surpluses."""
    import torch
    b = _batch(MIXED)
    b.set_option(_lib.SG_OPT_HIER_PRECISION, _lib.SG_HIER_FP64 if precision == "fp64" else _lib.SG_HIER_FP32)
    vals = inputs.uniform01(90, b.num_values) * 2 - 1
    b.set_values(vals)
    b.hierarchize()
    surplus = b.get_values()
    counts = [3, 1, 513, 1000, 257, 33, 2048, 600, 70, 511, 512, 1025]
    po = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    Xs = [inputs.uniform_points(400 + g, counts[g], MIXED[g][0]) for g in range(len(MIXED))]
    coords = torch.from_numpy(np.concatenate([x.reshape(-1) for x in Xs]).astype(np.float32)).to(cuda)
    out = torch.full((int(po[-1]),), np.nan, device=cuda)
    b.evaluate_device(po, coords, out)
    b.sync()
    res = out.cpu().numpy()
    for g, (d, n, lim) in enumerate(MIXED):
        o = Oracle(d, n, lim)
        nodal = b.grid_values(vals, g)
        want = (o.hierarchize_f32(nodal) if precision == "fp32"
                else o.hierarchize_f64(nodal.astype(np.float64)).astype(np.float32))
        got = b.grid_values(surplus, g)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), f"grid {g} ({d}, {n}, {lim})"
        # random nodal values: the norm-wise bound (conftest.check_eval)
        check_eval(res[po[g]:po[g + 1]], o.evaluate_f64(got.astype(np.float64), Xs[g]), f"grid {g}", per_point=False)


def test_batch_sample_quad_and_config_like_workload(cuda):
    import torch
    dims, levels, coef, counts = inputs.batch_workload(3, 64, max_points=200_000)
    b = sg.Batch(dims, levels)
    b.sample_function(_lib.SG_FN_QUAD, coef)
    b.hierarchize()
    surplus = b.get_values()
    po = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    Xs = [inputs.uniform_points(200 + g, int(counts[g]), int(dims[g])) for g in range(len(dims))]
    coords = torch.from_numpy(np.concatenate([x.reshape(-1) for x in Xs])).to(cuda)
    out = torch.empty(int(po[-1]), device=cuda)
    b.evaluate_device(po, coords, out)
    b.sync()
    res = out.cpu().numpy()
    for g in range(0, len(dims), 9):
        d, n = int(dims[g]), int(levels[g])
        one = sg.Grid(d, n)
        one.sample_function(_lib.SG_FN_QUAD, coef[g, :3 * d])
        vals = one.get_values()
        one.hierarchize()
        assert np.array_equal(one.get_values().view(np.uint32), b.grid_values(surplus, g).view(np.uint32))
        want = one.evaluate(Xs[g])
        assert np.array_equal(res[po[g]:po[g + 1]].view(np.uint32), want.view(np.uint32))
        assert vals.size == b.grid_values(surplus, g).size
        # and end to end against the oracle: hierarchize0's bits, and the
        # FP32 results within tolerance of FP64 hierarchize + evaluate
        o = Oracle(d, n)
        assert np.array_equal(b.grid_values(surplus, g).view(np.uint32), o.hierarchize_f32(vals).view(np.uint32))
        check_eval(res[po[g]:po[g + 1]], o.evaluate_f64(o.hierarchize_f64(vals.astype(np.float64)), Xs[g]),
                   f"config-4 grid {g} (d={d}, n={n})")


def test_batch_autotune_keeps_results(cuda):
    # the autotuner picks points per thread per dimension; results are the
    # same bits before and after, graph replay included
    import torch
    b = _batch(MIXED)
    vals = inputs.uniform01(79, b.num_values) * 2 - 1
    b.set_values(vals)
    b.hierarchize()
    counts = [5, 1, 513, 1000, 257, 33, 2048, 600, 70, 511, 512, 1025]
    po = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    coords = torch.from_numpy(np.concatenate(
        [inputs.uniform_points(300 + g, counts[g], MIXED[g][0]).reshape(-1) for g in range(len(MIXED))])).to(cuda)
    out = torch.empty(int(po[-1]), device=cuda)
    b.evaluate_device(po, coords, out)
    b.sync()
    before = out.cpu().numpy().copy()
    surplus = b.get_values()
    ms = b.autotune(po, coords, out)
    # the sweep tuning hierarchizes saved copies: the values are restored
    assert np.array_equal(b.get_values().view(np.uint32), surplus.view(np.uint32))
    dims_present = sorted({d for d, _, _ in MIXED})
    for d in range(1, _lib.SG_MAX_DIMS + 1):
        if d in dims_present:
            assert np.all(ms[:, :, d] > 0)
        else:
            assert np.all(ms[:, :, d] == -1)
    out.fill_(float("nan"))
    for rep in range(2):
        b.evaluate_device(po, coords, out)
        b.sync()
    assert np.array_equal(out.cpu().numpy().view(np.uint32), before.view(np.uint32))
    # the tuned sweep kernels give the same surpluses
    b.set_values(vals)
    b.hierarchize()
    assert np.array_equal(b.get_values().view(np.uint32), surplus.view(np.uint32))


def test_batch_graph_replays_on_a_stream_are_counted(cuda):
    """On a non-default stream the batch captures its launches once and
    replays the graph; every replay adds the captured kernels to the
    library's launch counter, and gives the same surpluses as direct
    launches."""
    import torch
    vals = inputs.uniform01(81, _batch(MIXED).num_values) * 2 - 1
    direct = _batch(MIXED)
    direct.set_option(_lib.SG_OPT_USE_GRAPH, 0)
    direct.set_values(vals)
    st = torch.cuda.Stream(device=cuda)
    l0 = _lib.kernel_launches()
    direct.hierarchize_async(st)
    direct.sync(st)
    per_run = _lib.kernel_launches() - l0
    assert per_run > 0
    want = direct.get_values()
    g = _batch(MIXED)
    g.set_values(vals)
    for rep in range(3):  # capture + launch, then two replays
        g.set_values(vals)
        l0 = _lib.kernel_launches()
        g.hierarchize_async(st)
        g.sync(st)
        assert _lib.kernel_launches() - l0 == per_run, f"run {rep}"
        assert np.array_equal(g.get_values().view(np.uint32), want.view(np.uint32))
