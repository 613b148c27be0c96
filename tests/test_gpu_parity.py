"""GPU parity: the sm_100a kernels through the C ABI against the oracle and
the reference's golden fixtures.

Tolerances (stated here, used below):
  - index bijection, grid structure: bit-exact;
  - FP32 hierarchization: bit-exact with hierarchize0 (c:557-571);
  - FP64 hierarchization: bit-exact with the FP64 oracle rounded once to FP32;
  - evaluation: |gpu - oracle_fp64| <= EVAL_ATOL_REL * max|oracle_fp64| + EVAL_ATOL_ULP
    (norm-wise relative error 1e-5 plus a few FP32 ulps of 1 for values near 0).
"""
import numpy as np
import pytest

import adaptive_sparse_grid_bench_b200 as sg
from adaptive_sparse_grid_bench_b200 import _lib, inputs
from conftest import golden_cases, load_golden
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

EVAL_RTOL_NORM = 1e-5
EVAL_ATOL = 2e-7


def _grid(d, n, lim=None, opt=None):
    g = sg.Grid(d, n, lim)
    for k, v in (opt or {}).items():
        g.set_option(k, v)
    return g


def assert_eval_close(got, ref64, what=""):
    ref64 = np.asarray(ref64, np.float64)
    scale = max(np.max(np.abs(ref64)), 1e-30)
    err = np.abs(got.astype(np.float64) - ref64)
    bound = EVAL_RTOL_NORM * scale + EVAL_ATOL
    assert np.all(err <= bound), f"{what}: max err {err.max():.3e} > {bound:.3e} (max|u| {scale:.3e})"


@pytest.mark.parametrize("name", golden_cases())
def test_golden_hierarchize_bitexact(cuda, name):
    gd = load_golden(name)
    g = sg.Grid(int(gd["d"]), int(gd["n"]), gd["limits"])
    assert g.num_points == int(gd["N"]) and g.num_subspaces == int(gd["S"])
    g.set_values(gd["values"])
    g.hierarchize()
    h = g.get_values()
    assert np.array_equal(h.view(np.uint32), gd["surplus"].view(np.uint32))


@pytest.mark.parametrize("name", golden_cases())
def test_golden_evaluate(cuda, name):
    gd = load_golden(name)
    d, n = int(gd["d"]), int(gd["n"])
    g = sg.Grid(d, n, gd["limits"])
    g.set_values(gd["surplus"])
    o = Oracle(d, n, gd["limits"])
    ref64 = o.evaluate_f64(gd["surplus"].astype(np.float64), gd["X"])
    for sort in (0, 1):
        g.set_option(sg.SG_OPT_EVAL_SORT, sort)
        out = g.evaluate(gd["X"])
        assert_eval_close(out, ref64, f"{name} sort={sort}")
        # and against the reference's own FP32 evaluate0 at its own accuracy
        np.testing.assert_allclose(out, gd["out"], rtol=0, atol=1e-5 * max(1.0, np.abs(gd["out"]).max()))
    # the reference's correctness test: interpolation at grid points
    outg = g.evaluate(gd["G"])
    np.testing.assert_allclose(outg, gd["outG"], rtol=0, atol=1e-6)


SHAPES = [
    (1, 1, None), (1, 12, None), (2, 9, None), (3, 7, [6, 2, 4]), (4, 8, None), (5, 6, [5, 0, 5, 3, 1]),
    (6, 6, None), (8, 5, None), (10, 5, None), (12, 4, None), (20, 3, None), (3, 12, None),
]


@pytest.mark.parametrize("d,n,lim", SHAPES)
@pytest.mark.parametrize("kernel", [0, 2])
def test_hierarchize_fp32_bitexact(cuda, d, n, lim, kernel):
    o = Oracle(d, n, lim)
    g = _grid(d, n, lim, {sg.SG_OPT_HIER_KERNEL: kernel})
    v = inputs.uniform01(d * 31 + n, g.num_points) * 2 - 1
    g.set_values(v)
    g.hierarchize()
    got = g.get_values()
    want = o.hierarchize_f32(v)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("d,n,lim", SHAPES)
@pytest.mark.parametrize("kernel", [0, 2])
def test_hierarchize_fp64_matches_fp64_oracle(cuda, d, n, lim, kernel):
    o = Oracle(d, n, lim)
    g = _grid(d, n, lim, {sg.SG_OPT_HIER_KERNEL: kernel, sg.SG_OPT_HIER_PRECISION: sg.SG_HIER_FP64})
    v = inputs.uniform01(d * 17 + n, g.num_points) * 2 - 1
    g.set_values(v)
    g.hierarchize()
    got = g.get_values()
    want = o.hierarchize_f64(v.astype(np.float64)).astype(np.float32)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("d,n,lim", [(4, 8, None), (3, 7, [6, 2, 4]), (10, 5, None), (1, 12, None), (6, 6, None)])
@pytest.mark.parametrize("ppt", [1, 2])
def test_evaluate_vs_fp64_oracle(cuda, d, n, lim, ppt):
    o = Oracle(d, n, lim)
    g = _grid(d, n, lim, {sg.SG_OPT_EVAL_PPT: ppt})
    vals = inputs.grid_values(g, inputs.f_gauss)
    g.set_values(vals)
    g.hierarchize()
    surplus = g.get_values()
    X = inputs.uniform_points(5, 777, d)
    ref64 = o.evaluate_f64(surplus.astype(np.float64), X)
    for sort in (1, 0):
        g.set_option(sg.SG_OPT_EVAL_SORT, sort)
        assert_eval_close(g.evaluate(X), ref64, f"d={d} n={n} sort={sort} ppt={ppt}")


@pytest.mark.parametrize("d,n,lim", [(10, 8, None), (4, 12, None), (6, 9, [8, 2, 5, 8, 8, 1]), (3, 12, [11, 4, 9]),
                                     (12, 6, None), (5, 10, [9, 9, 9, 3, 9])])
def test_blocking_presets_bit_identical(cuda, d, n, lim):
    # every subspace blocking (wide, medium) at one and two points
    # per thread gives the same bits, and they are within tolerance of FP64
    o = Oracle(d, n, lim)
    g = _grid(d, n, lim)
    g.set_values(inputs.grid_values(g, inputs.f_gauss))
    g.hierarchize()
    X = inputs.uniform_points(17, 3000, d)
    outs = {}
    for blocking in range(1, _lib.SG_EVAL_BLOCKINGS + 1):
        for ppt in (1, 2):
            g.set_option(sg.SG_OPT_EVAL_BLOCKING, blocking)
            g.set_option(sg.SG_OPT_EVAL_PPT, ppt)
            outs[blocking, ppt] = g.evaluate(X)
    first = outs[1, 1]
    for key, out in outs.items():
        assert np.array_equal(out.view(np.uint32), first.view(np.uint32)), f"blocking, ppt = {key}"
    assert_eval_close(first, o.evaluate_f64(g.get_values().astype(np.float64), X), f"d={d} n={n}")


def test_evaluate_edge_coordinates(cuda):
    d, n = 3, 6
    o = Oracle(d, n)
    g = sg.Grid(d, n)
    g.set_values(inputs.grid_values(g, inputs.f_prod4))
    g.hierarchize()
    s = g.get_values()
    below1 = np.nextafter(np.float32(1), np.float32(0))
    X = np.array([[0, 0, 0], [below1] * 3, [0.5, 0.5, 0.5], [0, 0.5, below1],
                  [2.0 ** -24, 0.25, 0.75]], np.float32)
    assert_eval_close(g.evaluate(X), o.evaluate_f64(s.astype(np.float64), X), "edges")
    # outside [0,1)^d every basis function vanishes: 0 (NaN stays NaN)
    Y = np.array([[1.0, 0.5, 0.5], [-0.1, 0.5, 0.5], [0.5, 3.0, 0.5], [np.nan, 0.5, 0.5]], np.float32)
    out = g.evaluate(Y)
    assert np.array_equal(out[:3], np.zeros(3, np.float32)) and np.isnan(out[3])


@pytest.mark.parametrize("m", [0, 1, 2, 31, 33, 255, 257, 4099])
def test_evaluate_ragged_counts(cuda, m):
    d, n = 5, 5
    o = Oracle(d, n)
    g = sg.Grid(d, n)
    g.set_values(inputs.grid_values(g, inputs.f_gauss))
    g.hierarchize()
    s = g.get_values()
    X = inputs.uniform_points(m + 3, m, d)
    out = g.evaluate(X)
    assert out.shape == (m,)
    if m:
        assert_eval_close(out, o.evaluate_f64(s.astype(np.float64), X), f"m={m}")


def test_evaluate_device_api_and_repeat(cuda):
    import torch
    d, n = 4, 8
    g = sg.Grid(d, n)
    vals = inputs.grid_values(g, inputs.f_prod4)
    dv = torch.from_numpy(vals).to(cuda)
    g.set_values_device(dv)
    g.hierarchize_async()
    X = inputs.uniform_points(0, 65536, d)
    dX = torch.from_numpy(X).to(cuda)
    out1 = torch.empty(X.shape[0], device=cuda)
    out2 = torch.empty(X.shape[0], device=cuda)
    g.evaluate_device(dX, out1)
    g.evaluate_device(dX, out2)
    g.sync()
    assert torch.equal(out1, out2)
    host = g.evaluate(X)
    assert np.array_equal(host, out1.cpu().numpy())
    back = torch.empty(g.num_points, device=cuda)
    g.get_values_device(back)
    g.sync()
    assert np.array_equal(back.cpu().numpy(), g.get_values())


def test_device_bijection(cuda):
    import torch
    for d, n, lim in [(4, 8, None), (3, 7, [6, 2, 4]), (10, 5, None)]:
        g = sg.Grid(d, n, lim)
        o = Oracle(d, n, lim)
        idx = torch.arange(g.num_points, dtype=torch.int64, device=cuda)
        lv = torch.empty((g.num_points, d), dtype=torch.int32, device=cuda)
        ix = torch.empty_like(lv)
        g.idx2gp_device(idx, lv, ix, g.num_points)
        back = torch.empty_like(idx)
        g.gp2idx_device(lv, ix, back, g.num_points)
        torch.cuda.synchronize()
        assert torch.equal(back, idx)
        lvh, ixh = lv.cpu().numpy(), ix.cpu().numpy()
        for i in range(0, g.num_points, max(1, g.num_points // 300)):
            a, b = o.idx2gp(i)
            assert np.array_equal(lvh[i], a) and np.array_equal(ixh[i], b)


@pytest.mark.parametrize("fn,params,host", [
    (0, (), inputs.f_reference), (1, (), inputs.f_prod4), (2, (), inputs.f_gauss),
    (3, (0.3, 50.0), inputs.f_bump), (4, None, None)])
def test_sample_function_on_device(cuda, fn, params, host):
    d, n, lim = 4, 7, [6, 3, 6, 2]
    g = sg.Grid(d, n, lim)
    if fn == 4:
        coef = (inputs.uniform01(3, 3 * d).astype(np.float64) * 2 - 1).reshape(d, 3)
        params = coef.reshape(-1)
        host = lambda X: inputs.f_quad(X, coef)  # noqa: E731
    g.sample_function(fn, params)
    got = g.get_values()
    want = host(inputs.grid_coordinates(g)).astype(np.float32)
    # FP64 evaluation order and libm may differ in the last FP64 bits: allow
    # one FP32 ulp after the single rounding
    ulp = np.spacing(np.abs(want).astype(np.float32))
    assert np.all(np.abs(got - want) <= ulp), np.max(np.abs(got - want) / ulp)


def test_errors_on_gpu(cuda):
    g = sg.Grid(3, 4)
    with pytest.raises(sg.SgError) as e:
        g.hierarchize()
    assert e.value.code == -5  # no values yet
    with pytest.raises(sg.SgError):
        g.evaluate(np.zeros((4, 3), np.float32))
    g.set_values(np.ones(g.num_points, np.float32))
    with pytest.raises(ValueError):
        g.set_values(np.ones(g.num_points + 1, np.float32))


@pytest.mark.parametrize("d,n,lim,precision", [(4, 8, None, "fp32"), (10, 6, None, "fp64"), (3, 16, None, "fp32"),
                                               (6, 9, [8, 2, 5, 8, 8, 1], "fp32")])
def test_autotune_keeps_values_and_results(cuda, d, n, lim, precision):
    # every setting the autotuner tries gives the same bits; the grid's
    # values are restored; the chosen options are valid settings
    import torch
    g = _grid(d, n, lim)
    g.precision = precision
    g.set_values(inputs.uniform01(5, g.num_points) * 2 - 1)
    g.hierarchize()
    surplus = g.get_values()
    X = inputs.uniform_points(6, 5000, d)
    want = g.evaluate(X)
    Xd = torch.from_numpy(X).to(cuda)
    out = torch.empty(X.shape[0], device=cuda)
    ms = g.autotune(Xd, out)
    assert all(v > 0 for k, v in ms.items() if k.startswith("eval"))
    assert ms["hier_gather"] > 0
    assert np.array_equal(g.get_values().view(np.uint32), surplus.view(np.uint32))
    assert np.array_equal(out.cpu().numpy().view(np.uint32), want.view(np.uint32))
    assert g.get_option(sg.SG_OPT_EVAL_PPT) in (1, 2) and g.get_option(sg.SG_OPT_EVAL_SORT) in (0, 1)
    assert g.get_option(sg.SG_OPT_HIER_KERNEL) in (1, 2)
    assert g.get_option(sg.SG_OPT_EVAL_BLOCKING) in (1, 2, 3)
    assert np.array_equal(g.evaluate(X).view(np.uint32), want.view(np.uint32))
    # the tuned sweep kernel still gives hierarchize0's bits
    g.set_values(inputs.uniform01(7, g.num_points) * 2 - 1)
    nodal = g.get_values()
    g.hierarchize()
    one = _grid(d, n, lim)
    one.precision = precision
    one.set_values(nodal)
    one.hierarchize()
    assert np.array_equal(g.get_values().view(np.uint32), one.get_values().view(np.uint32))
