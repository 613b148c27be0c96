"""GPU parity at the benchmarked configurations, through the C ABI.

  - config 1: d=4, n=8, f = prod_k 4 x_k (1 - x_k), 65,536 uniform points
    (seed 0), exactly as the reference's CPU case;
  - config 2: d=10, n=10 (N = 32,978,945), f = exp(-|x|^2), the points of
    the default benchmark (seed 1), including a full 2^24-point launch;
  - config 3: the limits-adaptive d=6 grid that the benchmark's refinement
    reaches (bump exp(-50 |x - 0.3|^2), tol 1e-4, level <= 13).

Checks and tolerances (stated here, used below):
  - FP32 surpluses bit-identical to the reference's own omp_hierarchize3
    (adaptive_sparse_grid_bench.c:1180) and hierarchize7 (c:1009), run from
    oracle/_ref on the same nodal values; grid structure (N, S, dp_mat,
    lidx_vect) identical to the reference's init() (c:101-140);
  - FP64 hierarchization bit-identical to the FP64 oracle rounded once;
  - evaluation of the FP32 surpluses against the FP64 oracle run end to end
    on the same nodal values (hierarchize0 + evaluate0 restated in double,
    c:557-571, c:1237-1274), within conftest.check_eval's bounds:
      norm-wise   |u - u64| <= 1e-5 max|u64| + 2e-7,
      per point   |u - u64| <= 1e-5 max(|u64|, 1e-2 max|u64|);
  - the reference's own correctness check (c:2027-2029): at grid points the
    interpolant reproduces the sampled f within 1e-6.
"""
import numpy as np
import pytest

import adaptive_sparse_grid_bench_b200 as sg
from adaptive_sparse_grid_bench_b200 import _lib, inputs
from conftest import check_eval
from oracle.oracle import Oracle, Reference

pytestmark = pytest.mark.gpu

GRIDPOINT_ATOL = 1e-6


def grid_point_coords(o: Oracle, idx):
    """Coordinates (2i+1)/2^(l+1) of the grid points with these linear
    indices (c:146-152)."""
    X = np.empty((len(idx), o.d), np.float32)
    for r, j in enumerate(idx):
        lv, ix = o.idx2gp(int(j))
        X[r] = (2 * ix + 1) / np.exp2(lv + 1)
    return X


def check_grid_points(g, o, nodal, count, seed):
    idx = np.unique((inputs.uniform01(seed, count).astype(np.float64) * g.num_points).astype(np.int64))
    out = g.evaluate(grid_point_coords(o, idx))
    err = np.abs(out.astype(np.float64) - nodal[idx].astype(np.float64))
    assert err.max() < GRIDPOINT_ATOL, f"interpolation at grid points: {err.max():.3e}"


def reference_surpluses(d, n, lim, nodal, variant):
    assert Reference.available(), "oracle/_ref/libasgb_ref.so is not built (make -C oracle)"
    r = Reference(d, n, lim)
    assert r.N == nodal.size
    r.set_values(nodal)
    r.hierarchize(variant)
    return r


def check_structure(g, r):
    assert (g.num_points, g.num_subspaces) == (r.N, r.S)
    dp, lidx = g.tables()
    rdp, rlidx = r.tables()
    assert np.array_equal(dp, rdp.astype(np.int64)) and np.array_equal(lidx[:-1], rlidx.astype(np.int64))


def test_config1_d4n8(cuda):
    d, n = 4, 8
    g = sg.Grid(d, n)
    nodal = inputs.grid_values(g, inputs.f_prod4)
    g.set_values(nodal)
    g.hierarchize()
    surplus = g.get_values()
    for variant in (9, 7, 0):  # omp_hierarchize3, hierarchize7, hierarchize0
        r = reference_surpluses(d, n, None, nodal, variant)
        check_structure(g, r)
        assert np.array_equal(surplus.view(np.uint32), r.values().view(np.uint32)), f"variant {variant}"
    o = Oracle(d, n)
    X = inputs.uniform_points(0, 65536, d)
    ref64 = o.evaluate_f64(o.hierarchize_f64(nodal.astype(np.float64)), X)
    for ppt in (1, 2):
        for sort in (1, 0):
            g.set_option(sg.SG_OPT_EVAL_PPT, ppt)
            g.set_option(sg.SG_OPT_EVAL_SORT, sort)
            check_eval(g.evaluate(X), ref64, f"config 1 ppt={ppt} sort={sort}")
    check_grid_points(g, o, nodal, 2048, 11)


@pytest.fixture(scope="module")
def config2():
    """The d=10, n=10 grid of exp(-|x|^2) sampled on the device, its nodal
    values and the FP64 oracle's surpluses."""
    import torch  # noqa: F401  (initialises the CUDA context first)
    d, n = 10, 10
    g = sg.Grid(d, n)
    g.sample_function(_lib.SG_FN_GAUSS)
    nodal = g.get_values()
    o = Oracle(d, n)
    s64 = o.hierarchize_f64(nodal.astype(np.float64))
    g.hierarchize()
    yield g, o, nodal, s64
    g.close()


def test_config2_hierarchize_bitexact_vs_reference(cuda, config2):
    g, o, nodal, s64 = config2
    surplus = g.get_values()
    for variant in (9, 7):  # omp_hierarchize3 (c:1180), hierarchize7 (c:1009)
        r = reference_surpluses(10, 10, None, nodal, variant)
        check_structure(g, r)
        same = surplus.view(np.uint32) == r.values().view(np.uint32)
        assert same.all(), f"variant {variant}: {np.count_nonzero(~same)} surpluses differ"


def test_config2_hierarchize_fp64(cuda, config2):
    g, o, nodal, s64 = config2
    h = sg.Grid(10, 10)
    h.precision = "fp64"
    h.set_values(nodal)
    h.hierarchize()
    assert np.array_equal(h.get_values().view(np.uint32), s64.astype(np.float32).view(np.uint32))
    h.close()


def test_config2_evaluate_vs_fp64(cuda, config2):
    g, o, nodal, s64 = config2
    X = inputs.uniform_points(1, 4096, 10)  # the benchmark's first 4096 points
    ref64 = o.evaluate_f64(s64, X)
    for ppt, sort in ((2, 1), (1, 1), (2, 0)):
        g.set_option(sg.SG_OPT_EVAL_PPT, ppt)
        g.set_option(sg.SG_OPT_EVAL_SORT, sort)
        check_eval(g.evaluate(X), ref64, f"config 2 ppt={ppt} sort={sort}")
    g.set_option(sg.SG_OPT_EVAL_PPT, 2)
    g.set_option(sg.SG_OPT_EVAL_SORT, 1)
    check_grid_points(g, o, nodal, 1024, 12)


def test_config2_full_launch_2p24(cuda, config2):
    """The benchmark's whole 2^24-point launch: every result is finite and
    equal, bit for bit, to the same points evaluated in a small launch; a
    sample spread over the whole array is within tolerance of FP64."""
    import torch
    g, o, nodal, s64 = config2
    m = 1 << 24
    X = inputs.uniform_points(1, m, 10)
    Xd = torch.from_numpy(X).to(cuda)
    out = torch.empty(m, dtype=torch.float32, device=cuda)
    g.evaluate_device(Xd, out, m)
    g.sync()
    full = out.cpu().numpy()
    del Xd, out
    assert np.all(np.isfinite(full))
    idx = np.linspace(0, m - 1, 3000).astype(np.int64)
    small = g.evaluate(X[idx])
    assert np.array_equal(full[idx].view(np.uint32), small.view(np.uint32))
    check_eval(full[idx], o.evaluate_f64(s64, X[idx]), "config 2, sample of the 2^24 launch")
    # the host-buffer call over the same points gives the same bits
    again = g.evaluate(X)
    assert np.array_equal(full.view(np.uint32), again.view(np.uint32))


@pytest.fixture(scope="module")
def config3():
    """The grid that the benchmark's refinement reaches (the same call)."""
    g, it = sg.refine(6, 4, _lib.SG_FN_BUMP, (0.3, 50.0), tol=1e-4, max_level=13, max_points=109_051_905,
                      max_iters=32)
    g.sample_function(_lib.SG_FN_BUMP, (0.3, 50.0))
    nodal = g.get_values()
    g.hierarchize()
    yield g, it, nodal
    g.close()


def test_config3_final_grid_bitexact_vs_reference(cuda, config3):
    g, it, nodal = config3
    assert it > 1 and g.n > 4
    r = reference_surpluses(6, g.n, list(g.limits), nodal, 9)
    check_structure(g, r)
    same = g.get_values().view(np.uint32) == r.values().view(np.uint32)
    assert same.all(), f"{np.count_nonzero(~same)} surpluses differ"


def test_config3_evaluate_vs_fp64(cuda, config3):
    g, it, nodal = config3
    d = 6
    o = Oracle(d, g.n, list(g.limits))
    s64 = o.hierarchize_f64(nodal.astype(np.float64))
    X = np.concatenate([inputs.uniform_points(2, 2048, d),
                        inputs.gaussian_points(2, 2048, d, 0.3, 0.1, start=1 << 40)])
    ref64 = o.evaluate_f64(s64, X)
    for ppt in (1, 2):
        g.set_option(sg.SG_OPT_EVAL_PPT, ppt)
        check_eval(g.evaluate(X), ref64, f"config 3 ppt={ppt}")
    check_grid_points(g, o, nodal, 1024, 13)
