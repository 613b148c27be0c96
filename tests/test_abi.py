"""CPU checks of the C ABI library: it loads, exports every function that
include/sgrid.h declares, and its host-side index algebra (no GPU needed:
sg_create touches no device) matches the golden fixtures bit-exactly."""
import ctypes as C
import os

import numpy as np
import pytest

import adaptive_sparse_grid_bench_b200 as sg
from adaptive_sparse_grid_bench_b200 import _lib
from conftest import golden_cases, load_golden


def test_library_exports_every_header_function():
    lib = sg.lib()
    declared = sg.header_functions()
    assert len(declared) >= 25
    for name in declared:
        assert hasattr(lib, name), f"{name} declared in sgrid.h but not exported"
    # the ctypes table covers the header exactly
    assert sorted(_lib.SIGNATURES) == declared
    assert lib.sg_version().startswith(b"sgb200")


def test_library_exports_nothing_else():
    path = _lib.LIB_PATH
    import subprocess
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True).stdout
    names = {line.split()[-1] for line in out.splitlines() if " T " in line}
    assert names == set(sg.header_functions())


def test_header_constants_match_bindings():
    text = open(_lib.HEADER).read()
    for name in ["SG_MAX_DIMS", "SG_MAX_LEVELS", "SG_OK", "SG_HIER_FP64", "SG_OPT_HIER_PRECISION",
                 "SG_OPT_EVAL_SORT", "SG_OPT_EVAL_PPT", "SG_OPT_HIER_KERNEL", "SG_OPT_PROFILE",
                 "SG_OPT_USE_GRAPH", "SG_OPT_SWEEP_GROUP", "SG_OPT_TEST_WAIT", "SG_OPT_EVAL_BLOCKING",
                 "SG_TUNE_TIMINGS", "SG_FN_GAUSS", "SG_FN_QUAD", "SG_NUM_PHASES"]:
        import re
        m = re.search(rf"#define {name} \(?(-?\d+)\)?", text)
        assert m, name
        assert int(m.group(1)) == getattr(_lib, name), name
    m = re.search(r"#define SG_BATCH_TUNE_TIMINGS \((\d+) \* \(SG_MAX_DIMS \+ 1\)\)", text)
    assert m and int(m.group(1)) * (_lib.SG_MAX_DIMS + 1) == _lib.SG_BATCH_TUNE_TIMINGS
    assert int(m.group(1)) == 2 * _lib.SG_EVAL_BLOCKINGS


@pytest.mark.parametrize("name", golden_cases())
def test_host_tables_and_bijection_match_golden(name):
    g = load_golden(name)
    d, n = int(g["d"]), int(g["n"])
    grid = sg.Grid(d, n, g["limits"])
    assert grid.num_points == int(g["N"]) and grid.num_subspaces == int(g["S"])
    dp, lidx = grid.tables()
    assert np.array_equal(dp, g["dp"].astype(np.int64))
    assert np.array_equal(lidx[:n], g["lidx"].astype(np.int64)) and lidx[n] == int(g["N"])
    for q, i in enumerate(g["sample"]):
        lv, ix = grid.idx2gp(int(i))
        assert np.array_equal(lv, g["levels"][q]) and np.array_equal(ix, g["indices"][q])
        assert grid.gp2idx(lv, ix) == int(i)


def test_l2idx_idx2l_roundtrip():
    grid = sg.Grid(5, 6, [5, 2, 5, 0, 3])
    dp, _ = grid.tables()
    for s in range(6):
        for pos in range(int(dp[4, s])):
            lv = grid.idx2l(pos, s)
            assert lv.sum() == s and grid.l2idx(lv) == pos
            assert all(lv <= grid.limits)


def test_subspace_order_within_group():
    """Dim 0's level varies first: (1,0,0), (0,1,0), (0,0,1) (c:245-264)."""
    grid = sg.Grid(3, 3)
    assert [list(grid.idx2l(p, 1)) for p in range(3)] == [[1, 0, 0], [0, 1, 0], [0, 0, 1]]


@pytest.mark.parametrize("d,n", [(0, 3), (3, 0), (-1, 2)])
def test_create_rejects_bad_shape(d, n):
    with pytest.raises(sg.SgError) as e:
        sg.Grid(d, n)
    assert e.value.code == _lib.SG_ERR_ARG


@pytest.mark.parametrize("d,n", [(21, 3), (3, 17)])
def test_create_rejects_unsupported_size(d, n):
    with pytest.raises(sg.SgError) as e:
        sg.Grid(d, n)
    assert e.value.code == _lib.SG_ERR_RANGE


def test_create_rejects_negative_limit():
    with pytest.raises(sg.SgError):
        sg.Grid(3, 4, [2, -1, 2])


def test_limits_clamp_to_n_minus_1():
    grid = sg.Grid(2, 4, [9, 9])
    assert list(grid.limits) == [3, 3]
    assert grid.num_points == sg.Grid(2, 4).num_points


def test_bijection_rejects_out_of_range():
    grid = sg.Grid(3, 4)
    with pytest.raises(sg.SgError):
        grid.idx2gp(grid.num_points)
    with pytest.raises(sg.SgError):
        grid.idx2gp(-1)
    with pytest.raises(sg.SgError):
        grid.gp2idx([1, 1, 2], [0, 0, 0])  # level sum 4 > n-1
    with pytest.raises(sg.SgError):
        grid.gp2idx([1, 0, 0], [2, 0, 0])  # index beyond 2^l


def test_options_validate():
    grid = sg.Grid(3, 4)
    assert grid.get_option(sg.SG_OPT_HIER_PRECISION) == sg.SG_HIER_FP32
    grid.precision = "fp64"
    assert grid.precision == "fp64"
    for opt, bad in [(sg.SG_OPT_HIER_PRECISION, 2), (sg.SG_OPT_EVAL_SORT, 3), (sg.SG_OPT_EVAL_PPT, 5),
                     (sg.SG_OPT_HIER_KERNEL, -1), (sg.SG_OPT_EVAL_BLOCKING, -1), (sg.SG_OPT_EVAL_BLOCKING, 4),
                     (99, 0)]:
        with pytest.raises(sg.SgError):
            grid.set_option(opt, bad)
    assert grid.get_option(sg.SG_OPT_EVAL_BLOCKING) == 0  # auto
    for ok in range(_lib.SG_EVAL_BLOCKINGS + 1):
        grid.set_option(sg.SG_OPT_EVAL_BLOCKING, ok)
        assert grid.get_option(sg.SG_OPT_EVAL_BLOCKING) == ok


def test_batch_sweep_group_option_validates():
    # host-only: the sweep tables are built by the batch's first device call
    b = sg.Batch([3, 10], [4, 6])
    for ok in (0, 1, 1 << 22):
        b.set_option(_lib.SG_OPT_SWEEP_GROUP, ok)
    for bad in (-1, 1 << 32):
        with pytest.raises(sg.SgError):
            b.set_option(_lib.SG_OPT_SWEEP_GROUP, bad)
    for ok in range(_lib.SG_EVAL_BLOCKINGS + 1):
        b.set_option(_lib.SG_OPT_EVAL_BLOCKING, ok)
    for bad in (-1, _lib.SG_EVAL_BLOCKINGS + 1):
        with pytest.raises(sg.SgError):
            b.set_option(_lib.SG_OPT_EVAL_BLOCKING, bad)
    b.close()


def test_calls_before_values_are_state_errors():
    grid = sg.Grid(3, 4)
    lib = sg.lib()
    assert lib.sg_hierarchize(grid.handle) == _lib.SG_ERR_STATE
    out = np.zeros(4, np.float32)
    x = np.zeros((4, 3), np.float32)
    assert lib.sg_evaluate(grid.handle, x.ctypes.data, out.ctypes.data, 4) == _lib.SG_ERR_STATE
    assert lib.sg_get_values(grid.handle, out.ctypes.data) == _lib.SG_ERR_STATE


def test_null_arguments():
    lib = sg.lib()
    v = C.c_int64()
    assert lib.sg_num_points(None, C.byref(v)) == _lib.SG_ERR_ARG
    assert lib.sg_create(3, 3, None, None) == _lib.SG_ERR_ARG
    assert lib.sg_destroy(None) == _lib.SG_OK
    assert b"NULL" in lib.sg_last_error() or lib.sg_last_error() != b""


def test_device_ops_fail_loudly_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    grid = sg.Grid(3, 4)
    with pytest.raises(sg.SgError) as e:
        grid.set_values(np.zeros(grid.num_points, np.float32))
    assert e.value.code == _lib.SG_ERR_CUDA


def test_sizes_of_the_benchmark_configs():
    """Point and subspace counts of the workload shapes (host tables only)."""
    assert (sg.Grid(4, 8).num_points, sg.Grid(4, 8).num_subspaces) == (23297, 330)
    g2 = sg.Grid(10, 10)
    assert (g2.num_points, g2.num_subspaces) == (32978945, 92378)
    g3 = sg.Grid(6, 14)
    assert (g3.num_points, g3.num_subspaces) == (109051905, 27132)
