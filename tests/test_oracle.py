"""Pins the CPU oracle (oracle/sg_oracle.c) to the reference.

Against the golden fixtures (made by the reference's own code, see
tests/golden/make_golden.py) and, where the in-place reference build is
present, against the reference live on further shapes.  Bit-exact for the
tables, the bijection, hierarchize0 and evaluate0.
"""
import numpy as np
import pytest

from conftest import golden_cases, load_golden
from oracle.oracle import Oracle, Reference


@pytest.mark.parametrize("name", golden_cases())
def test_oracle_matches_golden(name):
    g = load_golden(name)
    d, n = int(g["d"]), int(g["n"])
    o = Oracle(d, n, g["limits"])
    assert o.N == int(g["N"]) and o.S == int(g["S"])
    assert np.array_equal(o.dp, g["dp"])
    assert np.array_equal(o.lidx[:n], g["lidx"])
    for q, i in enumerate(g["sample"]):
        lv, ix = o.idx2gp(int(i))
        assert np.array_equal(lv, g["levels"][q]) and np.array_equal(ix, g["indices"][q])
        assert o.gp2idx(lv, ix) == int(i)
    h = o.hierarchize_f32(g["values"])
    assert np.array_equal(h.view(np.uint32), g["surplus"].view(np.uint32))
    e = o.evaluate_f32(g["surplus"], g["X"])
    assert np.array_equal(e.view(np.uint32), g["out"].view(np.uint32))
    # the reference's own correctness test: interpolation at grid points
    eg = o.evaluate_f32(g["surplus"], g["G"])
    assert np.array_equal(eg.view(np.uint32), g["outG"].view(np.uint32))


@pytest.mark.parametrize("name", golden_cases())
def test_golden_interpolation_property(name):
    """Evaluating the hierarchized grid at grid points gives back the sampled
    values (c:2027-2029 asserts |out - f| < 1e-6)."""
    g = load_golden(name)
    o = Oracle(int(g["d"]), int(g["n"]), g["limits"])
    idx = [o.gp2idx(*_lv_ix(x, o.d)) for x in g["G"]]
    np.testing.assert_allclose(g["outG"], g["values"][idx], rtol=0, atol=1e-6)


def _lv_ix(x, d):
    """(levels, indices) of a grid-point coordinate vector x = (2i+1)/2^(l+1)."""
    lv = np.zeros(d, np.int32)
    ix = np.zeros(d, np.int32)
    for k in range(d):
        num = int(round(x[k] * 2.0 ** 30))
        tz = (num & -num).bit_length() - 1
        lv[k] = 29 - tz           # x 2^30 = (2i+1) 2^(29-l)
        ix[k] = num >> (tz + 1)
    return lv, ix


def test_oracle_fp64_fast_equals_definition():
    o = Oracle(4, 6, [5, 3, 5, 2])
    v = np.random.default_rng(0).random(o.N)
    assert np.array_equal(o.hierarchize_f64(v, fast=True), o.hierarchize_f64(v, fast=False))


SHAPES = [(2, 7, None), (5, 5, None), (7, 4, None), (4, 6, [5, 3, 5, 2]), (4, 6, [1, 5, 0, 4]),
          (3, 8, [7, 2, 3]), (12, 3, None), (6, 5, [4, 4, 1, 0, 3, 2])]


@pytest.mark.skipif(not Reference.available(), reason="in-place reference build absent")
@pytest.mark.parametrize("d,n,lim", SHAPES)
def test_oracle_matches_reference_live(d, n, lim):
    r = Reference(d, n, lim)
    o = Oracle(d, n, lim)
    dp, lidx = r.tables()
    assert (o.N, o.S) == (r.N, r.S)
    assert np.array_equal(o.dp, dp) and np.array_equal(o.lidx[:n], lidx)
    for i in range(0, r.N, max(1, r.N // 500)):
        lv, ix = r.idx2gp(i)
        lv2, ix2 = o.idx2gp(i)
        assert np.array_equal(lv, lv2) and np.array_equal(ix, ix2)
    v = np.random.default_rng(d * 100 + n).random(r.N).astype(np.float32)
    r.set_values(v)
    r.hierarchize(0)
    ref_h = r.values()
    assert np.array_equal(o.hierarchize_f32(v).view(np.uint32), ref_h.view(np.uint32))
    X = np.random.default_rng(7).random((64, d), dtype=np.float32)
    assert np.array_equal(o.evaluate_f32(ref_h, X).view(np.uint32), r.evaluate(X, 0).view(np.uint32))


@pytest.mark.skipif(not Reference.available(), reason="in-place reference build absent")
def test_reference_variants_agree_on_regular_grid():
    """The reference's own variant cross-check (c:1798-2023) holds for the
    baselines timed here: omp_hierarchize3 and omp_evaluate5."""
    r = Reference(5, 6)
    v = r.values()
    r.hierarchize(0)
    h0 = r.values()
    r.set_values(v)
    r.hierarchize(9)
    assert np.array_equal(r.values(), h0)
    X = np.random.default_rng(3).random((1000, 5), dtype=np.float32)
    assert np.array_equal(r.evaluate(X, 7), r.evaluate(X, 0))


def test_reference_cuda_harness_refuses_unsafe_sizes():
    # every refusal happens on the host, before any CUDA call
    from oracle.oracle import ReferenceCUDA
    if not ReferenceCUDA.available():
        pytest.skip("reference CUDA harness not built (reference sources absent)")
    surplus = np.zeros(49, np.float32)  # d=2, n=4
    X = np.full((256, 2), 0.5, np.float32)
    X21 = np.full((256, 21), 0.5, np.float32)
    for args in ((2, 4, surplus, X, 33), (2, 4, surplus, X[:100], 32), (2, 11, surplus, X, 32),
                 (21, 4, surplus, X21, 32)):
        with pytest.raises(RuntimeError, match="returned -1"):
            ReferenceCUDA.evaluate5(*args)
    Y = X.copy()
    Y[3, 1] = 1.0
    with pytest.raises(RuntimeError, match="returned -1"):
        ReferenceCUDA.evaluate5(2, 4, surplus, Y, 32)
    # hierarchize7: its warp barriers need whole warps, so n < 6 is refused;
    # so are n > 10 and d > 20 (the constant tables' sizes)
    for d, n in ((2, 4), (4, 5), (2, 11), (21, 6)):
        with pytest.raises(RuntimeError, match="returned -1"):
            ReferenceCUDA.hierarchize7(d, n, np.zeros(49, np.float32))


def test_ref_cuda_patch_rules():
    # the warp-barrier patch of the reference's hierarchize7 (oracle/patch_ref_cuda.py),
    # on a stand-in text with the kernel's three hand-over shapes: each rule must match
    # exactly once inside hierarchize7, nothing outside it changes, and a missing shape
    # stops the build instead of yielding an unpatched kernel
    from oracle.patch_ref_cuda import patch
    head = "__global__ void hierarchize6(int x) { if (0 == lane)\n  --levels[crt_dim]; }\n"
    body = ("__global__ void hierarchize7(int x) {\n"
            "  if (0 == lane) { levels[crt_dim] = saved_level; }\n"
            "  for (; levels[crt_dim] >= 1; --crt_level) {\n"
            "    if (0 == lane) {\n"
            "      for (int l = d - 2; l >= 0; l--)\n"
            "        prefix_sums[l] = prefix_sums[l + 1] + levels[l];\n"
            "    }\n"
            "    work();\n"
            "    if (0 == lane)\n"
            "      --levels[crt_dim];\n"
            "  }\n}\n")
    tail = "__global__ void evaluate5(int x) { }\n"
    out = patch(head + body + tail)
    assert out.startswith(head) and out.endswith(tail)
    assert out.count("__syncwarp();") == 4
    assert "__syncwarp(); for (; levels[crt_dim] >= 1;" in out
    assert "__syncwarp(); if (0 == lane) --levels[crt_dim]; __syncwarp();" in out
    with pytest.raises(SystemExit):
        patch(head + body.replace("--levels[crt_dim];", "levels[crt_dim]--;") + tail)
