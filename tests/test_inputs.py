"""The seeded input generators (SplitMix64) and grid-point coordinates."""
import numpy as np

import adaptive_sparse_grid_bench_b200 as sg
from adaptive_sparse_grid_bench_b200 import inputs
from oracle.oracle import Oracle


def test_splitmix64_known_answers():
    # SplitMix64 with state 0: the published first outputs of the generator
    z = inputs.splitmix64(0, 0, 3)
    assert [int(v) for v in z] == [0xE220A8397B1DCDAF, 0x6E789E6AA1B965F4, 0x06C45D188009454F]


def test_uniform_is_24_bit_and_in_range():
    u = inputs.uniform01(1, 100000)
    assert u.dtype == np.float32 and u.min() >= 0 and u.max() < 1
    assert np.all((u * 16777216.0) == np.floor(u * 16777216.0))


def test_streams_are_counter_based():
    a = inputs.uniform01(7, 1000)
    b = inputs.uniform01(7, 500, start=500)
    assert np.array_equal(a[500:], b)
    assert not np.array_equal(inputs.uniform01(8, 1000), a)


def test_gaussian_points_clipped():
    x = inputs.gaussian_points(2, 10000, 6, 0.3, 0.1)
    assert x.min() >= 0 and x.max() < 1
    assert abs(float(x.mean()) - 0.3) < 0.01


def test_grid_coordinates_match_oracle():
    for d, n, lim in [(4, 6, None), (3, 7, [6, 1, 3])]:
        g = sg.Grid(d, n, lim)
        assert np.array_equal(inputs.grid_coordinates(g), Oracle(d, n, lim).grid_points())


def test_functions():
    X = np.array([[0.5, 0.5], [0.25, 0.75]])
    assert np.allclose(inputs.f_prod4(X), [1.0, 0.75 * 0.75])
    assert np.allclose(inputs.f_gauss(X), np.exp(-np.sum(X * X, axis=1)))
    assert np.allclose(inputs.f_reference(X), np.sum(X * X * (1 - X) ** 2, axis=1))
    coef = np.array([[1.0, 2.0, 3.0], [0.5, 0.0, -1.0]])
    assert np.allclose(inputs.f_quad(X, coef), np.prod(coef[:, 0] + coef[:, 1] * X + coef[:, 2] * X * X, axis=1))
