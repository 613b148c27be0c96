"""Seeded synthetic inputs for the sparse-grid workloads.

The reference draws query points as random grid points with ``random()``
(adaptive_sparse_grid_bench.c:1724-1736, _cuda.cu:152-165) and samples
f = sum x^2 (1-x)^2 (c:87-94).  Here every input is reproducible from a seed
with one counter-based generator, SplitMix64: element i of stream `seed` is
mix(seed + (i+1) * 0x9E3779B97F4A7C15), and a uniform float in [0, 1) takes
its top 24 bits, (z >> 40) * 2^-24.  The same definition is used by every
test, the benchmark and the fixtures.

Test functions are evaluated in float64 at the float32 grid coordinates and
rounded once to float32.
"""
from __future__ import annotations

import numpy as np

GAMMA = np.uint64(0x9E3779B97F4A7C15)
M1 = np.uint64(0xBF58476D1CE4E5B9)
M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, start: int, count: int) -> np.ndarray:
    """Raw 64-bit outputs start..start+count-1 of stream `seed`."""
    with np.errstate(over="ignore"):
        i = np.arange(start + 1, start + count + 1, dtype=np.uint64)
        z = np.uint64(seed) + i * GAMMA
        z = (z ^ (z >> np.uint64(30))) * M1
        z = (z ^ (z >> np.uint64(27))) * M2
        return z ^ (z >> np.uint64(31))


def uniform01(seed: int, count: int, start: int = 0) -> np.ndarray:
    """float32 in [0, 1) with 24 random bits each."""
    z = splitmix64(seed, start, count)
    return ((z >> np.uint64(40)).astype(np.float64) * (1.0 / 16777216.0)).astype(np.float32)


def uniform_points(seed: int, num: int, d: int) -> np.ndarray:
    """num x d query points, i.i.d. uniform on [0,1)^d (row-major stream)."""
    return uniform01(seed, num * d).reshape(num, d)


def gaussian_points(seed: int, num: int, d: int, mu: float, sigma: float, start: int = 0) -> np.ndarray:
    """num x d points N(mu, sigma^2) per coordinate via Box-Muller, clipped to
    [0, 1) (largest float below 1 at the top)."""
    u = uniform01(seed, 2 * num * d, start).astype(np.float64).reshape(-1, 2)
    u1 = np.maximum(u[:, 0], 2.0 ** -25)
    z = np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u[:, 1])
    x = np.clip(mu + sigma * z, 0.0, np.nextafter(np.float32(1.0), np.float32(0.0)))
    return x.astype(np.float32).reshape(num, d)


# ---- test functions (float64 in, float64 out) ------------------------------

def f_reference(X: np.ndarray) -> np.ndarray:
    """The reference's fct: sum_k x^2 (1-x)^2 (c:87-94)."""
    X = np.asarray(X, np.float64)
    return np.sum(X * X * (1 - X) * (1 - X), axis=-1)


def f_prod4(X: np.ndarray) -> np.ndarray:
    """prod_k 4 x_k (1 - x_k)."""
    X = np.asarray(X, np.float64)
    return np.prod(4.0 * X * (1.0 - X), axis=-1)


def f_gauss(X: np.ndarray) -> np.ndarray:
    """exp(-sum_k x_k^2)."""
    X = np.asarray(X, np.float64)
    return np.exp(-np.sum(X * X, axis=-1))


def f_bump(X: np.ndarray, c: float = 0.3, a: float = 50.0) -> np.ndarray:
    """exp(-a sum_k (x_k - c)^2): a localized Gaussian bump."""
    X = np.asarray(X, np.float64)
    return np.exp(-a * np.sum((X - c) ** 2, axis=-1))


def f_quad(X: np.ndarray, coef: np.ndarray) -> np.ndarray:
    """prod_k (a_k + b_k x_k + c_k x_k^2), coef shape (d, 3)."""
    X = np.asarray(X, np.float64)
    a, b, c = coef[:, 0], coef[:, 1], coef[:, 2]
    return np.prod(a + b * X + c * X * X, axis=-1)


FUNCTIONS = {"reference": f_reference, "prod4": f_prod4, "gauss": f_gauss, "bump": f_bump}


def grid_coordinates(grid, subspaces=None) -> np.ndarray:
    """Coordinates of every grid point in compact order, (N, d) float32.

    Built one subspace at a time: the points of subspace l are the tensor
    product of x_k = (2 i_k + 1) / 2^(l_k+1), row-major with dim 0 most
    significant (c:146-152, c:191-193)."""
    if subspaces is None:
        subspaces = grid.subspaces()
    d = grid.d
    out = np.empty((grid.num_points, d), np.float32)
    r = 0
    for lv in subspaces:
        axes = [((2 * np.arange(1 << int(l)) + 1) / float(1 << (int(l) + 1))).astype(np.float32) for l in lv]
        mesh = np.meshgrid(*axes, indexing="ij")
        m = mesh[0].size
        out[r:r + m] = np.stack([g.reshape(-1) for g in mesh], axis=1)
        r += m
    assert r == grid.num_points
    return out


def grid_values(grid, fn, subspaces=None, chunk: int = 1 << 22) -> np.ndarray:
    """f at every grid point, float64 arithmetic rounded once to float32."""
    X = grid_coordinates(grid, subspaces)
    out = np.empty(X.shape[0], np.float32)
    for s in range(0, X.shape[0], chunk):
        out[s:s + chunk] = fn(X[s:s + chunk]).astype(np.float32)
    return out


def regular_grid_size(d: int, n: int) -> tuple[int, int]:
    """(points, subspaces) of the regular grid: sum over level sums s < n of
    C(s+d-1, d-1) subspaces of 2^s points."""
    from math import comb
    pts = sum(comb(s + d - 1, d - 1) << s for s in range(n))
    return pts, comb(n - 1 + d, d)


def batch_workload(seed: int, num_grids: int, max_points: int = 2_000_000, d_range=(2, 12), n_range=(3, 9),
                   pts_range=(256, 65536)):
    """The batched workload: per grid d and n uniform in the ranges,
    resampled until the grid has <= max_points points; coefficients
    (a_k, b_k, c_k) ~ U(-1,1) of f = prod_k (a_k + b_k x_k + c_k x_k^2); a
    log-uniform number of query points.  Returns dims, levels, coefficient
    array (num_grids, 3*max_d) and query counts."""
    dims, levels, counts = [], [], []
    coef = np.zeros((num_grids, 3 * d_range[1]), np.float64)
    draw = 0
    for g in range(num_grids):
        while True:
            u = uniform01(seed, 2, start=draw).astype(np.float64)
            draw += 2
            d = d_range[0] + int(u[0] * (d_range[1] - d_range[0] + 1))
            n = n_range[0] + int(u[1] * (n_range[1] - n_range[0] + 1))
            if regular_grid_size(d, n)[0] <= max_points:
                break
        c = uniform01(seed + 1000, 3 * d, start=3 * d_range[1] * g).astype(np.float64) * 2 - 1
        coef[g, :3 * d] = c
        lu = uniform01(seed + 2000, 1, start=g).astype(np.float64)[0]
        m = int(round(np.exp(np.log(pts_range[0]) + lu * (np.log(pts_range[1]) - np.log(pts_range[0])))))
        dims.append(d)
        levels.append(n)
        counts.append(m)
    return np.array(dims, np.int32), np.array(levels, np.int32), coef, np.array(counts, np.int64)
