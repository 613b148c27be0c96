"""Seeded inputs of the benchmark workloads for the CPU checkers and the
reference arm (TEST INFRASTRUCTURE ONLY).

The same definitions as the library's own input generator: SplitMix64 with
element i of stream `seed` = mix(seed + (i+1) * 0x9E3779B97F4A7C15), a
uniform float in [0, 1) from the top 24 bits, test functions in float64
rounded once to float32.  Kept here, beside the oracle, so that the
reference arm of the benchmark builds its inputs without loading the product
library; a CPU test checks that both generators give the same bits.
"""
from __future__ import annotations

import numpy as np

_GAMMA = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def uniform01(seed: int, count: int, start: int = 0) -> np.ndarray:
    """float32 in [0, 1): outputs start..start+count-1 of stream `seed`."""
    with np.errstate(over="ignore"):
        i = np.arange(start + 1, start + count + 1, dtype=np.uint64)
        z = np.uint64(seed) + i * _GAMMA
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    return ((z >> np.uint64(40)).astype(np.float64) * (1.0 / 16777216.0)).astype(np.float32)


def uniform_points(seed: int, num: int, d: int) -> np.ndarray:
    """num x d points i.i.d. uniform on [0,1)^d (row-major stream)."""
    return uniform01(seed, num * d).reshape(num, d)


def f_gauss(X: np.ndarray) -> np.ndarray:
    """exp(-sum_k x_k^2) in float64."""
    X = np.asarray(X, np.float64)
    return np.exp(-np.sum(X * X, axis=-1))


def grid_values(oracle, fn, chunk: int = 1 << 22) -> np.ndarray:
    """fn at every grid point of the oracle's layout (compact order, the
    coordinates (2i+1)/2^(l+1) of c:146-152), rounded once to float32."""
    X = oracle.grid_points()
    out = np.empty(X.shape[0], np.float32)
    for s in range(0, X.shape[0], chunk):
        out[s:s + chunk] = fn(X[s:s + chunk]).astype(np.float32)
    return out
