"""Generates the golden fixtures in this directory from the REFERENCE itself.

Runs the reference benchmark's own C code (adaptive_sparse_grid_bench.c,
compiled in place by oracle/Makefile into oracle/_ref/libasgb_ref.so) and
stores, per case, what it computes: the index tables, the bijection on a
sample of indices, the nodal values its init() samples (the reference's own
fct, c:87-94, c:146-152), the surpluses of hierarchize0 (c:557), and the
outputs of evaluate0 (c:1237) at seeded query points.  The reference cannot
travel to the GPU box; these files do.

Usage (needs the reference sources or the prebuilt library):
    make -C oracle && python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from adaptive_sparse_grid_bench_b200 import inputs  # noqa: E402
from oracle.oracle import Reference  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))

# (name, d, n, limits, query seed, number of query points)
CASES = [
    ("d4n8", 4, 8, None, 0, 512),          # config 1's shape
    ("d3n5", 3, 5, None, 10, 256),
    ("d3n5_lim412", 3, 5, [4, 1, 2], 11, 256),
    ("d3n5_lim244", 3, 5, [2, 4, 4], 12, 256),
    ("d1n9", 1, 9, None, 13, 128),
    ("d2n6_lim05", 2, 6, [0, 5], 14, 128),
    ("d6n4", 6, 4, None, 15, 256),          # config 3's starting grid
    ("d10n4", 10, 4, None, 16, 128),
    ("d5n1", 5, 1, None, 17, 32),
]


def main() -> None:
    for name, d, n, lim, seed, m in CASES:
        r = Reference(d, n, lim)
        dp, lidx = r.tables()
        vals = r.values()
        sample = np.unique(np.linspace(0, r.N - 1, min(r.N, 2000)).astype(np.int64))
        lv = np.zeros((sample.size, d), np.int32)
        ix = np.zeros((sample.size, d), np.int32)
        for q, i in enumerate(sample):
            lv[q], ix[q] = r.idx2gp(int(i))
        r.hierarchize(0)
        surplus = r.values()
        X = inputs.uniform_points(seed, m, d)
        out0 = r.evaluate(X, 0)
        # grid points as query points: the reference's own correctness test
        G = np.zeros((min(r.N, 256), d), np.float32)
        for q in range(G.shape[0]):
            li, ii = r.idx2gp(int(sample[q * len(sample) // G.shape[0]]))
            G[q] = (2 * ii + 1) / (2.0 ** (li + 1))
        outg = r.evaluate(G, 0)
        np.savez_compressed(
            os.path.join(HERE, f"{name}.npz"), d=d, n=n,
            limits=np.array(lim if lim is not None else [n - 1] * d, np.int32),
            N=r.N, S=r.S, dp=dp, lidx=lidx, sample=sample, levels=lv, indices=ix,
            values=vals, surplus=surplus, X=X, out=out0, G=G, outG=outg)
        print(f"{name}: N={r.N} S={r.S}")


if __name__ == "__main__":
    main()
